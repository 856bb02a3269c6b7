// gxy_table.cu -- PosTable::build (src/pos_table.rs:35-83) on the device, for
// one view of a sequence or for many views at once (the driver's chunk
// tables, src/driver.rs:156-210).
//
// The reference counts every seedable window's word, scans the counts into
// bucket starts and drops the positions into their buckets in ascending order
// through per-word cursors (src/pos_table.rs:42-75).  Here the views share
// one bucket space, view v's word w being bucket g = v * 4^w + w:
//
//  1. k_count_words counts the windows of every bucket (atomics on an array
//     that stays in L2 for a chromosome-sized view);
//  2. one exclusive scan turns the counts into global bucket starts, and
//     leaves a copy in the counts array: the cursors;
//  3. k_fill_buckets drops every window's position into its bucket through
//     an atomic cursor -- in an arbitrary order inside the bucket;
//  4. k_sort_small_buckets writes the occupancy bitmap and orders every
//     bucket of 2 or 3 positions on the spot, k_sort_warp_buckets those up to
//     32 a warp each, k_sort_block_buckets those up to kBlockBucket in shared
//     memory, and the radix sort the few larger ones, so every bucket holds
//     the reference's order when the build returns.
//
// View v's table is a window onto the shared arrays: its starts are the
// global starts g = v * 4^w .. v * 4^w + 4^w (global indices into the shared
// positions array, which the searches use as they are; the download
// subtracts the view's first index), and its occupancy bitmap is the shared
// bitmap's words from v * 4^w / 32 on.  One count, one scan, one fill and one
// sort serve all the views.
#include "gxy_engine.cuh"
#include "gxy_kernels.cuh"

#include <vector>

namespace gxy {

namespace {

constexpr uint32_t kBlockBucket = 4096;   // the largest bucket sorted in shared memory

// Each thread takes four windows at a time (stride apart, so a warp's loads
// stay coalesced): four independent word loads and atomics in flight instead
// of one dependent chain per window.
__global__ void k_count_words(SeqView view, Pattern pat, uint32_t step, uint32_t nwin, uint32_t* counts) {
    const uint32_t S = gridDim.x * blockDim.x;
    for (uint32_t k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 < nwin; k0 += 4 * S) {
        uint32_t w[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint32_t k = k0 + u * S;
            ok[u] = k < nwin && word_at(view, pat, k * step, w[u]);
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (ok[u]) atomicAdd(&counts[w[u]], 1u);
    }
}

__global__ void k_fill_buckets(SeqView view, Pattern pat, uint32_t step, uint32_t nwin, uint32_t* cursor,
                               uint32_t* positions) {
    const uint32_t S = gridDim.x * blockDim.x;
    for (uint32_t k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 < nwin; k0 += 4 * S) {
        uint32_t w[4], slot[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint32_t k = k0 + u * S;
            ok[u] = k < nwin && word_at(view, pat, k * step, w[u]);
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (ok[u]) slot[u] = atomicAdd(&cursor[w[u]], 1u);
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (ok[u]) positions[slot[u]] = (k0 + u * S) * step;
    }
}

__device__ __forceinline__ void cswap(uint32_t& x, uint32_t& y) {
    const uint32_t lo = min(x, y), hi = max(x, y);
    x = lo;
    y = hi;
}

// Files bucket g (first index b, n positions) for the sort that fits it.
__device__ __forceinline__ void order_bucket(uint32_t* __restrict__ pos, uint32_t b, uint32_t n, uint2* mid,
                                             uint32_t* n_mid, uint2* big, uint32_t* n_big, uint2* huge,
                                             uint32_t* n_huge) {
    if (n <= 1) return;
    if (n > 3) {
        if (n > kBlockBucket) huge[atomicAdd(n_huge, 1u)] = make_uint2(b, n);
        else if (n > 32) big[atomicAdd(n_big, 1u)] = make_uint2(b, n);
        else mid[atomicAdd(n_mid, 1u)] = make_uint2(b, n);
        return;
    }
    uint32_t x = pos[b], y = pos[b + 1];
    if (n == 2) {
        if (x > y) {
            pos[b] = y;
            pos[b + 1] = x;
        }
        return;
    }
    uint32_t z = pos[b + 2];
    cswap(x, y);
    cswap(y, z);
    cswap(x, y);
    pos[b] = x;
    pos[b + 1] = y;
    pos[b + 2] = z;
}

// One pass over the bucket starts, four buckets a thread (one 16-byte load;
// the fifth start comes from the next lane): each group of eight lanes
// assembles one 32-bucket occupancy word; buckets of 2 or 3 positions --
// nearly all the buckets that need it at chromosome scale -- are put in
// order on the spot, larger ones listed for the warp sort (mid, <= 32), the
// block sort (big, <= kBlockBucket) or the radix sort (huge), as (first
// index, size) pairs.  The lists hold every such bucket: at most n / 4 + 1,
// n / 33 + 1 and n / (kBlockBucket + 1) + 1 of them for n positions.
__global__ void k_sort_small_buckets(const uint32_t* __restrict__ starts, uint64_t nb, uint32_t* __restrict__ pos,
                                     uint32_t* __restrict__ occ, uint2* __restrict__ mid, uint32_t* n_mid,
                                     uint2* __restrict__ big, uint32_t* n_big, uint2* __restrict__ huge,
                                     uint32_t* n_huge) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nb128 = (nb + 127) & ~(uint64_t)127;   // whole warps: every lane reaches the shuffles
    for (uint64_t g0 = 4 * (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x); g0 < nb128;
         g0 += 4 * (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s[4] = {0, 0, 0, 0};
        if (g0 + 3 < nb) {
            const uint4 v = *reinterpret_cast<const uint4*>(starts + g0);
            s[0] = v.x;
            s[1] = v.y;
            s[2] = v.z;
            s[3] = v.w;
        } else {
            // starts has nb + 1 entries: the next lane's first may be starts[nb].
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (g0 + k <= nb) s[k] = starts[g0 + k];
        }
        uint32_t next = __shfl_down_sync(kFull, s[0], 1);
        if (lane == 31 && g0 + 4 <= nb) next = starts[g0 + 4];
        uint32_t n[4], nib = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t e = k < 3 ? s[k + 1] : next;
            n[k] = g0 + k < nb ? e - s[k] : 0u;
            nib |= (n[k] != 0 ? 1u : 0u) << k;
        }
        // Eight lanes cover 32 buckets: OR their nibbles into one word.
        uint32_t word = nib << (4 * (lane & 7));
        word |= __shfl_xor_sync(kFull, word, 1);
        word |= __shfl_xor_sync(kFull, word, 2);
        word |= __shfl_xor_sync(kFull, word, 4);
        if ((lane & 7) == 0 && g0 < nb) occ[g0 >> 5] = word;
#pragma unroll
        for (int k = 0; k < 4; k++) order_bucket(pos, s[k], n[k], mid, n_mid, big, n_big, huge, n_huge);
    }
}

// Listed buckets of 4..32 positions, a warp each: a bitonic sort across the
// lanes by shuffles.
__global__ void k_sort_warp_buckets(const uint2* __restrict__ mid, const uint32_t* n_mid, uint32_t* __restrict__ pos) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nl = *n_mid;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t e = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < nl; e += warps) {
        const uint32_t b = mid[e].x, n = mid[e].y;
        uint32_t x = lane < n ? pos[b + lane] : 0xffffffffu;
#pragma unroll
        for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                const uint32_t y = __shfl_xor_sync(kFull, x, j);
                const bool up = (lane & k) == 0;
                const bool low = (lane & j) == 0;
                // the lower lane of a pair keeps the smaller in an ascending run
                x = (low == up) ? min(x, y) : max(x, y);
            }
        }
        if (lane < n) pos[b + lane] = x;
    }
}

// Bitonic sort of listed buckets (33 .. kBlockBucket positions) in shared
// memory, a block each.
__global__ __launch_bounds__(256) void k_sort_block_buckets(const uint2* __restrict__ big, const uint32_t* n_big,
                                                             uint32_t* __restrict__ pos) {
    __shared__ uint32_t s[kBlockBucket];
    const uint32_t nl = *n_big;
    for (uint32_t e = blockIdx.x; e < nl; e += gridDim.x) {
        const uint32_t b = big[e].x, n = big[e].y;
        uint32_t m = 1;
        while (m < n) m <<= 1;
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) s[i] = i < n ? pos[b + i] : 0xffffffffu;
        __syncthreads();
        for (uint32_t k = 2; k <= m; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                    const uint32_t l = i ^ j;
                    if (l > i) {
                        const uint32_t x = s[i], y = s[l];
                        const bool up = (i & k) == 0;
                        if (up ? x > y : x < y) {
                            s[i] = y;
                            s[l] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) pos[b + i] = s[i];
        __syncthreads();
    }
}

// first[v] = global start of view v's buckets; first[n] = all positions.
__global__ void k_view_firsts(const uint32_t* __restrict__ starts, uint64_t nw, uint32_t n_views, uint32_t* first) {
    for (uint32_t v = threadIdx.x; v <= n_views; v += blockDim.x) first[v] = starts[(uint64_t)v * nw];
}

// ilv[j] = word first + j's codes (low, high half), valid and mask bits.
__global__ void k_interleave(const uint64_t* __restrict__ codes, const uint32_t* __restrict__ valid,
                             const uint32_t* __restrict__ mask, uint64_t first, uint64_t n, uint4* __restrict__ ilv) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = codes[first + j];
        ilv[j] = make_uint4((uint32_t)c, (uint32_t)(c >> 32), valid[first + j], mask[first + j]);
    }
}

}  // namespace

void table_init() {}

void launch_interleave(const uint64_t* codes, const uint32_t* valid, const uint32_t* mask, uint64_t first, uint64_t n,
                       uint4* ilv, cudaStream_t st) {
    if (!n) return;
    count_launch();
    k_interleave<<<(int)std::min<uint64_t>((n + 255) / 256, 148 * 16), 256, 0, st>>>(codes, valid, mask, first, n, ilv);
}

gxy_status atomic_build_views(const gxy_dseq* seq, uint32_t n_views, const uint64_t* lo, const uint64_t* hi,
                              const Pattern& pat, uint32_t step, uint32_t* starts, uint32_t* positions,
                              uint32_t* occ, uint32_t* first_host, Worker* W) {
    cudaStream_t st = W->st;
    const uint64_t nw = 1ull << (2 * pat.weight);
    const uint64_t G = (uint64_t)n_views * nw;
    if (n_views == 0 || (n_views > 1 && nw < 32)) {
        set_error("a multi-view build needs at least 32 buckets per view");
        return GXY_EUNSUPPORTED;
    }
    uint64_t total = 0;
    std::vector<uint32_t> nwin(n_views);
    for (uint32_t v = 0; v < n_views; v++) {
        nwin[v] = n_windows(hi[v] - lo[v], pat.len, step);
        total += nwin[v];
    }
    if (total >= (1ull << 32)) {
        set_error("more than 2^32 windows in one table build");
        return GXY_EUNSUPPORTED;
    }
    const uint64_t n_mid_cap = total / 4 + 1, n_big_cap = total / 33 + 1,
                   n_huge_cap = total / (kBlockBucket + 1) + 1;
    GXY_CK(W->tk0.ensure((G + 1) * 4));
    GXY_CK(W->tv0.ensure((n_mid_cap + n_big_cap + n_huge_cap) * 8));
    GXY_CK(W->tv1.ensure(64 + ((size_t)n_views + 1) * 4));
    uint32_t* counts = W->tk0.as<uint32_t>();
    uint2* mid = W->tv0.as<uint2>();
    uint2* big = mid + n_mid_cap;
    uint2* huge = big + n_big_cap;
    uint32_t* ctr = W->tv1.as<uint32_t>();   // [0] big buckets, [1] huge buckets, [2] mid buckets
    uint32_t* first = ctr + 16;
    GXY_CK(cudaMemsetAsync(counts, 0, (G + 1) * 4, st));
    GXY_CK(cudaMemsetAsync(ctr, 0, 12, st));
    std::vector<SeqView> views(n_views);
    for (uint32_t v = 0; v < n_views; v++) views[v] = view_of(seq, lo[v], hi[v]);
    const int cblocks = 148 * 16;
    for (uint32_t v = 0; v < n_views; v++) {
        if (!nwin[v]) continue;
        count_launch();
        k_count_words<<<(int)std::min<uint64_t>((nwin[v] + 255) / 256, cblocks), 256, 0, st>>>(
            views[v], pat, step, nwin[v], counts + (uint64_t)v * nw);
    }
    // Global starts, and their copy back in counts: the fill's cursors (a
    // fill that decremented the counts and read the start instead measured
    // 169 us against 96 us: one more random load per window).
    scan_u32(counts, starts, nullptr, G, G, true, nullptr, W->ps, st, counts);
    for (uint32_t v = 0; v < n_views; v++) {
        if (!nwin[v]) continue;
        count_launch();
        k_fill_buckets<<<(int)std::min<uint64_t>((nwin[v] + 255) / 256, cblocks), 256, 0, st>>>(
            views[v], pat, step, nwin[v], counts + (uint64_t)v * nw, positions);
    }
    count_launch(4);
    k_sort_small_buckets<<<148 * 16, 256, 0, st>>>(starts, G, positions, occ, mid, ctr + 2, big, ctr, huge, ctr + 1);
    k_sort_warp_buckets<<<148 * 4, 256, 0, st>>>(mid, ctr + 2, positions);
    k_sort_block_buckets<<<148 * 2, 256, 0, st>>>(big, ctr, positions);
    k_view_firsts<<<1, 256, 0, st>>>(starts, nw, n_views, first);
    GXY_CK(cudaGetLastError());
    std::vector<uint32_t> h(16 + (size_t)n_views + 1);
    GXY_CK(cudaMemcpyAsync(h.data(), ctr, h.size() * 4, cudaMemcpyDeviceToHost, st));
    GXY_CK(cudaStreamSynchronize(st));
    const uint32_t n_huge = h[1];
    if (n_huge) {
        // Buckets past kBlockBucket (long repeats): the radix sort, one at a time.
        std::vector<uint2> hb(n_huge);
        GXY_CK(cudaMemcpyAsync(hb.data(), huge, (size_t)n_huge * 8, cudaMemcpyDeviceToHost, st));
        GXY_CK(cudaStreamSynchronize(st));
        int bits = 1;
        uint64_t span = 0;
        for (uint32_t v = 0; v < n_views; v++) span = std::max<uint64_t>(span, hi[v] - lo[v]);
        while (bits < 32 && (1ull << bits) < span) bits++;
        RadixPass passes[8];
        const int np = plan_radix(0, bits, 0, 0, passes, 8);
        for (const uint2& e : hb) {
            GXY_CK(W->tk1.ensure((size_t)e.y * 4));
            GXY_CK(W->tv0.ensure((size_t)e.y * 4));
            GXY_CK(W->tk0.ensure((size_t)e.y * 4));
            const int which = radix_sort_u32(positions + e.x, W->tv0.as<uint32_t>(), W->tk1.as<uint32_t>(),
                                             W->tk0.as<uint32_t>(), nullptr, e.y, e.y, passes, np, W->ps, st);
            if (which)
                GXY_CK(cudaMemcpyAsync(positions + e.x, W->tk1.p, (size_t)e.y * 4, cudaMemcpyDeviceToDevice, st));
        }
        GXY_CK(cudaStreamSynchronize(st));
        GXY_CK(cudaGetLastError());
    }
    if (first_host) memcpy(first_host, h.data() + 16, ((size_t)n_views + 1) * 4);
    return GXY_OK;
}

}  // namespace gxy
