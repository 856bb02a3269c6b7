// gxy_prims.cu -- fixed-grid scan and stable LSD radix sort (see gxy_prims.cuh).
#include "gxy_prims.cuh"

#include <algorithm>

#include "gxy_device.cuh"
#include "gxy_radix.cuh"

namespace gxy {

namespace {

template <typename T>
__global__ __launch_bounds__(kScanThreads) void k_scan_reduce(const T* in, const uint32_t* n_dev,
                                                               uint64_t n_host, uint64_t n_cap,
                                                               uint32_t* block_sums) {
    const uint64_t n = read_n(n_dev, n_host, n_cap);
    uint64_t beg, end;
    block_range(n, (uint64_t)kScanThreads * kScanItems, beg, end);
    uint32_t s = 0;
    if (sizeof(T) == 4 && (reinterpret_cast<uintptr_t>(in) & 15u) == 0) {
        // 16-byte loads: the block's range starts on a tile (4096 items) boundary.
        const uint64_t nv = (end - beg) / 4;
        const uint4* v4 = reinterpret_cast<const uint4*>(in + beg);
        for (uint64_t i = threadIdx.x; i < nv; i += kScanThreads) {
            const uint4 x = v4[i];
            s += x.x + x.y + x.z + x.w;
        }
        for (uint64_t i = beg + nv * 4 + threadIdx.x; i < end; i += kScanThreads) s += (uint32_t)in[i];
    } else {
        for (uint64_t i = beg + threadIdx.x; i < end; i += kScanThreads) s += (uint32_t)in[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    __shared__ uint32_t s_w[kScanThreads / 32];
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < kScanThreads / 32; i++) t += s_w[i];
        block_sums[blockIdx.x] = t;
    }
}

// Single-block exclusive scan of a short array in place (the block sums of a
// scan); a[n] = total.  Each
// warp owns a contiguous run of 256-element chunks; a lane holds 8
// consecutive elements (two 16-byte loads when a is 16-byte aligned), so
// every warp access is one contiguous kilobyte.
__global__ __launch_bounds__(1024) void k_scan_small(uint32_t* a, int n) {
    __shared__ uint32_t s_w[33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool vec = (reinterpret_cast<uintptr_t>(a) & 15u) == 0;
    const int nch = (n + 255) / 256;
    const int per = (nch + 31) / 32;
    const int beg = min(n, w * per * 256), end = min(n, beg + per * 256);
    auto load8 = [&](int i, uint32_t (&v)[8]) {
        if (vec && i + 8 <= end) {
            const uint4 x = *reinterpret_cast<const uint4*>(a + i);
            const uint4 y = *reinterpret_cast<const uint4*>(a + i + 4);
            v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
            v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
        } else {
#pragma unroll
            for (int k = 0; k < 8; k++) v[k] = i + k < end ? a[i + k] : 0u;
        }
    };
    uint32_t s = 0;
    for (int i = beg + lane * 8; i < end; i += 256) {
        uint32_t v[8];
        load8(i, v);
#pragma unroll
        for (int k = 0; k < 8; k++) s += v[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0) s_w[w] = s;
    __syncthreads();
    if (w == 0) {
        const uint32_t x = s_w[lane];
        uint32_t incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        s_w[lane] = incl - x;
        if (lane == 31) s_w[32] = incl;
    }
    __syncthreads();
    uint32_t carry = s_w[w];
    for (int c = beg; c < end; c += 256) {
        const int i = c + lane * 8;
        uint32_t v[8];
        load8(i, v);
        uint32_t t = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) t += v[k];
        uint32_t incl = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        uint32_t run = carry + incl - t;
        if (vec && i + 8 <= end) {
            uint32_t o8[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                o8[k] = run;
                run += v[k];
            }
            *reinterpret_cast<uint4*>(a + i) = make_uint4(o8[0], o8[1], o8[2], o8[3]);
            *reinterpret_cast<uint4*>(a + i + 4) = make_uint4(o8[4], o8[5], o8[6], o8[7]);
        } else {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                if (i + k < end) a[i + k] = run;
                run += v[k];
            }
        }
        carry += __shfl_sync(kFull, incl, 31);
    }
    if (threadIdx.x == 0) a[n] = s_w[32];
}

template <typename T>
__global__ __launch_bounds__(kScanThreads) void k_scan_down(const T* in, uint32_t* out, const uint32_t* n_dev,
                                                             uint64_t n_host, uint64_t n_cap,
                                                             const uint32_t* block_sums,
                                                             int write_total_at_n, uint32_t* total,
                                                             uint32_t* out2) {
    const uint64_t n = read_n(n_dev, n_host, n_cap);
    uint64_t beg, end;
    block_range(n, (uint64_t)kScanThreads * kScanItems, beg, end);
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_total;
    uint32_t carry = block_sums[blockIdx.x];
    static_assert(kScanItems == 8, "the 16-byte path moves 8 items per thread");
    const bool vec = sizeof(T) == 4 &&
                     ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out) |
                       reinterpret_cast<uintptr_t>(out2)) & 15u) == 0;
    for (uint64_t base = beg; base < end; base += (uint64_t)kScanThreads * kScanItems) {
        // Each thread takes kScanItems consecutive items (two 16-byte loads
        // and stores when aligned and whole).
        const uint64_t i0 = base + (uint64_t)threadIdx.x * kScanItems;
        const bool whole = vec && i0 + kScanItems <= end;
        uint32_t v[kScanItems];
        uint32_t s = 0;
        if (whole) {
            const uint4 x = *reinterpret_cast<const uint4*>(in + i0);
            const uint4 y = *reinterpret_cast<const uint4*>(in + i0 + 4);
            v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
            v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
#pragma unroll
            for (int k = 0; k < kScanItems; k++) s += v[k];
        } else {
#pragma unroll
            for (int k = 0; k < kScanItems; k++) {
                v[k] = (i0 + k < end) ? (uint32_t)in[i0 + k] : 0u;
                s += v[k];
            }
        }
        uint32_t ex = block_excl_scan<kScanThreads>(s, s_warp, &s_total) + carry;
        if (whole) {
            uint32_t o[kScanItems];
#pragma unroll
            for (int k = 0; k < kScanItems; k++) {
                o[k] = ex;
                ex += v[k];
            }
            *reinterpret_cast<uint4*>(out + i0) = make_uint4(o[0], o[1], o[2], o[3]);
            *reinterpret_cast<uint4*>(out + i0 + 4) = make_uint4(o[4], o[5], o[6], o[7]);
            if (out2) {
                *reinterpret_cast<uint4*>(out2 + i0) = make_uint4(o[0], o[1], o[2], o[3]);
                *reinterpret_cast<uint4*>(out2 + i0 + 4) = make_uint4(o[4], o[5], o[6], o[7]);
            }
        } else {
#pragma unroll
            for (int k = 0; k < kScanItems; k++) {
                if (i0 + k < end) {
                    out[i0 + k] = ex;
                    if (out2) out2[i0 + k] = ex;
                }
                ex += v[k];
            }
        }
        carry += s_total;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        const uint32_t t = block_sums[gridDim.x];   // total from k_scan_small
        if (write_total_at_n) out[n] = t;
        if (total) *total = t;
    }
}

template <typename T>
void scan_impl(const T* in, uint32_t* out, const uint32_t* n_dev, uint64_t n_host, uint64_t n_cap,
               bool write_total_at_n, uint32_t* total, const PrimScratch& ps, cudaStream_t st,
               uint32_t* out2 = nullptr) {
    // Blocks: enough for every block to own about two tiles at capacity, up
    // to the larger of the scratch's two grids (its block_sums hold that many).
    const uint64_t tile = (uint64_t)kScanThreads * kScanItems;
    const int cap_grid = std::max(ps.grid, ps.sort_grid_max);
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((n_cap + 2 * tile - 1) / (2 * tile),
                                                                 (uint64_t)cap_grid));
    count_launch();
    k_scan_reduce<T><<<grid, kScanThreads, 0, st>>>(in, n_dev, n_host, n_cap, ps.block_sums);
    count_launch();
    k_scan_small<<<1, 1024, 0, st>>>(ps.block_sums, grid);
    count_launch();
    k_scan_down<T><<<grid, kScanThreads, 0, st>>>(in, out, n_dev, n_host, n_cap, ps.block_sums,
                                                   write_total_at_n ? 1 : 0, total, out2);
}

template <typename K>
void radix_attr() {
    cudaFuncSetAttribute(k_radix_scatter<K, ArraySrc<K>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(SortSmem<K>));
}

template <typename K>
int radix_impl(K* ka, uint32_t* va, K* kb, uint32_t* vb, const uint32_t* n_dev, uint64_t n_host, uint64_t n_cap,
               const RadixPass* passes, int npass, const PrimScratch& ps, cudaStream_t st) {
    const size_t smem = sizeof(SortSmem<K>);
    // Blocks: enough for every block to own about two tiles at capacity, so
    // that large sorts fill the GPU and small ones keep their per-digit
    // histogram scans (grid entries each) short.
    const uint64_t want = (n_cap + 2 * (uint64_t)kSortTile - 1) / (2 * (uint64_t)kSortTile);
    const int cap_grid = ps.sort_grid_max > 0 ? ps.sort_grid_max : ps.grid;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)cap_grid));
    K* kin = ka;
    uint32_t* vin = va;
    K* kout = kb;
    uint32_t* vout = vb;
    for (int p = 0; p < npass; p++) {
        const int radix = 1 << passes[p].bits;
        count_launch();
        k_radix_hist<K><<<grid, kSortThreads, 0, st>>>(ArraySrc<K>{kin, vin}, n_dev, n_host, n_cap, passes[p].shift,
                                                       passes[p].bits, ps.hist);
        count_launch();
        k_radix_digit_scan<<<radix, 256, 0, st>>>(ps.hist, grid, ps.block_sums);
        count_launch();
        k_radix_scatter<K><<<grid, kSortThreads, smem, st>>>(ArraySrc<K>{kin, vin}, kout, vout, n_dev, n_host,
                                                             n_cap, passes[p].shift, passes[p].bits, ps.hist,
                                                             ps.block_sums);
        K* tk = kin; kin = kout; kout = tk;
        uint32_t* tv = vin; vin = vout; vout = tv;
    }
    return (npass & 1) ? 1 : 0;
}

}  // namespace

void prims_init() {
    radix_attr<uint32_t>();
    radix_attr<uint64_t>();
}

void scan_u32(const uint32_t* in, uint32_t* out, const uint32_t* n_dev, uint64_t n_host, uint64_t n_cap,
              bool write_total_at_n, uint32_t* total, const PrimScratch& ps, cudaStream_t st, uint32_t* out2) {
    scan_impl<uint32_t>(in, out, n_dev, n_host, n_cap, write_total_at_n, total, ps, st, out2);
}
void scan_u8(const uint8_t* in, uint32_t* out, const uint32_t* n_dev, uint64_t n_host, uint64_t n_cap,
             bool write_total_at_n, uint32_t* total, const PrimScratch& ps, cudaStream_t st) {
    scan_impl<uint8_t>(in, out, n_dev, n_host, n_cap, write_total_at_n, total, ps, st);
}

int plan_radix(int lo0, int w0, int lo1, int w1, RadixPass* passes, int max_passes) {
    int np = 0;
    const int lo[2] = {lo0, lo1}, wd[2] = {w0, w1};
    for (int f = 0; f < 2; f++) {
        if (wd[f] <= 0) continue;
        const int k = (wd[f] + 7) / 8;
        int shift = lo[f];
        for (int i = 0; i < k; i++) {
            const int b = wd[f] / k + (i < wd[f] % k ? 1 : 0);
            if (np < max_passes) passes[np] = RadixPass{shift, b};
            np++;
            shift += b;
        }
    }
    return np;
}

int radix_sort_u64(uint64_t* ka, uint32_t* va, uint64_t* kb, uint32_t* vb, const uint32_t* n_dev, uint64_t n_host,
                   uint64_t n_cap, const RadixPass* passes, int npass, const PrimScratch& ps, cudaStream_t st) {
    return radix_impl<uint64_t>(ka, va, kb, vb, n_dev, n_host, n_cap, passes, npass, ps, st);
}
int radix_sort_u32(uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, const uint32_t* n_dev, uint64_t n_host,
                   uint64_t n_cap, const RadixPass* passes, int npass, const PrimScratch& ps, cudaStream_t st) {
    return radix_impl<uint32_t>(ka, va, kb, vb, n_dev, n_host, n_cap, passes, npass, ps, st);
}

}  // namespace gxy
