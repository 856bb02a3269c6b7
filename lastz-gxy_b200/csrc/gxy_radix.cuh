// gxy_radix.cuh -- the device side of the scan and the stable LSD radix sort
// (gxy_prims.cuh has the host entry points).  The radix kernels read their
// items through a source type (ArraySrc: key and value arrays); a source
// whose load returns false leaves that item out of the output.
#pragma once

#include <cstdint>

#include "gxy_device.cuh"
#include "gxy_prims.cuh"

namespace gxy {
namespace {

__device__ __forceinline__ uint64_t read_n(const uint32_t* n_dev, uint64_t n_host, uint64_t n_cap) {
    if (!n_dev) return n_host;
    uint64_t n = *n_dev;
    return n < n_cap ? n : n_cap;
}

// The contiguous range [beg, end) of block b when n items are split into
// `grid` ranges of whole `tile`s.
__device__ __forceinline__ void block_range(uint64_t n, uint64_t tile, uint64_t& beg, uint64_t& end) {
    const uint64_t ntiles = (n + tile - 1) / tile;
    const uint64_t per = (ntiles + gridDim.x - 1) / gridDim.x;
    beg = min(n, (uint64_t)blockIdx.x * per * tile);
    end = min(n, beg + per * tile);
}

// Block-wide exclusive scan of one u32 per thread; returns the exclusive
// prefix and writes the block total to *total_out (shared).
template <int NT>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t* total_out) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < NT / 32 ? s_warp[lane] : 0;
        uint32_t t = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, t, o);
            if (lane >= o) t += y;
        }
        if (lane < NT / 32) s_warp[lane] = t - s;
        if (lane == NT / 32 - 1) *total_out = t;
    }
    __syncthreads();
    const uint32_t r = s_warp[w] + x - v;
    __syncthreads();
    return r;
}

// Items i of two arrays.
template <typename K>
struct ArraySrc {
    const K* __restrict__ keys;
    const uint32_t* __restrict__ vals;
    __device__ __forceinline__ bool key(uint64_t i, K& k) const {
        k = keys[i];
        return true;
    }
    __device__ __forceinline__ bool load(uint64_t i, K& k, uint32_t& v) const {
        k = keys[i];
        v = vals[i];
        return true;
    }
};

template <typename K, typename Src>
__global__ __launch_bounds__(kSortThreads) void k_radix_hist(Src src, const uint32_t* n_dev, uint64_t n_host,
                                                              uint64_t n_cap, int shift, int bits, uint32_t* hist) {
    const uint64_t n = read_n(n_dev, n_host, n_cap);
    __shared__ uint32_t s_hist[kSortWarps][kRadixMax];
    const int radix = 1 << bits;
    const uint32_t dmask = (uint32_t)radix - 1;
    const int w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * kRadixMax; i += kSortThreads) (&s_hist[0][0])[i] = 0;
    __syncthreads();
    uint64_t beg, end;
    block_range(n, kSortTile, beg, end);
    for (uint64_t i = beg + threadIdx.x; i < end; i += kSortThreads) {
        K key;
        if (!src.key(i, key)) continue;   // an item the source leaves out (an unseedable window)
        const uint32_t d = (uint32_t)(key >> shift) & dmask;
        atomicAdd(&s_hist[w][d], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < radix; d += kSortThreads) {
        uint32_t s = 0;
        for (int k = 0; k < kSortWarps; k++) s += s_hist[k][d];
        hist[(uint64_t)d * gridDim.x + blockIdx.x] = s;
    }
}

// One block per digit d: exclusive scan, in place, of the digit's per-block
// counts hist[d * grid .. + grid), and totals[d] = their sum.  The scatter
// adds the digits' exclusive prefix over totals (radix entries) itself, so
// no single block has to scan the whole radix x grid histogram.
__global__ __launch_bounds__(256) void k_radix_digit_scan(uint32_t* hist, int grid, uint32_t* totals) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_total;
    uint32_t* h = hist + (uint64_t)blockIdx.x * grid;
    uint32_t carry = 0;
    for (int base = 0; base < grid; base += 256) {
        const int i = base + (int)threadIdx.x;
        const uint32_t v = i < grid ? h[i] : 0u;
        const uint32_t ex = block_excl_scan<256>(v, s_warp, &s_total);
        if (i < grid) h[i] = carry + ex;
        carry += s_total;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

template <typename K>
struct SortSmem {
    K keys[kSortTile];
    uint32_t vals[kSortTile];
    uint32_t wcnt[kSortWarps][kRadixMax];
    uint32_t tile_excl[kRadixMax];
    uint32_t tile_tot[kRadixMax];
    uint32_t off[kRadixMax];
    uint32_t warp_tmp[32];
    uint32_t total;
};

// Items the source leaves out are dropped (the output holds the kept items
// only, in stable order).
template <typename K, typename Src>
__global__ __launch_bounds__(kSortThreads) void k_radix_scatter(Src src, K* __restrict__ kout,
                                                                 uint32_t* __restrict__ vout,
                                                                 const uint32_t* n_dev, uint64_t n_host, uint64_t n_cap,
                                                                 int shift, int bits, const uint32_t* hist,
                                                                 const uint32_t* totals) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<K>& S = *reinterpret_cast<SortSmem<K>*>(smem_raw);
    const uint64_t n = read_n(n_dev, n_host, n_cap);
    const int radix = 1 << bits;
    const uint32_t dmask = (uint32_t)radix - 1;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t lt = lanemask_lt();
    uint64_t beg, end;
    block_range(n, kSortTile, beg, end);
    {
        // Output offset of digit d for this block: all smaller digits' totals
        // plus digit d's count in the blocks before this one.
        static_assert(kSortThreads == kRadixMax, "one thread per digit");
        const int d = threadIdx.x;
        const uint32_t t = d < radix ? totals[d] : 0u;
        const uint32_t g = block_excl_scan<kSortThreads>(t, S.warp_tmp, &S.total);
        S.off[d] = d < radix ? g + hist[(uint64_t)d * gridDim.x + blockIdx.x] : 0u;
    }
    for (uint64_t tb = beg; tb < end; tb += kSortTile) {
        for (int i = threadIdx.x; i < kSortWarps * kRadixMax; i += kSortThreads) (&S.wcnt[0][0])[i] = 0;
        __syncthreads();
        K k[kSortItems];
        uint32_t v[kSortItems], d[kSortItems], rk[kSortItems];
#pragma unroll
        for (int it = 0; it < kSortItems; it++) {
            const uint64_t idx = tb + (uint64_t)w * 32 * kSortItems + (uint64_t)it * 32 + lane;
            k[it] = (K)0;
            v[it] = 0u;
            const bool ok = idx < end && src.load(idx, k[it], v[it]);
            d[it] = ok ? ((uint32_t)(k[it] >> shift) & dmask) : (uint32_t)kRadixMax;
        }
#pragma unroll
        for (int it = 0; it < kSortItems; it++) {
            const uint32_t peers = __match_any_sync(kFull, d[it]);
            uint32_t base = 0;
            if (d[it] < (uint32_t)kRadixMax) base = S.wcnt[w][d[it]];
            __syncwarp();
            if (d[it] < (uint32_t)kRadixMax && (peers & lt) == 0) S.wcnt[w][d[it]] = base + __popc(peers);
            __syncwarp();
            rk[it] = base + __popc(peers & lt);
        }
        __syncthreads();
        // Per digit: exclusive prefix over warps and the tile total.
        {
            const int dd = threadIdx.x;   // kSortThreads == kRadixMax
            uint32_t run = 0;
#pragma unroll
            for (int ww = 0; ww < kSortWarps; ww++) {
                const uint32_t c = S.wcnt[ww][dd];
                S.wcnt[ww][dd] = run;
                run += c;
            }
            S.tile_tot[dd] = run;
            const uint32_t ex = block_excl_scan<kSortThreads>(run, S.warp_tmp, &S.total);
            S.tile_excl[dd] = ex;
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < kSortItems; it++) {
            if (d[it] < (uint32_t)kRadixMax) {
                const uint32_t p = S.tile_excl[d[it]] + S.wcnt[w][d[it]] + rk[it];
                S.keys[p] = k[it];
                S.vals[p] = v[it];
            }
        }
        __syncthreads();
        const uint32_t cnt = S.total;   // the tile's kept items
        for (uint32_t j = threadIdx.x; j < cnt; j += kSortThreads) {
            const K key = S.keys[j];
            const uint32_t dd = (uint32_t)(key >> shift) & dmask;
            const uint32_t g = S.off[dd] + (j - S.tile_excl[dd]);
            kout[g] = key;
            vout[g] = S.vals[j];
        }
        __syncthreads();
        S.off[threadIdx.x] += S.tile_tot[threadIdx.x];
        __syncthreads();
    }
}

}  // namespace
}  // namespace gxy
