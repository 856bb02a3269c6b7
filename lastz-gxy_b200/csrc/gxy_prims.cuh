// gxy_prims.cuh -- scan and stable LSD radix sort written for this stage.
//
// Both run on a fixed grid and read their element count from device memory,
// so a pipeline whose sizes are only known on the device (the candidate count
// after the screen) needs no host round trip and can be captured in a graph.
// Every block owns one contiguous range of the input; the radix sort's
// per-block digit histograms are scanned one digit per block, and each block
// ranks its tiles with warp match-any so equal digits keep their input order
// (stable).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gxy {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixMax = 256;

// Scratch a caller provides for the primitives (device memory).
struct PrimScratch {
    uint32_t* block_sums;   // >= max(grid, sort_grid_max, kRadixMax) entries (+1)
    uint32_t* hist;         // >= kRadixMax * max(grid, sort_grid_max) entries (+1)
    int grid;               // scan blocks (at most max(grid, sort_grid_max), sized by the capacity)
    int sort_grid_max;      // radix passes use min(this, one block per two tiles of n_cap) blocks
};

// Exclusive scan of n u32 (or u8) values into out[0..n); out[n] and *total
// (either may be null) receive the sum.  n is min(*n_dev, n_cap) when n_dev is
// not null, else n_host.  The sum must fit in u32.
// out2 (optional) receives a second copy of out[0..n); it may be `in` itself.
void scan_u32(const uint32_t* in, uint32_t* out, const uint32_t* n_dev, uint64_t n_host, uint64_t n_cap,
              bool write_total_at_n, uint32_t* total, const PrimScratch& ps, cudaStream_t st,
              uint32_t* out2 = nullptr);
void scan_u8(const uint8_t* in, uint32_t* out, const uint32_t* n_dev, uint64_t n_host, uint64_t n_cap,
             bool write_total_at_n, uint32_t* total, const PrimScratch& ps, cudaStream_t st);

// Per-device kernel attributes of the primitives; call once with the device
// current, before any stream capture.
void prims_init();

// One digit pass: shift/bits select the digit (bits <= 8).
struct RadixPass {
    int shift;
    int bits;
};
// Splits the bit ranges [lo0, lo0+w0) and [lo1, lo1+w1) into passes of at
// most 8 bits, least significant first.  Returns the number of passes.
int plan_radix(int lo0, int w0, int lo1, int w1, RadixPass* passes, int max_passes);

// Stable sort of (key, value) pairs by the digits of `passes`.  keys/vals are
// ping-ponged between the a and b buffers; the result ends in a when the
// pass count is even, in b otherwise (the return value is 0 for a, 1 for b).
// n_dev/n_host as for scan; n_cap bounds the element count read from n_dev.
int radix_sort_u64(uint64_t* ka, uint32_t* va, uint64_t* kb, uint32_t* vb, const uint32_t* n_dev,
                   uint64_t n_host, uint64_t n_cap, const RadixPass* passes, int npass,
                   const PrimScratch& ps, cudaStream_t st);
int radix_sort_u32(uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, const uint32_t* n_dev,
                   uint64_t n_host, uint64_t n_cap, const RadixPass* passes, int npass,
                   const PrimScratch& ps, cudaStream_t st);

}  // namespace gxy
