// gxy_noalloc.cu -- PosTable::build without any device allocation.
//
// Some callers cannot call cudaMalloc: code whose device memory is owned by
// another allocator (a framework's caching allocator or a fixed serving
// arena, which budget every byte and would be bypassed), and code on a path
// where an allocation's implicit device synchronisation is not acceptable.
// For them gxy_table_build_static builds a position table into output
// buffers they provide, and keeps every intermediate -- the staged target,
// the seed-word key/value ping-pong buffers of the stable sort, its digit
// histograms and block sums -- in one file-scope device array of fixed size.
//
// The array is part of this library's device code: every GPU that loads the
// library holds its kStaticScratchBytes until the process exits.  Host code
// must not pass the array's name to a kernel (on the host it is only a
// stand-in symbol); the device address comes from cudaGetSymbolAddress on
// each call, made with the caller's device current.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "gxy_engine.cuh"

namespace gxy {
namespace {

// Limits of the allocation-free build.
constexpr uint64_t kStaticMaxLen = 1ull << 20;     // target length (bp)
constexpr uint32_t kStaticMaxGrid = 296;           // primitive grid (blocks)

// Layout of the scratch array, in bytes.
constexpr uint64_t kSeqWords = ((kPad + kStaticMaxLen + kTailPad + 31) / 32 + 3) & ~3ull;
constexpr uint64_t kOffCodes = 0;
constexpr uint64_t kOffValid = kOffCodes + kSeqWords * 8;
constexpr uint64_t kOffMask = kOffValid + kSeqWords * 4;
constexpr uint64_t kOffKeys0 = (kOffMask + kSeqWords * 4 + 255) & ~255ull;
constexpr uint64_t kOffVals0 = kOffKeys0 + kStaticMaxLen * 4;
constexpr uint64_t kOffKeys1 = kOffVals0 + kStaticMaxLen * 4;
constexpr uint64_t kOffVals1 = kOffKeys1 + kStaticMaxLen * 4;
constexpr uint64_t kOffHist = kOffVals1 + kStaticMaxLen * 4;
constexpr uint64_t kOffSums = (kOffHist + ((uint64_t)kRadixMax * kStaticMaxGrid + 1) * 4 + 255) & ~255ull;
constexpr uint64_t kStaticScratchBytes = (kOffSums + (kStaticMaxGrid + 1) * 4 + 255) & ~255ull;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct DeviceSlot {
    std::mutex mu;          // one build at a time per device within this process
    unsigned char* ptr = nullptr;
    int sm_count = 0;
};
DeviceSlot g_slots[64];

gxy_status fail(gxy_status s, const std::string& m) {
    set_error(m);
    return s;
}

// The device address of the scratch array on the current device.  It is
// looked up on every call (a cheap host call) rather than cached, so a
// device reset between calls, which reloads the module and moves the array,
// cannot leave a stale address behind; the primitives' kernel attributes are
// set again for the same reason.
gxy_status scratch_address(int dev, DeviceSlot& slot) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
        return fail(GXY_ECUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(GXY_ECUDA, std::string("device attribute: ") + cudaGetErrorString(e));
    prims_init();
    slot.sm_count = sms;
    slot.ptr = static_cast<unsigned char*>(p);
    return GXY_OK;
}

}  // namespace
}  // namespace gxy

using namespace gxy;

extern "C" gxy_status gxy_table_build_static(const gxy_packed_seq* target, const char* pattern01, uint32_t step,
                                             uint32_t* starts_out, uint64_t starts_cap, uint32_t* positions_out,
                                             uint64_t positions_cap, uint64_t* n_positions) {
    if (!target || !starts_out || !positions_out || !n_positions) return fail(GXY_EINVAL, "null argument");
    if (target->len && (!target->codes || !target->valid || !target->mask)) return fail(GXY_EINVAL, "null sequence");
    if (step < 1) return fail(GXY_EINVAL, "step must be >= 1");
    if (target->len > kStaticMaxLen)
        return fail(GXY_EINVAL, "target longer than " + std::to_string(kStaticMaxLen) +
                                    " bp: too large for the allocation-free table build");
    Pattern pat;
    gxy_status s = parse_pattern(pattern01, pat);
    if (s != GXY_OK) return s;
    const uint64_t nw = 1ull << (2 * pat.weight);
    if (starts_cap < nw + 1) return fail(GXY_EINVAL, "starts_out holds fewer than num_words + 1 entries");
    const uint64_t len = target->len;
    const uint32_t nwin = len < pat.len ? 0u : (uint32_t)((len - pat.len) / step + 1);
    if (positions_cap < nwin)
        return fail(GXY_EINVAL, "positions_out holds fewer entries than the target has windows (" +
                                    std::to_string(nwin) + ")");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return fail(GXY_ECUDA, "no current CUDA device");
    DeviceSlot& slot = g_slots[dev];
    std::lock_guard<std::mutex> guard(slot.mu);
    s = scratch_address(dev, slot);
    if (s != GXY_OK) return s;
    unsigned char* base = slot.ptr;
    const cudaStream_t st = 0;

    // Stage the target in the array's sequence region; the pads must read as zero.
    uint64_t* codes = reinterpret_cast<uint64_t*>(base + kOffCodes);
    uint32_t* valid = reinterpret_cast<uint32_t*>(base + kOffValid);
    uint32_t* mask = reinterpret_cast<uint32_t*>(base + kOffMask);
    e = cudaMemsetAsync(base, 0, kOffKeys0, st);
    if (e == cudaSuccess && len) {
        e = cudaMemcpyAsync(reinterpret_cast<char*>(codes) + kPad / 4, target->codes, (len + 3) / 4,
                            cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(reinterpret_cast<char*>(valid) + kPad / 8, target->valid, (len + 7) / 8,
                                cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(reinterpret_cast<char*>(mask) + kPad / 8, target->mask, (len + 7) / 8,
                                cudaMemcpyHostToDevice, st);
    }
    // counts[word] -> exclusive scan in place -> starts (src/pos_table.rs:42-58),
    // then the stable sort of (word, position) by word (src/pos_table.rs:69-75).
    if (e == cudaSuccess) e = cudaMemsetAsync(starts_out, 0, (nw + 1) * 4, st);
    if (e != cudaSuccess) return fail(GXY_ECUDA, std::string("static table build staging: ") + cudaGetErrorString(e));
    PrimScratch ps;
    ps.grid = (int)std::min<uint32_t>(kStaticMaxGrid, (uint32_t)slot.sm_count * 2);
    ps.sort_grid_max = ps.grid;
    ps.hist = reinterpret_cast<uint32_t*>(base + kOffHist);
    ps.block_sums = reinterpret_cast<uint32_t*>(base + kOffSums);
    uint32_t* k0 = reinterpret_cast<uint32_t*>(base + kOffKeys0);
    uint32_t* v0 = reinterpret_cast<uint32_t*>(base + kOffVals0);
    uint32_t* k1 = reinterpret_cast<uint32_t*>(base + kOffKeys1);
    uint32_t* v1 = reinterpret_cast<uint32_t*>(base + kOffVals1);
    SeqView view;
    view.codes = codes;
    view.valid = valid;
    view.mask = mask;
    view.base = kPad;
    view.len = (uint32_t)len;
    view.key_base = 0;
    launch_seed_words(view, pat, step, nwin, (uint32_t)nw, k0, v0, starts_out, st);
    scan_u32(starts_out, starts_out, nullptr, nw, nw, true, nullptr, ps, st);
    RadixPass passes[8];
    int bits = 0;
    while ((1ull << bits) <= nw) bits++;
    const int np = plan_radix(0, bits, 0, 0, passes, 8);
    const int which = radix_sort_u32(k0, v0, k1, v1, nullptr, nwin, nwin, passes, np, ps, st);
    const uint32_t* sorted_pos = which ? v1 : v0;
    // A failed launch above leaves the array unwritten: report it before
    // anything is read back or copied out.
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(GXY_ECUDA, std::string("static table build: ") + cudaGetErrorString(e));
    uint32_t total = 0;
    e = cudaMemcpyAsync(&total, starts_out + nw, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && total)
        e = cudaMemcpyAsync(positions_out, sorted_pos, (size_t)total * 4, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail(GXY_ECUDA, std::string("static table build: ") + cudaGetErrorString(e));
    *n_positions = total;
    return GXY_OK;
}
