// gxy_engine.cuh -- host-side engine shared by the plain, batched and serving
// entry points.
#pragma once

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gxy_device.cuh"
#include "gxy_kernels.cuh"
#include "gxy_prims.cuh"
#include "gxy_seed.h"

namespace gxy {

void set_error(const std::string& msg);

// Grow-only device buffer.
// Grow-only device buffer, allocated and freed in stream order on `st` (the
// owning worker's stream; the legacy stream when unset), so growing it never
// synchronises the whole device.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t st = nullptr;
    cudaError_t ensure(size_t need);
    void release();
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct Worker {
    cudaStream_t st = nullptr;
    DevBuf tk0, tv0, tk1, tv1;    // table-build temporaries
    DevBuf tocc;                  // table build: occupancy bitmap over all views' buckets and its word ranks
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};   // start, screen end, end, filter end, enumerate end
    PrimScratch ps{};
    DevBuf prim_sums, prim_hist;
    DevBuf counters;              // u32[8] + u64[4]
    DevBuf d_units, d_tsegs, d_qsegs;
    DevBuf ck0, ck1, cv0, cv1, cands, flags, offsets, ohsp;
    DevBuf rhsp, runit, rhsp2, runit2, perm, perm2;
    DevBuf d_place, rrec;         // driver records: per-unit places, records
    DevBuf rk0, rk1, rv0, rv1;    // driver records: sort keys and values (the candidates' arrays
                                  // stay intact, so a later round of passes can add to them)
    DevBuf hits;                  // raw hits of one pass
    uint64_t hit_cap = 0;
    DevBuf surv;                  // hits of one pass that pass the upper-bound filter
    uint64_t surv_cap = 0;
    DevBuf redo;                  // the two lists of tiles a pass hands to the next one
    DevBuf gpool, gruns, gaux;    // gapped extension: traceback row blocks, side runs, per-anchor arrays
    DevBuf gscr;                  // gapped extension: one run scratch per CUDA block of the first pass
    uint64_t gpool_want = 0;      // gapped extension: the traceback pool an earlier call would have needed
    cudaGraphExec_t gexec = nullptr;   // the last batched launch's graph, updated in place when it fits
    uint64_t graph_updates = 0;
    uint32_t cand_cap = 0;
    uint32_t res_cap = 0;
    void* h_pinned = nullptr;     // small host staging: counters, unit and segment descriptors
    size_t h_pinned_bytes = 0;
    void* h_res = nullptr;        // pinned staging of results (grown on demand)
    size_t h_res_bytes = 0;
    // Host-query staging for gxy_search.
    gxy_dseq* qstage = nullptr;
    gxy_dseq* tstage = nullptr;
    std::vector<gxy_dseq*> rc_tmp;
};

// One unit as the engine plans it (host side).
struct UnitPlan {
    uint32_t tseg;
    uint32_t qseg;
    const uint32_t* starts;
    const uint32_t* positions;
    const uint32_t* occ;   // the table's bucket occupancy bitmap
    uint32_t nwin;
    uint32_t primary_lo;
    uint32_t primary_hi;
    double avg_bucket;   // table positions / words: sizes the raw-hit buffer before the first pass
};

// Candidate arrays are sized up front at one candidate per this many
// estimated raw hits (the estimate carries a 1.5x margin; about 3 % of raw
// hits become candidates), up to a bound.  Larger arrays also widen the
// capacity-sized sort and scan grids of every later launch on the worker.
constexpr uint64_t kHitsPerCandidate = 32;
// With the upper-bound filter the hit buffer is sized at one slot per this
// many estimated raw hits (survivors are a few percent of the raw hits).
constexpr double kRawPerSurvivorSlot = 8.0;
constexpr uint64_t kMaxPresizedCandidates = 1ull << 25;

struct RunResult {
    std::vector<gxy_hsp> hsps;
    std::vector<uint32_t> unit;
    gxy_stats stats{};
    // With want_view set (single-unit searches), the HSPs are left in the
    // worker's pinned staging instead: view[0, n_view), valid until the
    // worker's next call; hsps and unit stay empty.
    bool want_view = false;
    const gxy_hsp* view = nullptr;
    uint64_t n_view = 0;
    // With places set (one per unit), the HSPs become driver records on the
    // device instead (global t, per-group order, dedup): records is filled,
    // hsps and unit stay empty.
    const Place* places = nullptr;
    std::vector<Record> records;
};

}  // namespace gxy

struct gxy_dseq {
    gxy_ctx* ctx = nullptr;
    int device = 0;   // the context's device, kept so that the sequence can be freed after its context
    void* alloc = nullptr;
    size_t bytes = 0;
    uint64_t* codes = nullptr;
    uint32_t* valid = nullptr;
    uint32_t* mask = nullptr;
    uint64_t len = 0;
    uint64_t nwords = 0;   // 32-position words, pads included
    cudaStream_t st = nullptr;   // stream the allocation is ordered on
};

// The device arrays of the tables built together by one sort (one table, or
// every view of a multi-view build); freed when the last of them is freed.
struct TableMem {
    int device = 0;
    uint32_t* starts = nullptr;      // tables x num_words + 1 global bucket starts
    uint32_t* positions = nullptr;   // the tables' positions, one after the other
    uint32_t* occ = nullptr;         // occupancy bits of all tables' buckets
    uint4* ilv = nullptr;            // interleaved copy of the sequence words the views cover
    uint64_t ilv_first = 0;          // the first of those words
    ~TableMem();
};

struct gxy_table {
    gxy_ctx* ctx = nullptr;
    int device = 0;   // as gxy_dseq::device
    gxy_dseq* owned = nullptr;
    const gxy_dseq* seq = nullptr;
    uint64_t lo = 0, hi = 0;
    std::shared_ptr<TableMem> mem;
    uint32_t* starts = nullptr;      // in mem, or this table's own array after a prune
    uint32_t* positions = nullptr;   // likewise
    bool own_arrays = false;         // starts and positions are this table's own (after a prune)
    uint32_t* occ = nullptr;   // bit (w & 31) of occ[w >> 5]: bucket w is non-empty (in mem)
    // starts[w] index the shared positions array (positions points at its
    // start); this table's positions begin at pos_base (0 after a prune).
    uint32_t pos_base = 0;
    uint64_t num_words = 0;
    uint64_t npos = 0;
    // Positions within a bucket are in ascending order, the reference's order.
    gxy::Pattern pat{};
    uint32_t step = 1;
    const void* hc = nullptr;
    const void* hv = nullptr;
    const void* hm = nullptr;
    uint64_t hlen = 0;
};

struct gxy_ctx {
    int device = 0;
    int sm_count = 148;
    std::mutex mu;
    std::vector<gxy::Worker*> free_workers;   // the primary worker (all_workers[0]) is taken first
    std::vector<gxy::Worker*> all_workers;
    // Screen column cap 192 (the packed screen's limit): on the 10 Mbp plain
    // launch, longer screening leaves fewer candidates for the walk to
    // re-extend (two searches 4.27 ms, against 4.31 ms at 128 and 4.51 at 64).
    gxy_tuning tuning{8, 192, 4, 8, 256u << 20, 0, 96, 1, 0, 4};
    cudaEvent_t marks[16] = {};
};

namespace gxy {

// Stream-ordered pool allocation; dev_free waits for the device first.
cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st);
void dev_free(void* p);

Worker* checkout(gxy_ctx* ctx, gxy_status* err);
void checkin(gxy_ctx* ctx, Worker* w);

gxy_status dseq_alloc(gxy_ctx* ctx, uint64_t len, gxy_dseq** out, cudaStream_t st);
void dseq_destroy(gxy_dseq* s);
// Frees in stream order on st: for sequences only st has used.
void dseq_destroy_async(gxy_dseq* s, cudaStream_t st);
gxy_status dseq_fill_host(gxy_dseq* d, const gxy_packed_seq* h, cudaStream_t st);
SeqView view_of(const gxy_dseq* s, uint64_t lo, uint64_t hi);
// A table's target view, with the table's interleaved copy of it.
SeqView table_view(const gxy_table* t);

// Returns from the calling function with a status when a CUDA call fails.
#define GXY_CK(call)                                                                         \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                    \
            return e_ == cudaErrorMemoryAllocation ? GXY_ENOMEM : GXY_ECUDA;                 \
        }                                                                                    \
    } while (0)

// Windows of a sequence of len bases for a pattern of span L:
// iter_with_stride (src/seeds.rs:151-161) visits 0, step, ... <= len - L.
inline uint32_t n_windows(uint64_t len, uint32_t L, uint32_t step) {
    if (len < L) return 0;
    return (uint32_t)((len - L) / step + 1);
}

// PosTable::build (src/pos_table.rs:35-83) for n views [lo[v], hi[v]) of one
// sequence at once (csrc/gxy_table.cu), view v's word w being bucket
// g = v * 4^w + w: fills starts (n * 4^w + 1 global bucket starts), positions
// (all views' positions, each bucket ascending) and the occupancy bitmap
// over all buckets, then first_host[0 .. n] = starts[v * 4^w] (a host sync).
// More than one view needs at least 32 buckets per view.
gxy_status atomic_build_views(const gxy_dseq* seq, uint32_t n_views, const uint64_t* lo, const uint64_t* hi,
                              const Pattern& pat, uint32_t step, uint32_t* starts, uint32_t* positions,
                              uint32_t* occ, uint32_t* first_host, Worker* W);
// ilv[j] = the 16-byte record (codes, valid, mask) of sequence word first + j,
// for j < n (SeqView::ilv).
void launch_interleave(const uint64_t* codes, const uint32_t* valid, const uint32_t* mask, uint64_t first, uint64_t n,
                       uint4* ilv, cudaStream_t st);
// Kernel attributes of the table build; once per device, before any capture.
void table_init();

// SeedPattern::parse (src/seeds.rs:38-51) with the engine's limits: at most
// 32 positions (src/seeds.rs:28-32), weight at most kMaxWeight.
gxy_status parse_pattern(const char* s, Pattern& pat);

// Validates params and the i32 envelope for a search over sequences whose
// diagonal spans are at most max_cols columns.
gxy_status check_params(const gxy_search_params* p, uint64_t max_cols);

// Runs units through screen -> sort -> walk -> compaction on worker W.
// Grows every buffer run_units sizes from a raw-hit estimate -- raw hits,
// survivors, candidates, the redo lists, the plan arrays for max_units units
// and the pinned result staging -- to what an estimate of est_hits raw hits
// and `candidates` candidates needs, so that no later call of that size pays
// for an allocation.
gxy_status reserve_worker(gxy_ctx* ctx, Worker* W, uint64_t est_hits, uint64_t candidates, uint32_t max_units);
gxy_status run_units(gxy_ctx* ctx, Worker* W, const std::vector<UnitPlan>& units, std::vector<SeqView>& tsegs,
                     std::vector<SeqView>& qsegs, const Pattern& pat, const gxy_search_params& p, bool use_graph,
                     RunResult& out);

}  // namespace gxy
