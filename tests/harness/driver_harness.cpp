// driver_harness.cpp -- a C++ caller of the C ABI (include/gxy_seed.h) that
// makes the calls the reference's driver makes for `--nogapped` output
// (src/driver.rs:156-256 and :362-391), from a pool of host threads:
//
//   chunk_target -> per chunk PosTable::build over the chunk copy (+ prune)
//   -> for every (chunk, query, strand) a search() call, the strands of one
//      chunk running concurrently on that chunk's shared table
//   -> keep HSPs anchored in the chunk's primary region, shift t_start to
//      global coordinates (build_ungapped_record, src/driver.rs:437-468)
//   -> group by (query, strand), sort by (t_start, q_start, span), drop
//      duplicates.  (The reference sorts each chunk's records separately and
//      concatenates them in thread completion order; the records are the
//      same set, sorted here across chunks so the output is deterministic.)
//
// It stands in for the Rust -sys binding the reference would use (no Rust
// toolchain here) and shows that the library is a drop-in for those calls.
//
// MODE 1 makes the same records with one gxy_batch_records call instead:
// the target and query stay on the device, every chunk's table is a view of
// the target, and the filter, global coordinates, order and dedup all run
// on the device.
//
// usage: driver_harness TARGET QUERY OUT PRIMARY_BP HALO_BP THREADS TRANSITIONS MAX_WORD_COUNT [MODE]
//   TARGET / QUERY: files of raw ASCII bases.  OUT: binary records, see write_out().
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "gxy_seed.h"

namespace {

struct HostSeq {   // a PackedSeq in host memory (src/sequences.rs:53-66)
    std::vector<uint8_t> codes, valid, mask;
    uint64_t len = 0;
    gxy_packed_seq view() const { return gxy_packed_seq{codes.data(), valid.data(), mask.data(), len}; }
};

struct Record {    // the ungapped record fields the driver fills
    uint32_t query, strand, t_start, q_start, span;
    int32_t score;
};

void die(const char* what, gxy_status s) {
    fprintf(stderr, "%s: %s (%s)\n", what, gxy_status_string(s), gxy_last_error());
    exit(2);
}

std::string read_file(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        perror(path);
        exit(2);
    }
    std::string s;
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, n);
    fclose(f);
    return s;
}

// PackedSeq::from_ascii of bytes [lo, hi), packed on the device and read back.
HostSeq pack(gxy_ctx* ctx, const std::string& ascii, uint64_t lo, uint64_t hi, bool rc) {
    gxy_dseq* d = nullptr;
    gxy_status s =
        gxy_dseq_from_ascii(ctx, reinterpret_cast<const uint8_t*>(ascii.data()) + lo, hi - lo, &d);
    if (s != GXY_OK) die("gxy_dseq_from_ascii", s);
    if (rc) {
        gxy_dseq* r = nullptr;
        s = gxy_dseq_reverse_complement(ctx, d, &r);
        if (s != GXY_OK) die("gxy_dseq_reverse_complement", s);
        gxy_dseq_free(d);
        d = r;
    }
    HostSeq h;
    h.len = hi - lo;
    h.codes.assign((h.len + 3) / 4 + 1, 0);
    h.valid.assign((h.len + 7) / 8 + 1, 0);
    h.mask.assign((h.len + 7) / 8 + 1, 0);
    s = gxy_dseq_download(d, h.codes.data(), h.valid.data(), h.mask.data());
    if (s != GXY_OK) die("gxy_dseq_download", s);
    gxy_dseq_free(d);
    return h;
}

void write_out(const char* path, const std::vector<Record>& recs) {
    FILE* f = fopen(path, "wb");
    if (!f) {
        perror(path);
        exit(2);
    }
    const uint64_t n = recs.size();
    fwrite(&n, 8, 1, f);
    if (n) fwrite(recs.data(), sizeof(Record), n, f);
    fclose(f);
}

gxy_search_params driver_params(uint32_t transitions) {
    gxy_search_params p{};
    const int32_t hoxd70[16] = {91, -114, -31, -123, -114, 100, -125, -31,
                                -31, -125, 100, -114, -123, -31, -114, 91};   // src/scoring.rs:17-23
    memcpy(p.sub, hoxd70, sizeof p.sub);
    p.ambig = -100;
    p.xdrop = 910;
    p.hspthresh = 3000;
    p.step = 1;
    p.transitions = (uint8_t)transitions;
    return p;
}

// MODE 1: the whole driver flow of one (target, query) pair in one batch.
int batched(const std::string& target, const std::string& query, const char* out, uint32_t primary,
            uint32_t halo, uint32_t transitions, uint32_t mwc, const char* pattern) {
    gxy_ctx* ctx = nullptr;
    gxy_status s = gxy_ctx_create(0, &ctx);
    if (s != GXY_OK) die("gxy_ctx_create", s);
    gxy_dseq *T = nullptr, *Q = nullptr;
    s = gxy_dseq_from_ascii(ctx, reinterpret_cast<const uint8_t*>(target.data()), target.size(), &T);
    if (s != GXY_OK) die("gxy_dseq_from_ascii", s);
    s = gxy_dseq_from_ascii(ctx, reinterpret_cast<const uint8_t*>(query.data()), query.size(), &Q);
    if (s != GXY_OK) die("gxy_dseq_from_ascii", s);
    uint64_t nchunks = 0;
    gxy_chunk_plan(target.size(), primary, halo, nullptr, 0, &nchunks);
    std::vector<uint64_t> quads(4 * std::max<uint64_t>(nchunks, 1));
    s = gxy_chunk_plan(target.size(), primary, halo, quads.data(), nchunks, &nchunks);
    if (s != GXY_OK) die("gxy_chunk_plan", s);
    std::vector<gxy_table*> tables(nchunks, nullptr);
    std::vector<gxy_unit> units;
    std::vector<gxy_unit_place> places;
    for (uint64_t c = 0; c < nchunks; c++) {
        s = gxy_table_build_view(ctx, T, quads[4 * c], quads[4 * c + 1], pattern, 1, mwc, &tables[c]);
        if (s != GXY_OK) die("gxy_table_build_view", s);
        for (uint32_t strand = 0; strand < 2; strand++) {
            units.push_back(gxy_unit{(uint32_t)c, 0, strand, (uint32_t)quads[4 * c + 2], (uint32_t)quads[4 * c + 3]});
            places.push_back(gxy_unit_place{strand, (uint32_t)quads[4 * c]});
        }
    }
    const gxy_search_params p = driver_params(transitions);
    const gxy_dseq* qs[1] = {Q};
    gxy_record_result rr{};
    s = gxy_batch_records(ctx, (uint32_t)nchunks, tables.data(), 1, qs, (uint32_t)units.size(), units.data(),
                          places.data(), &p, nullptr, &rr, nullptr);
    if (s != GXY_OK) die("gxy_batch_records", s);
    std::vector<Record> recs;
    recs.reserve(rr.n_records);
    for (uint64_t i = 0; i < rr.n_records; i++) {
        const gxy_record& r = rr.records[i];
        recs.push_back(Record{0, r.group, r.t_start, r.q_start, r.span, r.score});
    }
    write_out(out, recs);
    gxy_record_result_free(&rr);
    for (gxy_table* t : tables) gxy_table_free(t);
    gxy_dseq_free(T);
    gxy_dseq_free(Q);
    gxy_ctx_destroy(ctx);
    printf("chunks %llu records %zu\n", (unsigned long long)nchunks, recs.size());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 9 && argc != 10) {
        fprintf(stderr, "usage: %s TARGET QUERY OUT PRIMARY_BP HALO_BP THREADS TRANSITIONS MAX_WORD_COUNT [MODE]\n",
                argv[0]);
        return 2;
    }
    const std::string target = read_file(argv[1]), query = read_file(argv[2]);
    const uint32_t primary = (uint32_t)atoi(argv[4]), halo = (uint32_t)atoi(argv[5]);
    const int threads = std::max(1, atoi(argv[6]));
    const uint32_t transitions = (uint32_t)atoi(argv[7]), mwc = (uint32_t)atoi(argv[8]);
    const char* pattern = "1110100110010101111";   // 12of19 (src/seeds.rs:56)
    if (argc == 10 && atoi(argv[9]) == 1)
        return batched(target, query, argv[3], primary, halo, transitions, mwc, pattern);

    gxy_ctx* ctx = nullptr;
    gxy_status s = gxy_ctx_create(0, &ctx);
    if (s != GXY_OK) die("gxy_ctx_create", s);

    // chunk_target (src/driver.rs:156-194).
    uint64_t nchunks = 0;
    gxy_chunk_plan(target.size(), primary, halo, nullptr, 0, &nchunks);
    std::vector<uint64_t> quads(4 * std::max<uint64_t>(nchunks, 1));
    s = gxy_chunk_plan(target.size(), primary, halo, quads.data(), nchunks, &nchunks);
    if (s != GXY_OK) die("gxy_chunk_plan", s);

    // Per chunk: the chunk copy and its table (src/driver.rs:212-215), built
    // by the thread pool.
    std::vector<HostSeq> chunk_seq(nchunks);
    std::vector<gxy_table*> tables(nchunks, nullptr);
    const HostSeq qplus = pack(ctx, query, 0, query.size(), false);
    const HostSeq qminus = pack(ctx, query, 0, query.size(), true);   // rc_cache (src/driver.rs:221)
    {
        std::atomic<uint64_t> next{0};
        std::vector<std::thread> pool;
        for (int k = 0; k < threads; k++)
            pool.emplace_back([&] {
                for (uint64_t c; (c = next.fetch_add(1)) < nchunks;) {
                    chunk_seq[c] = pack(ctx, target, quads[4 * c], quads[4 * c + 1], false);
                    const gxy_packed_seq v = chunk_seq[c].view();
                    gxy_status e = gxy_table_build(ctx, &v, pattern, 1, mwc, &tables[c]);
                    if (e != GXY_OK) die("gxy_table_build", e);
                }
            });
        for (auto& t : pool) t.join();
    }

    // search() per (chunk, query, strand); the pool interleaves the units so
    // that both strands of a chunk run at once on its shared table.
    const gxy_search_params p = driver_params(transitions);
    std::vector<Record> recs;
    std::mutex mu;
    {
        std::atomic<uint64_t> next{0};
        const uint64_t nunits = nchunks * 2;
        std::vector<std::thread> pool;
        for (int k = 0; k < threads; k++)
            pool.emplace_back([&] {
                for (uint64_t u; (u = next.fetch_add(1)) < nunits;) {
                    const uint64_t c = u / 2;
                    const uint32_t strand = (uint32_t)(u % 2);
                    const gxy_packed_seq t = chunk_seq[c].view();
                    const gxy_packed_seq q = (strand ? qminus : qplus).view();
                    gxy_hsp_buf buf{};
                    gxy_status e = gxy_search(ctx, tables[c], &t, &q, &p, &buf, nullptr);
                    if (e != GXY_OK) die("gxy_search", e);
                    std::vector<Record> mine;
                    for (uint64_t i = 0; i < buf.len; i++) {
                        const gxy_hsp& h = buf.hsps[i];
                        // Primary-region filter (src/driver.rs:250-256).
                        if (h.t_start < quads[4 * c + 2] || h.t_start >= quads[4 * c + 3]) continue;
                        mine.push_back(Record{0, strand, (uint32_t)(h.t_start + quads[4 * c]), h.q_start,
                                              h.length, h.score});
                    }
                    gxy_hsp_buf_free(&buf);
                    std::lock_guard<std::mutex> g(mu);
                    recs.insert(recs.end(), mine.begin(), mine.end());
                }
            });
        for (auto& t : pool) t.join();
    }

    // Group order (query, strand), records by (t_start, q_start, span), then
    // dedup of equal coordinates (src/driver.rs:362-391).
    std::stable_sort(recs.begin(), recs.end(), [](const Record& a, const Record& b) {
        return std::tie(a.query, a.strand, a.t_start, a.q_start, a.span) <
               std::tie(b.query, b.strand, b.t_start, b.q_start, b.span);
    });
    recs.erase(std::unique(recs.begin(), recs.end(),
                           [](const Record& a, const Record& b) {
                               return a.query == b.query && a.strand == b.strand && a.t_start == b.t_start &&
                                      a.q_start == b.q_start && a.span == b.span;
                           }),
               recs.end());
    write_out(argv[3], recs);
    for (gxy_table* t : tables) gxy_table_free(t);
    gxy_ctx_destroy(ctx);
    printf("chunks %llu records %zu\n", (unsigned long long)nchunks, recs.size());
    return 0;
}
