// gxy_input.cu -- FASTA and 2bit input straight into device sequences.
//
// The reference parses on the host byte by byte and packs with
// PackedSeq::push_ascii (src/sequences.rs:338-377, src/bit2.rs:73-163).
// Here the host only walks the structure (FASTA header lines; 2bit index,
// N-block and mask-block lists) and the per-base work runs on the device:
//  - FASTA: the file goes to the device once; a flag pass drops ASCII
//    whitespace and header lines, a scan + compaction gathers each record's
//    bases, and the ASCII packer encodes them (codes, valid, soft mask).
//  - 2bit: each record's packed DNA goes to the device as is; one thread per
//    32 positions reverses the 2bit byte order, remaps T/C/A/G = 0/1/2/3 to
//    the PackedSeq codes A/C/G/T = 0/1/2/3, and applies the N and mask blocks
//    (N: invalid, code 0, never masked; mask: soft-masked).
// The results equal the reference's parse followed by PackedSeq::from_ascii,
// bit for bit (the ASCII the reference decodes 2bit into only ever holds
// T/C/A/G/N/t/c/a/g).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "gxy_engine.cuh"

using namespace gxy;

namespace gxy {
gxy_status dseq_alloc(gxy_ctx* ctx, uint64_t len, gxy_dseq** out, cudaStream_t st);
void dseq_destroy(gxy_dseq* s);
}

namespace {

// u8::is_ascii_whitespace: space, tab, LF, FF, CR.
__device__ __forceinline__ bool ascii_ws(uint8_t b) {
    return b == ' ' || b == '\t' || b == '\n' || b == '\f' || b == '\r';
}

__global__ void k_fasta_keep(const uint8_t* __restrict__ bytes, uint64_t n, uint8_t* keep) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        keep[i] = ascii_ws(bytes[i]) ? 0 : 1;
}

// Header lines [lo, hi) are not bases: one block per header line.
__global__ void k_fasta_drop_headers(const uint64_t* ranges, uint8_t* keep) {
    const uint64_t lo = ranges[2 * blockIdx.x], hi = ranges[2 * blockIdx.x + 1];
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) keep[i] = 0;
}

__global__ void k_fasta_compact(const uint8_t* __restrict__ bytes, const uint8_t* __restrict__ keep,
                                const uint32_t* __restrict__ off, uint64_t n, uint8_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (keep[i]) out[off[i]] = bytes[i];
}

__global__ void k_fasta_offsets_at(const uint32_t* __restrict__ off, const uint64_t* at, uint32_t n, uint32_t* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = off[at[i]];
}

// Positions [32w, 32w + 32) of one 2bit record.  Blocks are sorted, disjoint
// (start, end) pairs; the ones that meet this word are found by binary search.
__device__ __forceinline__ uint32_t range_bits(const uint32_t* r, uint32_t nr, uint64_t p0) {
    uint32_t lo = 0, hi = nr;   // first range with end > p0
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (r[2 * mid + 1] > p0) hi = mid;
        else lo = mid + 1;
    }
    uint32_t bits = 0;
    for (uint32_t k = lo; k < nr && r[2 * k] < p0 + 32; k++) {
        const uint64_t a = r[2 * k] > p0 ? r[2 * k] - p0 : 0;
        const uint64_t b = r[2 * k + 1] - p0 < 32 ? r[2 * k + 1] - p0 : 32;
        if (b > a) bits |= (uint32_t)((b - a >= 32 ? 0xffffffffull : ((1ull << (b - a)) - 1)) << a);
    }
    return bits;
}

__global__ void k_2bit_decode(const uint8_t* __restrict__ packed, uint64_t len, const uint32_t* nblk, uint32_t n_n,
                              const uint32_t* mblk, uint32_t n_m, uint64_t* codes, uint32_t* valid,
                              uint32_t* mask) {
    // 2bit byte -> PackedSeq byte: four bases, first base in the high bits
    // there and in the low bits here; T C A G (0 1 2 3) -> 3 1 0 2.
    __shared__ uint8_t s_lut[256];
    for (int b = threadIdx.x; b < 256; b += blockDim.x) {
        const uint8_t remap[4] = {3, 1, 0, 2};
        uint8_t o = 0;
        for (int k = 0; k < 4; k++) o |= (uint8_t)(remap[(b >> (6 - 2 * k)) & 3] << (2 * k));
        s_lut[b] = o;
    }
    __syncthreads();
    const uint64_t nw = (len + 31) / 32;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p0 = w * 32;
        const uint32_t present = len - p0 >= 32 ? 0xffffffffu : (uint32_t)((1ull << (len - p0)) - 1);
        const uint32_t nbits = range_bits(nblk, n_n, p0);
        const uint32_t v = present & ~nbits;
        const uint32_t m = range_bits(mblk, n_m, p0) & v;
        uint64_t c = 0;
        const uint64_t nbytes = (len + 3) / 4;
        for (int k = 0; k < 8; k++) {
            const uint64_t j = w * 8 + k;
            if (j < nbytes) c |= (uint64_t)s_lut[packed[j]] << (8 * k);
        }
        // Invalid positions (N, and past the end) carry code 0 (encode_base).
        uint64_t keepc = 0;
        for (int k = 0; k < 32; k++)
            if ((v >> k) & 1u) keepc |= 3ull << (2 * k);
        codes[kPad / 32 + w] = c & keepc;
        valid[kPad / 32 + w] = v;
        mask[kPad / 32 + w] = m;
    }
}

struct Reader {   // the reference's Cursor (src/bit2.rs:166-215)
    const uint8_t* b;
    uint64_t n, pos;
    bool be;
    bool ok = true;
    uint64_t need_at = 0, need = 0;
    bool take(uint64_t k) {
        if (!ok) return false;
        if (pos + k > n) {
            ok = false;
            need_at = pos;
            need = k;
            return false;
        }
        return true;
    }
    uint32_t u32() {
        if (!take(4)) return 0;
        uint32_t x;
        memcpy(&x, b + pos, 4);
        pos += 4;
        if (be) x = __builtin_bswap32(x);
        return x;
    }
    uint8_t u8() {
        if (!take(1)) return 0;
        return b[pos++];
    }
};

gxy_status fail_set(gxy_seq_set* out, const std::string& msg, gxy_status s) {
    gxy_seq_set_free(out);
    set_error(msg);
    return s;
}

gxy_status alloc_set(gxy_seq_set* out, uint64_t n) {
    out->n = n;
    out->seqs = static_cast<gxy_dseq**>(calloc(std::max<uint64_t>(n, 1), sizeof(gxy_dseq*)));
    out->names = static_cast<char**>(calloc(std::max<uint64_t>(n, 1), sizeof(char*)));
    if (!out->seqs || !out->names) return GXY_ENOMEM;
    return GXY_OK;
}

char* dup_name(const uint8_t* p, uint64_t k) {
    char* s = static_cast<char*>(malloc(k + 1));
    if (s) {
        memcpy(s, p, k);
        s[k] = 0;
    }
    return s;
}

struct WorkerLease {
    gxy_ctx* ctx;
    Worker* w;
    gxy_status err;
    explicit WorkerLease(gxy_ctx* c) : ctx(c), w(nullptr), err(GXY_OK) { w = checkout(c, &err); }
    ~WorkerLease() {
        if (w) checkin(ctx, w);
    }
};

}  // namespace

extern "C" {

void gxy_seq_set_free(gxy_seq_set* set) {
    if (!set) return;
    for (uint64_t i = 0; i < set->n; i++) {
        if (set->seqs && set->seqs[i]) dseq_destroy(set->seqs[i]);
        if (set->names) free(set->names[i]);
    }
    free(set->seqs);
    free(set->names);
    set->seqs = nullptr;
    set->names = nullptr;
    set->n = 0;
}

gxy_status gxy_parse_fasta(gxy_ctx* ctx, const uint8_t* bytes, uint64_t n, gxy_seq_set* out) {
    if (!ctx || (!bytes && n) || !out) return GXY_EINVAL;
    memset(out, 0, sizeof(*out));
    if (n >= (1ull << 32)) {
        set_error("FASTA input of 4 GiB or more is not supported");
        return GXY_EUNSUPPORTED;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return GXY_ECUDA;
    // Header lines: a line (split at LF) whose first byte is '>' (src/sequences.rs:354).
    // Line i starts after the i-th LF.  Empty lines are skipped by the
    // reference; they hold no bytes here either.
    std::vector<uint64_t> hdr;          // header line [start, end) pairs, end excludes the LF
    std::vector<std::string> names;
    for (uint64_t pos = 0; pos < n;) {
        const void* gt = memchr(bytes + pos, '>', n - pos);
        if (!gt) break;
        const uint64_t i = static_cast<const uint8_t*>(gt) - bytes;
        if (i == 0 || bytes[i - 1] == '\n') {
            const void* lf = memchr(bytes + i, '\n', n - i);
            const uint64_t e = lf ? (uint64_t)(static_cast<const uint8_t*>(lf) - bytes) : n;
            // The name: the first whitespace-delimited token after '>'.
            uint64_t a = i + 1;
            auto ws = [](uint8_t c) { return c == ' ' || c == '\t' || c == '\n' || c == '\f' || c == '\r'; };
            while (a < e && ws(bytes[a])) a++;
            uint64_t b = a;
            while (b < e && !ws(bytes[b])) b++;
            if (b == a) {
                uint64_t line = 1;
                for (uint64_t k = 0; k < i; k++) line += bytes[k] == '\n';
                set_error("empty FASTA header at line " + std::to_string(line) + " (src/sequences.rs:357-361)");
                return GXY_EINVAL;
            }
            names.emplace_back(reinterpret_cast<const char*>(bytes + a), b - a);
            hdr.push_back(i);
            hdr.push_back(e);
            pos = e;
        } else {
            pos = i + 1;
        }
    }
    const uint64_t nrec = names.size();
    if (alloc_set(out, nrec) != GXY_OK) return fail_set(out, "host allocation of the sequence set", GXY_ENOMEM);
    for (uint64_t r = 0; r < nrec; r++) {
        out->names[r] = dup_name(reinterpret_cast<const uint8_t*>(names[r].data()), names[r].size());
        if (!out->names[r]) return fail_set(out, "host allocation of FASTA names", GXY_ENOMEM);
    }
    if (nrec == 0) return GXY_OK;   // no header: the reference returns no sequences
    WorkerLease L(ctx);
    if (!L.w) return fail_set(out, "no worker", L.err);
    Worker* W = L.w;
    cudaStream_t st = W->st;
    // Device buffers: file bytes, keep flags, offsets, compacted bases.
    uint8_t *dbytes = nullptr, *dkeep = nullptr, *dcomp = nullptr;
    uint32_t* doff = nullptr;
    uint64_t* dhdr = nullptr;
    uint64_t* dat = nullptr;
    uint32_t* dbound = nullptr;
    auto release = [&]() {
        cudaFreeAsync(dbytes, st);
        cudaFreeAsync(dkeep, st);
        cudaFreeAsync(dcomp, st);
        cudaFreeAsync(doff, st);
        cudaFreeAsync(dhdr, st);
        cudaFreeAsync(dat, st);
        cudaFreeAsync(dbound, st);
        cudaStreamSynchronize(st);
    };
    cudaError_t e = cudaMallocAsync((void**)&dbytes, n, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dkeep, n, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dcomp, n, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&doff, (n + 1) * 4, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dhdr, hdr.size() * 8, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dat, (nrec + 1) * 8, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dbound, (nrec + 1) * 4, st);
    if (e != cudaSuccess) {
        release();
        return fail_set(out, std::string("FASTA device buffers: ") + cudaGetErrorString(e), GXY_ENOMEM);
    }
    // Record r's bases are those kept in [boundary r, boundary r + 1): record
    // 0 also takes bases before the first header, as the reference does.
    std::vector<uint64_t> at(nrec + 1);
    at[0] = 0;
    for (uint64_t r = 1; r < nrec; r++) at[r] = hdr[2 * r];
    at[nrec] = n;
    e = cudaMemcpyAsync(dbytes, bytes, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dhdr, hdr.data(), hdr.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dat, at.data(), at.size() * 8, cudaMemcpyHostToDevice, st);
    const int grid = ctx->sm_count * 8;
    if (e == cudaSuccess) {
        count_launch(3);
        k_fasta_keep<<<grid, 256, 0, st>>>(dbytes, n, dkeep);
        k_fasta_drop_headers<<<(unsigned)nrec, 256, 0, st>>>(dhdr, dkeep);
        scan_u8(dkeep, doff, nullptr, n, n, true, nullptr, W->ps, st);
        k_fasta_compact<<<grid, 256, 0, st>>>(dbytes, dkeep, doff, n, dcomp);
        count_launch();
        k_fasta_offsets_at<<<1, 256, 0, st>>>(doff, dat, (uint32_t)(nrec + 1), dbound);
    }
    std::vector<uint32_t> bound(nrec + 1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bound.data(), dbound, (nrec + 1) * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    for (uint64_t r = 0; r < nrec && e == cudaSuccess; r++) {
        const uint64_t len = bound[r + 1] - bound[r];
        gxy_status s = dseq_alloc(ctx, len, &out->seqs[r], st);
        if (s != GXY_OK) {
            release();
            gxy_seq_set_free(out);
            return s;
        }
        launch_pack_ascii(dcomp + bound[r], len, out->seqs[r]->codes, out->seqs[r]->valid, out->seqs[r]->mask, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    release();
    if (e != cudaSuccess) return fail_set(out, std::string("FASTA parse: ") + cudaGetErrorString(e), GXY_ECUDA);
    return GXY_OK;
}

gxy_status gxy_parse_2bit(gxy_ctx* ctx, const uint8_t* bytes, uint64_t n, gxy_seq_set* out) {
    if (!ctx || (!bytes && n) || !out) return GXY_EINVAL;
    memset(out, 0, sizeof(*out));
    auto truncated = [&](const Reader& r) {
        return fail_set(out, "truncated 2bit file (needed " + std::to_string(r.need) + " bytes at offset " +
                                 std::to_string(r.need_at) + ", src/bit2.rs:51-52)",
                        GXY_EINVAL);
    };
    if (n < 4) {
        Reader r{bytes, n, 0, false};
        r.take(4);
        return truncated(r);
    }
    uint32_t m0;
    memcpy(&m0, bytes, 4);
    bool be;
    if (m0 == 0x1A412743u) be = false;
    else if (m0 == 0x4327411Au) be = true;
    else {
        char buf[64];
        snprintf(buf, sizeof buf, "not a 2bit file (magic = 0x%08x)", m0);
        set_error(buf);
        return GXY_EINVAL;
    }
    Reader r{bytes, n, 0, be};
    r.u32();
    const uint32_t version = r.u32();
    if (r.ok && version != 0) {
        set_error("unsupported 2bit version " + std::to_string(version));
        return GXY_EINVAL;
    }
    const uint32_t count = r.u32();
    r.u32();
    if (!r.ok) return truncated(r);
    std::vector<std::pair<std::string, uint32_t>> index;
    for (uint32_t i = 0; i < count; i++) {
        const uint32_t ns = r.u8();
        if (!r.take(ns)) return truncated(r);
        std::string name(reinterpret_cast<const char*>(bytes + r.pos), ns);
        r.pos += ns;
        const uint32_t off = r.u32();
        if (!r.ok) return truncated(r);
        index.emplace_back(std::move(name), off);
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return GXY_ECUDA;
    if (alloc_set(out, count) != GXY_OK) return fail_set(out, "host allocation of the sequence set", GXY_ENOMEM);
    for (uint32_t i = 0; i < count; i++) {
        out->names[i] = dup_name(reinterpret_cast<const uint8_t*>(index[i].first.data()), index[i].first.size());
        if (!out->names[i]) return fail_set(out, "host allocation of 2bit names", GXY_ENOMEM);
    }
    WorkerLease L(ctx);
    if (!L.w) return fail_set(out, "no worker", L.err);
    cudaStream_t st = L.w->st;
    for (uint32_t i = 0; i < count; i++) {
        Reader q{bytes, n, 0, be};
        if (index[i].second > n) {
            q.need_at = 0;
            q.need = index[i].second;
            return truncated(q);
        }
        q.pos = index[i].second;
        const uint32_t dna = q.u32();
        auto blocks = [&](std::vector<uint32_t>& out_ranges) {
            const uint32_t k = q.u32();
            std::vector<uint32_t> s(k), z(k);
            for (uint32_t j = 0; j < k; j++) s[j] = q.u32();
            for (uint32_t j = 0; j < k; j++) z[j] = q.u32();
            // Sorted, merged [start, end) ranges clamped to the record.
            std::vector<std::pair<uint64_t, uint64_t>> v;
            for (uint32_t j = 0; j < k; j++) {
                const uint64_t a = std::min<uint64_t>(s[j], dna), b = std::min<uint64_t>((uint64_t)s[j] + z[j], dna);
                if (b > a) v.emplace_back(a, b);
            }
            std::sort(v.begin(), v.end());
            for (auto& x : v) {
                if (!out_ranges.empty() && x.first <= out_ranges.back()) {
                    out_ranges.back() = std::max<uint32_t>(out_ranges.back(), (uint32_t)x.second);
                } else {
                    out_ranges.push_back((uint32_t)x.first);
                    out_ranges.push_back((uint32_t)x.second);
                }
            }
        };
        std::vector<uint32_t> nr, mr;
        blocks(nr);
        blocks(mr);
        q.u32();
        const uint64_t pb = (uint64_t)(dna + 3) / 4;
        if (!q.take(pb)) return truncated(q);
        const uint8_t* packed = bytes + q.pos;
        gxy_status s = dseq_alloc(ctx, dna, &out->seqs[i], st);
        if (s != GXY_OK) {
            gxy_seq_set_free(out);
            return s;
        }
        if (dna == 0) continue;
        uint8_t* dpk = nullptr;
        uint32_t* drng = nullptr;
        cudaError_t e = cudaMallocAsync((void**)&dpk, pb, st);
        if (e == cudaSuccess) e = cudaMallocAsync((void**)&drng, (nr.size() + mr.size() + 2) * 4, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dpk, packed, pb, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && !nr.empty())
            e = cudaMemcpyAsync(drng, nr.data(), nr.size() * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && !mr.empty())
            e = cudaMemcpyAsync(drng + nr.size(), mr.data(), mr.size() * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            gxy_dseq* d = out->seqs[i];
            const uint64_t nw = (dna + 31) / 32;
            count_launch();
            k_2bit_decode<<<(unsigned)std::min<uint64_t>((nw + 255) / 256, (uint64_t)ctx->sm_count * 16), 256, 0,
                            st>>>(dpk, dna, drng, (uint32_t)(nr.size() / 2), drng + nr.size(),
                                  (uint32_t)(mr.size() / 2), d->codes, d->valid, d->mask);
            e = cudaStreamSynchronize(st);   // the host buffers of this record die here
        }
        cudaFreeAsync(dpk, st);
        cudaFreeAsync(drng, st);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) return fail_set(out, std::string("2bit decode: ") + cudaGetErrorString(e), GXY_ECUDA);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail_set(out, "2bit decode", GXY_ECUDA);
    return GXY_OK;
}

}  // extern "C"
