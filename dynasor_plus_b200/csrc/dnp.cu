// ============================================================================
//  dnp.cu -- processed-tensor files (.dnp) for the PingPong and NCopy layouts.
//
//  The reference's runtime-only mode (src/dynasor_dnp.cpp, format in
//  include/dynasor_dnp.h:29-98) saves the state after build_flycoo -- shard
//  geometry, touched-row bitmaps, shard tables, the thread-specific LPT
//  schedule and cursor table, and the slab(s) -- so later runs skip the
//  preprocessing.  This file reads and writes the same bytes:
//
//    header   "DNP1", version 1, value/index bytes (4/4), layout kind
//             (0 Morton, 1 NCopy, 2 PingPong, 3 InPlace), num_modes, nnz,
//             mode_size[8], num_threads, tnorm_sq, reserved[14]
//    FLYCOO   shards[8], mn[8], mn_shift[8], shard_size, avg_fiber_len[8],
//             kernel_class[8], inplace mode (i8) + 7 pad, remap row stride,
//             per mode: touched count, bitmap bytes, bitmap;
//             per mode: K, shard_begin[K], shard_end[K];
//             per mode: thread count, per thread: length, shard ids (u64);
//             per mode: cursor count, cursors (u64)
//    slab     PingPong: vals, idx[0..N-1];  NCopy: fiber_sorted[8], csr[8],
//             then per copy k: vals, idx[0..N-1], rowptr[I_k + 1] if csr[k]
//
//  A plan built from a file uses its slabs, shard tables and schedule as
//  they are (no device sort); the cursor table and touched bitmaps are read
//  and kept only for writing the file back, since the device remap derives
//  its offsets from per-chunk histograms.  On saving, the cursor table,
//  bitmaps and NCopy row pointers are recomputed from the slab exactly as
//  build_flycoo defines them (src/dynasor_preprocess.cpp:136-281, 332-463,
//  1914-1944), so a plan built from the same tensor and thread count writes
//  the file the reference writes.
// ============================================================================
#include "dgpu_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace dgpu;

namespace {

constexpr char kMagic[4] = {'D', 'N', 'P', '1'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kKindMorton = 0, kKindNCopy = 1, kKindPingPong = 2, kKindInPlace = 3;
constexpr uint32_t kShardSize = 16;     // build_flycoo's default group size g (main.cpp --shard-size)

struct FileCloser {
    void operator()(std::FILE* f) const { if (f) std::fclose(f); }
};
using File = std::unique_ptr<std::FILE, FileCloser>;

struct Reader {
    std::FILE* fp;
    bool ok = true;
    template <typename T> void get(T& v) { if (ok) ok = std::fread(&v, sizeof(T), 1, fp) == 1; }
    void bytes(void* p, size_t n) { if (ok && n) ok = std::fread(p, 1, n, fp) == n; }
};
struct Writer {
    std::FILE* fp;
    bool ok = true;
    template <typename T> void put(const T& v) { if (ok) ok = std::fwrite(&v, sizeof(T), 1, fp) == 1; }
    void bytes(const void* p, size_t n) { if (ok && n) ok = std::fwrite(p, 1, n, fp) == n; }
};

struct Header {
    char     magic[4];
    uint32_t version, value_bytes, index_bytes, kind, num_modes;
    uint64_t nnz;
    uint32_t dims[DGPU_MAX_MODES];
    uint32_t threads;
    double   tnorm_sq;
    uint32_t reserved[14];
};

bool read_header(Reader& r, Header& h) {
    r.bytes(h.magic, 4);
    r.get(h.version);
    r.get(h.value_bytes);
    r.get(h.index_bytes);
    r.get(h.kind);
    r.get(h.num_modes);
    r.get(h.nnz);
    r.bytes(h.dims, sizeof(h.dims));
    r.get(h.threads);
    r.get(h.tnorm_sq);
    r.bytes(h.reserved, sizeof(h.reserved));
    return r.ok;
}

// The reference's header checks (src/dynasor_dnp.cpp:153-196).
int check_header(const Header& h, const char* path) {
    if (std::memcmp(h.magic, kMagic, 4) != 0) {
        set_error("dnp: %s: bad magic (not a processed-tensor file)", path);
        return DGPU_ERR_IO;
    }
    if (h.version != kVersion) {
        set_error("dnp: %s: version %u not supported (expected %u)", path, h.version, kVersion);
        return DGPU_ERR_IO;
    }
    if (h.value_bytes != 4 || h.index_bytes != 4) {
        set_error("dnp: %s: value/index bytes %u/%u, only 4/4 is supported", path, h.value_bytes,
                  h.index_bytes);
        return DGPU_ERR_IO;
    }
    if (h.num_modes == 0 || h.num_modes > (uint32_t)DGPU_MAX_MODES) {
        set_error("dnp: %s: invalid num_modes %u (max %d)", path, h.num_modes, DGPU_MAX_MODES);
        return DGPU_ERR_IO;
    }
    if (h.nnz == 0) {
        set_error("dnp: %s: nnz = 0 is not supported", path);
        return DGPU_ERR_IO;
    }
    if (h.kind > kKindInPlace) {
        set_error("dnp: %s: unknown layout kind %u", path, h.kind);
        return DGPU_ERR_IO;
    }
    return DGPU_OK;
}

const char* kind_name(uint32_t k) {
    switch (k) {
        case kKindMorton: return "Morton";
        case kKindNCopy: return "NCopy";
        case kKindPingPong: return "PingPong";
        default: return "InPlace";
    }
}

int read_flycoo(Reader& r, DnpImage& img) {
    const int N = img.N;
    uint32_t spm[DGPU_MAX_MODES], mn[DGPU_MAX_MODES], kcls[DGPU_MAX_MODES];
    int32_t shft[DGPU_MAX_MODES];
    double afl[DGPU_MAX_MODES];
    r.bytes(spm, sizeof(spm));
    r.bytes(mn, sizeof(mn));
    r.bytes(shft, sizeof(shft));
    r.get(img.shard_size);
    r.bytes(afl, sizeof(afl));
    r.bytes(kcls, sizeof(kcls));
    r.get(img.inplace_mode);
    uint8_t pad[7];
    r.bytes(pad, 7);
    r.get(img.remap_stride);
    if (!r.ok) return DGPU_ERR_IO;
    for (int n = 0; n < N; ++n) {
        img.K[n] = spm[n];
        img.mn[n] = mn[n];
        img.shift[n] = shft[n];
        img.afl[n] = afl[n];
        img.kclass[n] = kcls[n];
        // rows per shard a power of two, K = ceil(I_n / mn)
        const bool pow2 = mn[n] != 0 && (mn[n] & (mn[n] - 1)) == 0;
        const uint64_t want = pow2 ? ((uint64_t)img.dims[n] + mn[n] - 1) / mn[n] : 0;
        if (!pow2 || spm[n] != std::max<uint64_t>(want, 1) || shft[n] < 0 || shft[n] > 31 ||
            (1u << shft[n]) != mn[n]) {
            set_error("dnp: mode %d geometry (%u shards, %u rows per shard, shift %d) does not fit "
                      "%u rows", n, spm[n], mn[n], shft[n], img.dims[n]);
            return DGPU_ERR_IO;
        }
    }
    img.touched_count.assign(N, 0);
    img.touched.assign(N, {});
    for (int n = 0; n < N; ++n) {
        uint64_t cnt = 0, nb = 0;
        r.get(cnt);
        r.get(nb);
        if (!r.ok) return DGPU_ERR_IO;
        if (nb > ((uint64_t)img.dims[n] + 7) / 8) {
            set_error("dnp: mode %d touched bitmap of %llu bytes for %u rows", n,
                      (unsigned long long)nb, img.dims[n]);
            return DGPU_ERR_IO;
        }
        img.touched_count[n] = cnt;
        img.touched[n].resize(nb);
        r.bytes(img.touched[n].data(), nb);
    }
    img.sbeg.assign(N, {});
    img.send.assign(N, {});
    for (int n = 0; n < N; ++n) {
        uint64_t K = 0;
        r.get(K);
        if (!r.ok || K != img.K[n]) {
            set_error("dnp: shard count mismatch in mode %d (header %u, stream %llu)", n, img.K[n],
                      (unsigned long long)K);
            return DGPU_ERR_IO;
        }
        img.sbeg[n].resize(K);
        img.send[n].resize(K);
        r.bytes(img.sbeg[n].data(), K * 8);
        r.bytes(img.send[n].data(), K * 8);
    }
    img.sched.assign(N, {});
    for (int n = 0; n < N; ++n) {
        uint64_t nt = 0;
        r.get(nt);
        if (!r.ok || nt != (uint64_t)img.threads) {
            set_error("dnp: schedule of mode %d holds %llu thread lists, the header %d", n,
                      (unsigned long long)nt, img.threads);
            return DGPU_ERR_IO;
        }
        img.sched[n].assign(img.threads, {});
        for (int t = 0; t < img.threads; ++t) {
            uint64_t len = 0;
            r.get(len);
            if (!r.ok) return DGPU_ERR_IO;
            if (len > img.K[n]) {
                set_error("dnp: mode %d thread %d lists %llu of %u shards", n, t,
                          (unsigned long long)len, img.K[n]);
                return DGPU_ERR_IO;
            }
            std::vector<uint64_t> wide(len);
            r.bytes(wide.data(), len * 8);
            img.sched[n][t].resize(len);
            for (uint64_t k = 0; k < len; ++k) {
                if (wide[k] >= img.K[n]) {
                    set_error("dnp: mode %d schedule names shard %llu of %u", n,
                              (unsigned long long)wide[k], img.K[n]);
                    return DGPU_ERR_IO;
                }
                img.sched[n][t][k] = (uint32_t)wide[k];
            }
        }
    }
    img.cursor.assign(N, {});
    for (int n = 0; n < N; ++n) {
        uint64_t len = 0;
        r.get(len);
        const uint64_t knext = img.K[(n + 1) % N];
        if (!r.ok) return DGPU_ERR_IO;
        if (len > (uint64_t)img.threads * (knext + 8)) {
            set_error("dnp: mode %d cursor table of %llu entries", n, (unsigned long long)len);
            return DGPU_ERR_IO;
        }
        img.cursor[n].resize(len);
        r.bytes(img.cursor[n].data(), len * 8);
    }
    return r.ok ? DGPU_OK : DGPU_ERR_IO;
}

void read_copy(Reader& r, DnpImage& img, int k) {
    img.vals[k].resize(img.nnz);
    r.bytes(img.vals[k].data(), img.nnz * 4);
    for (int m = 0; m < img.N; ++m) {
        img.idx[k][m].resize(img.nnz);
        r.bytes(img.idx[k][m].data(), img.nnz * 4);
    }
}

// Header (+ body unless header_only) of `path`; `threads` > 0 must match the
// file's thread count (src/dynasor_dnp.cpp:731-743).
int dnp_read(const char* path, int threads, bool header_only, DnpImage& img, uint32_t* kind_out) {
    File f(std::fopen(path, "rb"));
    if (!f) {
        set_error("dnp: cannot open '%s'", path);
        return DGPU_ERR_IO;
    }
    Reader r{f.get()};
    Header h{};
    if (!read_header(r, h)) {
        set_error("dnp: %s: truncated header", path);
        return DGPU_ERR_IO;
    }
    DGPU_TRY(check_header(h, path));
    if (kind_out) *kind_out = h.kind;
    img.N = (int)h.num_modes;
    img.nnz = h.nnz;
    for (int n = 0; n < DGPU_MAX_MODES; ++n) img.dims[n] = n < img.N ? h.dims[n] : 0u;
    img.threads = (int)h.threads;
    img.tnorm_sq = h.tnorm_sq;
    img.layout = h.kind == kKindNCopy ? DGPU_LAYOUT_NCOPY
               : h.kind == kKindMorton ? DGPU_LAYOUT_MORTON : DGPU_LAYOUT_PINGPONG;
    if (header_only) return DGPU_OK;
    if (threads > 0 && (int)h.threads != threads) {
        set_error("dnp: %s was saved with %u threads but %d were requested; the schedule and "
                  "cursors are specific to the thread count", path, h.threads, threads);
        return DGPU_ERR_ARG;
    }
    if (h.kind == kKindInPlace) {
        set_error("dnp: %s holds the %s layout; this engine reads PingPong, NCopy and Morton "
                  "files", path, kind_name(h.kind));
        return DGPU_ERR_ARG;
    }
    if (img.N < 2) {
        set_error("dnp: %s: %d modes (this engine needs 2..%d)", path, img.N, DGPU_MAX_MODES);
        return DGPU_ERR_ARG;
    }
    if (img.nnz >= 0xffffffffull) {
        set_error("dnp: %s: nnz %llu exceeds the 32-bit slab positions", path,
                  (unsigned long long)img.nnz);
        return DGPU_ERR_ARG;
    }
    if (h.kind == kKindMorton) {
        // mask[8] (u64), bits[8] (u8; 8 bytes, so no padding), keys, values
        // (src/dynasor_dnp.cpp:203-264)
        r.bytes(img.mmask, sizeof(img.mmask));
        r.bytes(img.mbits, sizeof(img.mbits));
        const long here = std::ftell(f.get());
        std::fseek(f.get(), 0, SEEK_END);
        const long end = std::ftell(f.get());
        std::fseek(f.get(), here, SEEK_SET);
        const uint64_t need = img.nnz * 12ull;
        if (!r.ok || here < 0 || end < here || (uint64_t)(end - here) < need) {
            set_error("dnp: %s (Morton) body truncated", path);
            return DGPU_ERR_IO;
        }
        img.mkeys.resize(img.nnz);
        img.mvals.resize(img.nnz);
        r.bytes(img.mkeys.data(), img.nnz * 8);
        r.bytes(img.mvals.data(), img.nnz * 4);
        if (!r.ok) {
            set_error("dnp: %s (Morton) body truncated", path);
            return DGPU_ERR_IO;
        }
        return DGPU_OK;
    }
    int rc = read_flycoo(r, img);
    if (rc != DGPU_OK) {
        if (rc == DGPU_ERR_IO && r.ok) return rc;     // message already set
        set_error("dnp: %s: FLYCOO metadata truncated or malformed", path);
        return DGPU_ERR_IO;
    }
    // the slab bytes must be present before they are allocated
    {
        const long here = std::ftell(f.get());
        std::fseek(f.get(), 0, SEEK_END);
        const long end = std::ftell(f.get());
        std::fseek(f.get(), here, SEEK_SET);
        const uint64_t copy = img.nnz * 4ull * (uint64_t)(img.N + 1);
        const uint64_t need = h.kind == kKindPingPong ? copy : 2ull * DGPU_MAX_MODES + img.N * copy;
        if (here < 0 || end < here || (uint64_t)(end - here) < need) {
            set_error("dnp: %s (%s) body truncated: %lld bytes left, the slab needs %llu", path,
                      kind_name(h.kind), (long long)(end - here), (unsigned long long)need);
            return DGPU_ERR_IO;
        }
    }
    if (h.kind == kKindPingPong) {
        read_copy(r, img, 0);
    } else {
        r.bytes(img.fiber_sorted, DGPU_MAX_MODES);
        r.bytes(img.csr, DGPU_MAX_MODES);
        for (int k = 0; k < img.N && r.ok; ++k) {
            read_copy(r, img, k);
            if (img.csr[k]) {
                img.rowptr[k].resize((size_t)img.dims[k] + 1);
                r.bytes(img.rowptr[k].data(), img.rowptr[k].size() * 8);
            }
        }
    }
    if (!r.ok) {
        set_error("dnp: %s (%s) body truncated", path, kind_name(h.kind));
        return DGPU_ERR_IO;
    }
    return DGPU_OK;
}

int dnp_write(const char* path, const DnpImage& img) {
    File f(std::fopen(path, "wb"));
    if (!f) {
        set_error("dnp: cannot create '%s'", path);
        return DGPU_ERR_IO;
    }
    Writer w{f.get()};
    const int N = img.N;
    const uint32_t kind = img.layout == DGPU_LAYOUT_NCOPY ? kKindNCopy
                        : img.layout == DGPU_LAYOUT_MORTON ? kKindMorton : kKindPingPong;
    w.bytes(kMagic, 4);
    w.put(kVersion);
    w.put((uint32_t)4);
    w.put((uint32_t)4);
    w.put(kind);
    w.put((uint32_t)N);
    w.put(img.nnz);
    w.bytes(img.dims, sizeof(uint32_t) * DGPU_MAX_MODES);
    w.put((uint32_t)img.threads);
    w.put(img.tnorm_sq);
    const uint32_t reserved[14] = {};
    w.bytes(reserved, sizeof(reserved));
    if (kind == kKindMorton) {
        w.bytes(img.mmask, sizeof(img.mmask));
        w.bytes(img.mbits, sizeof(img.mbits));
        w.bytes(img.mkeys.data(), img.nnz * 8);
        w.bytes(img.mvals.data(), img.nnz * 4);
        const bool ok = w.ok;
        f.reset();
        if (!ok) {
            std::remove(path);
            set_error("dnp: I/O failure writing '%s'", path);
            return DGPU_ERR_IO;
        }
        return DGPU_OK;
    }

    uint32_t spm[DGPU_MAX_MODES] = {}, mn[DGPU_MAX_MODES] = {}, kcls[DGPU_MAX_MODES] = {};
    int32_t shft[DGPU_MAX_MODES] = {};
    double afl[DGPU_MAX_MODES] = {};
    for (int n = 0; n < N; ++n) {
        spm[n] = img.K[n];
        mn[n] = img.mn[n];
        shft[n] = img.shift[n];
        afl[n] = img.afl[n];
        kcls[n] = img.kclass[n];
    }
    w.bytes(spm, sizeof(spm));
    w.bytes(mn, sizeof(mn));
    w.bytes(shft, sizeof(shft));
    w.put(img.shard_size);
    w.bytes(afl, sizeof(afl));
    w.bytes(kcls, sizeof(kcls));
    w.put(img.inplace_mode);
    const uint8_t pad[7] = {};
    w.bytes(pad, 7);
    w.put(img.remap_stride);
    for (int n = 0; n < N; ++n) {
        w.put(img.touched_count[n]);
        w.put((uint64_t)img.touched[n].size());
        w.bytes(img.touched[n].data(), img.touched[n].size());
    }
    for (int n = 0; n < N; ++n) {
        w.put((uint64_t)img.K[n]);
        w.bytes(img.sbeg[n].data(), img.sbeg[n].size() * 8);
        w.bytes(img.send[n].data(), img.send[n].size() * 8);
    }
    for (int n = 0; n < N; ++n) {
        w.put((uint64_t)img.threads);
        for (int t = 0; t < img.threads; ++t) {
            const auto& lst = img.sched[n][t];
            w.put((uint64_t)lst.size());
            for (uint32_t s : lst) w.put((uint64_t)s);
        }
    }
    for (int n = 0; n < N; ++n) {
        w.put((uint64_t)img.cursor[n].size());
        w.bytes(img.cursor[n].data(), img.cursor[n].size() * 8);
    }
    const int copies = kind == kKindNCopy ? N : 1;
    if (kind == kKindNCopy) {
        w.bytes(img.fiber_sorted, DGPU_MAX_MODES);
        w.bytes(img.csr, DGPU_MAX_MODES);
    }
    for (int k = 0; k < copies; ++k) {
        w.bytes(img.vals[k].data(), img.nnz * 4);
        for (int m = 0; m < N; ++m) w.bytes(img.idx[k][m].data(), img.nnz * 4);
        if (kind == kKindNCopy && img.csr[k]) w.bytes(img.rowptr[k].data(), img.rowptr[k].size() * 8);
    }
    const bool ok = w.ok;
    f.reset();
    if (!ok) {
        std::remove(path);
        set_error("dnp: I/O failure writing '%s'", path);
        return DGPU_ERR_IO;
    }
    return DGPU_OK;
}

// Touched-row bitmap and count of one mode (bit r of byte r >> 3 set iff a
// nonzero has row r; src/dynasor_preprocess.cpp:136-172, 255-281).
void touched_rows(const std::vector<uint32_t>& idx, uint32_t dim, std::vector<uint8_t>& bits,
                  uint64_t& count) {
    bits.assign(((size_t)dim + 7) / 8, 0);
    for (uint32_t r : idx) bits[r >> 3] |= (uint8_t)(1u << (r & 7u));
    count = 0;
    for (uint8_t b : bits) count += (uint64_t)__builtin_popcount((unsigned)b);
}

// Cursor table of mode n (src/dynasor_preprocess.cpp:332-463): row stride =
// K_{n+1} rounded up to 8; cursor[tid * stride + s'] = shard_begin[n+1][s'] +
// the nonzeros of shards owned by threads < tid whose next-mode shard is s'.
// Counts depend only on which nonzeros lie in each (shard, next shard) pair,
// so any element order gives the table.
void cursor_table(const Plan& p, int n, const std::vector<uint32_t>& idx_n,
                  const std::vector<uint32_t>& idx_next, std::vector<uint64_t>& out) {
    const int nm = (n + 1) % p.N;
    const size_t stride = ((size_t)p.K[nm] + 7) & ~(size_t)7;
    std::vector<int> owner(p.K[n], -1);
    for (int t = 0; t < p.T; ++t)
        for (uint32_t s : p.sched[n][t]) owner[s] = t;
    std::vector<uint64_t> hist((size_t)p.T * stride, 0);
    for (size_t i = 0; i < idx_n.size(); ++i) {
        const int t = owner[idx_n[i] >> p.shift[n]];
        if (t >= 0) ++hist[(size_t)t * stride + (idx_next[i] >> p.shift[nm])];
    }
    out.assign((size_t)p.T * stride, 0);
    for (uint32_t s = 0; s < p.K[nm]; ++s) {
        uint64_t c = p.sbeg[nm][s];
        for (int t = 0; t < p.T; ++t) {
            out[(size_t)t * stride + s] = c;
            c += hist[(size_t)t * stride + s];
        }
    }
}

// CSR row pointers of a fiber-sorted NCopy copy (src/dynasor_preprocess.cpp:
// 1914-1944): rowptr[r] = first position of row r, rowptr[I_k] = nnz.
void row_pointers(const Plan& p, int k, const std::vector<uint32_t>& ik, std::vector<uint64_t>& rp) {
    const uint32_t I = p.dims[k];
    rp.assign((size_t)I + 1, 0);
    rp[I] = p.nnz;
    for (uint32_t s = 0; s < p.K[k]; ++s) {
        const uint64_t b = p.sbeg[k][s], e = p.send[k][s];
        const uint32_t lo = s << p.shift[k];
        const uint32_t hi = std::min<uint64_t>((uint64_t)(s + 1) << p.shift[k], I);
        uint64_t i = b;
        for (uint32_t r = lo; r < hi; ++r) {
            rp[r] = i;
            while (i < e && ik[i] == r) ++i;
        }
        rp[hi] = i;
    }
}

int download_copy(Plan& p, const Slab& s, DnpImage& img, int k) {
    img.vals[k].resize(p.nnz);
    DGPU_CUDA(cudaMemcpyAsync(img.vals[k].data(), s.vals, p.nnz * 4, cudaMemcpyDeviceToHost,
                              p.stream));
    for (int m = 0; m < p.N; ++m) {
        img.idx[k][m].resize(p.nnz);
        DGPU_CUDA(cudaMemcpyAsync(img.idx[k][m].data(), s.idx[m], p.nnz * 4,
                                  cudaMemcpyDeviceToHost, p.stream));
    }
    return DGPU_OK;
}

int plan_to_dnp(Plan& p, DnpImage& img) {
    if (p.layout == DGPU_LAYOUT_PINGPONG && p.next_mode != 0) {
        set_error("dgpu_plan_save_dnp: the PingPong slab is remapped for mode %d; save between "
                  "sweeps (next mode 0)", p.next_mode);
        return DGPU_ERR_ORDER;
    }
    const int N = p.N;
    img.layout = p.layout;
    img.N = N;
    img.nnz = p.nnz;
    for (int n = 0; n < DGPU_MAX_MODES; ++n) img.dims[n] = n < N ? p.dims[n] : 0u;
    img.threads = p.T;
    img.tnorm_sq = 0.0;             // in-core tensors carry no cached norm
    if (p.layout == DGPU_LAYOUT_MORTON) {
        for (int n = 0; n < N; ++n) {
            img.mmask[n] = p.mmask[n];
            img.mbits[n] = p.mbits[n];
        }
        img.mkeys.resize(p.nnz);
        img.mvals.resize(p.nnz);
        DGPU_CUDA(cudaMemcpyAsync(img.mkeys.data(), p.mkeys, p.nnz * 8, cudaMemcpyDeviceToHost,
                                  p.stream));
        DGPU_CUDA(cudaMemcpyAsync(img.mvals.data(), p.mvals, p.nnz * 4, cudaMemcpyDeviceToHost,
                                  p.stream));
        return sync_checked(p);
    }
    img.shard_size = kShardSize;
    img.inplace_mode = 0;
    for (int n = 0; n < N; ++n) {
        img.K[n] = p.K[n];
        img.mn[n] = p.mn[n];
        img.shift[n] = p.shift[n];
        img.afl[n] = p.afl[n];
        img.kclass[n] = (uint32_t)p.kclass[n];
    }
    img.remap_stride = ((uint64_t)p.K[1 % N] + 7) & ~(uint64_t)7;
    img.sbeg = p.sbeg;
    img.send = p.send;
    img.sched = p.sched;
    const int copies = p.layout == DGPU_LAYOUT_NCOPY ? N : 1;
    for (int k = 0; k < copies; ++k)
        DGPU_TRY(download_copy(p, p.slab[p.layout == DGPU_LAYOUT_NCOPY ? k : p.cur], img, k));
    DGPU_TRY(sync_checked(p));
    img.touched.assign(N, {});
    img.touched_count.assign(N, 0);
    img.cursor.assign(N, {});
    // per mode: bitmap + cursor table, one host thread each
    std::vector<std::thread> th;
    for (int n = 0; n < N; ++n)
        th.emplace_back([&, n] {
            touched_rows(img.idx[0][n], p.dims[n], img.touched[n], img.touched_count[n]);
            cursor_table(p, n, img.idx[0][n], img.idx[0][(n + 1) % N], img.cursor[n]);
        });
    for (auto& t : th) t.join();
    if (p.layout == DGPU_LAYOUT_NCOPY) {
        for (int k = 0; k < N; ++k) {
            img.fiber_sorted[k] = (p.fiber && p.kclass[k] == 2) ? 1 : 0;
            img.csr[k] = img.fiber_sorted[k];
            if (img.csr[k]) row_pointers(p, k, img.idx[k][k], img.rowptr[k]);
        }
    }
    return DGPU_OK;
}

}  // namespace

extern "C" {

int dgpu_dnp_peek(const char* path, dgpu_dnp_info* info) {
    if (!path || !info) {
        set_error("dgpu_dnp_peek: null argument");
        return DGPU_ERR_ARG;
    }
    std::memset(info, 0, sizeof(*info));
    DnpImage img;
    uint32_t kind = 0;
    try {
        DGPU_TRY(dnp_read(path, 0, true, img, &kind));
    } catch (...) {
        set_error("dgpu_dnp_peek: host allocation failed");
        return DGPU_ERR_NOMEM;
    }
    info->layout_kind = (int)kind;
    info->num_modes = img.N;
    info->nnz = img.nnz;
    for (int n = 0; n < DGPU_MAX_MODES; ++n) info->mode_size[n] = img.dims[n];
    info->num_threads = img.threads;
    return DGPU_OK;
}

int dgpu_plan_create_from_dnp(const char* path, const dgpu_plan_opts* o, dgpu_plan** out) {
    if (!path || !o || !out) {
        set_error("dgpu_plan_create_from_dnp: null argument");
        return DGPU_ERR_ARG;
    }
    *out = nullptr;
    if (o->threads < 1) {
        set_error("dgpu_plan_create_from_dnp: threads %d < 1", o->threads);
        return DGPU_ERR_ARG;
    }
    if (o->rank < 1 || o->rank > 1024) {
        set_error("dgpu_plan_create_from_dnp: rank %d outside [1,1024]", o->rank);
        return DGPU_ERR_ARG;
    }
    if (o->precision != DGPU_PREC_FP32 && o->precision != DGPU_PREC_BF16) {
        set_error("dgpu_plan_create_from_dnp: unknown precision %d", o->precision);
        return DGPU_ERR_ARG;
    }
    if (o->accum < DGPU_ACCUM_AUTO || o->accum > DGPU_ACCUM_PRIVATE) {
        set_error("dgpu_plan_create_from_dnp: unknown accumulation mode %d", o->accum);
        return DGPU_ERR_ARG;
    }
    std::unique_ptr<DnpImage> img;
    try {
        img = std::make_unique<DnpImage>();
        DGPU_TRY(dnp_read(path, o->threads, false, *img, nullptr));
    } catch (...) {
        set_error("dgpu_plan_create_from_dnp: host allocation failed reading '%s'", path);
        return DGPU_ERR_NOMEM;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("dgpu_plan_create_from_dnp: no CUDA device available");
        return DGPU_ERR_CUDA;
    }
    if (o->device < 0 || o->device >= ndev) {
        set_error("dgpu_plan_create_from_dnp: device %d outside [0,%d)", o->device, ndev);
        return DGPU_ERR_ARG;
    }
    Plan* p = new (std::nothrow) Plan();
    if (!p) {
        set_error("dgpu_plan_create_from_dnp: host OOM");
        return DGPU_ERR_NOMEM;
    }
    int rc;
    try {
        rc = plan_build_dnp(*p, *img, *o);
    } catch (...) {
        set_error("dgpu_plan_create_from_dnp: host allocation failed");
        rc = DGPU_ERR_NOMEM;
    }
    if (rc != DGPU_OK) {
        delete p;
        return rc;
    }
    *out = reinterpret_cast<dgpu_plan*>(p);
    return DGPU_OK;
}

int dgpu_plan_save_dnp(const dgpu_plan* plan, const char* path) {
    if (!plan || !path) {
        set_error("dgpu_plan_save_dnp: null argument");
        return DGPU_ERR_ARG;
    }
    Plan& p = *const_cast<Plan*>(reinterpret_cast<const Plan*>(plan));
    DGPU_CUDA(cudaSetDevice(p.device));
    try {
        auto img = std::make_unique<DnpImage>();
        DGPU_TRY(plan_to_dnp(p, *img));
        return dnp_write(path, *img);
    } catch (...) {
        set_error("dgpu_plan_save_dnp: host allocation failed");
        return DGPU_ERR_NOMEM;
    }
}

}  // extern "C"
