// ============================================================================
//  io.cu -- host-side tensor loaders and dumps of libdynasor_b200.so.
//
//  Same formats and dispatch as the reference (src/dynasor_io.cpp):
//    * .tns text: "<i0> ... <iN-1> <val>" per line, 1-based indices, '#'
//      comments, optional SPLATT header (a line with N, then a line with
//      the N mode sizes); mode sizes grow to max index + 1.  [:576-745]
//    * .dnb binary cache "DNB1" v1: magic, version, value_bytes, index_bytes,
//      num_modes, nnz (u64), mode_size[8], reserved[7], vals, idx[0..N-1];
//      written to <path>.tmp and renamed.  [:747-893]
//    * load_coo_tensor: use <path>.dnb when it exists, holds a header and is
//      not older than <path>; else parse the text and (optionally) write the
//      cache.  [:776-803, :1184-1261]
//    * DYFM factor dump: magic, version, value_bytes, rank, rows (u64), then
//      rows x rank float32 with the padding stripped.  [:1287-1348]
//  Duplicates are kept, as in the reference loaders.
// ============================================================================
#include "dgpu_internal.h"

#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

using namespace dgpu;

namespace {

constexpr char kDnbMagic[4] = {'D', 'N', 'B', '1'};
constexpr uint32_t kDnbVersion = 1;
constexpr size_t kDnbHeader = 4 + 4 + 4 + 4 + 4 + 8 + 4 * DGPU_MAX_MODES + 4 * 7;

void coo_reset(dgpu_coo* c) {
    std::memset(c, 0, sizeof(*c));
}

int coo_alloc(dgpu_coo* c, int N, uint64_t nnz) {
    c->num_modes = N;
    c->nnz = nnz;
    const size_t n = nnz ? nnz : 1;
    c->vals = static_cast<float*>(std::malloc(n * sizeof(float)));
    if (!c->vals) return DGPU_ERR_NOMEM;
    for (int m = 0; m < N; ++m) {
        c->idx[m] = static_cast<uint32_t*>(std::malloc(n * sizeof(uint32_t)));
        if (!c->idx[m]) return DGPU_ERR_NOMEM;
    }
    return DGPU_OK;
}

bool dnb_is_fresh(const std::string& tns, const std::string& dnb) {
    struct stat b {};
    if (::stat(dnb.c_str(), &b) != 0) return false;
    if ((uint64_t)b.st_size < (uint64_t)kDnbHeader) return false;
    struct stat a {};
    if (::stat(tns.c_str(), &a) != 0) return true;   // no source: trust the cache
    return b.st_mtime >= a.st_mtime;
}

int parse_tns(const char* path, dgpu_coo* out) {
    std::FILE* fp = std::fopen(path, "rb");
    if (!fp) {
        set_error("cannot open tensor file '%s' (%s)", path, std::strerror(errno));
        return DGPU_ERR_IO;
    }
    int N = 0;
    uint32_t dims[DGPU_MAX_MODES] = {0};
    std::vector<float> vals;
    std::vector<uint32_t> idx[DGPU_MAX_MODES];
    int header_expect = 0;
    bool header_done = false;
    char line[8192];
    double tok[DGPU_MAX_MODES + 1];
    int rc = DGPU_OK;
    while (std::fgets(line, sizeof line, fp)) {
        char* p = line;
        while (*p && std::isspace((unsigned char)*p)) ++p;
        if (*p == '\0' || *p == '#') continue;
        int nt = 0;
        while (*p) {
            while (*p && std::isspace((unsigned char)*p)) ++p;
            if (!*p) break;
            if (nt >= DGPU_MAX_MODES + 1) {
                set_error("%s: line has more than %d tokens", path, DGPU_MAX_MODES + 1);
                rc = DGPU_ERR_IO;
                break;
            }
            char* end = nullptr;
            const double v = std::strtod(p, &end);
            if (end == p) {
                set_error("%s: cannot parse token near: %.40s", path, p);
                rc = DGPU_ERR_IO;
                break;
            }
            tok[nt++] = v;
            p = end;
        }
        if (rc != DGPU_OK) break;
        if (!header_done) {
            if (nt == 1 && N == 0 && tok[0] == (double)(int)tok[0] && tok[0] >= 2 &&
                tok[0] <= DGPU_MAX_MODES) {
                N = (int)tok[0];
                header_expect = N;
                continue;
            }
            if (header_expect > 0 && nt == header_expect) {
                for (int n = 0; n < nt; ++n) dims[n] = (uint32_t)tok[n];
                header_expect = 0;
                header_done = true;
                continue;
            }
            header_done = true;
        }
        if (nt < 2) continue;
        const int nm = nt - 1;
        if (N == 0) {
            if (nm > DGPU_MAX_MODES) {
                set_error("%s: tensor has %d modes (max %d)", path, nm, DGPU_MAX_MODES);
                rc = DGPU_ERR_IO;
                break;
            }
            N = nm;
        } else if (nm != N) {
            set_error("%s: inconsistent mode count (expected %d, got %d)", path, N, nm);
            rc = DGPU_ERR_IO;
            break;
        }
        for (int n = 0; n < nm; ++n) {
            const long long i1 = (long long)tok[n];
            if (i1 <= 0) {
                set_error("%s: non-positive index %lld", path, i1);
                rc = DGPU_ERR_IO;
                break;
            }
            const uint32_t i0 = (uint32_t)(i1 - 1);
            idx[n].push_back(i0);
            if (i0 + 1 > dims[n]) dims[n] = i0 + 1;
        }
        if (rc != DGPU_OK) break;
        vals.push_back((float)tok[nm]);
    }
    std::fclose(fp);
    if (rc != DGPU_OK) return rc;
    if (N == 0) {
        set_error("%s: no nonzeros", path);
        return DGPU_ERR_EMPTY;
    }
    DGPU_TRY(coo_alloc(out, N, vals.size()));
    for (int n = 0; n < N; ++n) out->mode_size[n] = dims[n];
    std::memcpy(out->vals, vals.data(), vals.size() * sizeof(float));
    for (int n = 0; n < N; ++n) std::memcpy(out->idx[n], idx[n].data(), vals.size() * 4);
    return DGPU_OK;
}

int read_dnb(const char* path, dgpu_coo* out) {
    std::FILE* fp = std::fopen(path, "rb");
    if (!fp) {
        set_error("cannot open '%s' (%s)", path, std::strerror(errno));
        return DGPU_ERR_IO;
    }
    char magic[4];
    uint32_t version, vb, ib, nm;
    uint64_t nnz;
    uint32_t ms[DGPU_MAX_MODES];
    uint32_t reserved[7];
    const bool ok = std::fread(magic, 4, 1, fp) == 1 && std::fread(&version, 4, 1, fp) == 1 &&
                    std::fread(&vb, 4, 1, fp) == 1 && std::fread(&ib, 4, 1, fp) == 1 &&
                    std::fread(&nm, 4, 1, fp) == 1 && std::fread(&nnz, 8, 1, fp) == 1 &&
                    std::fread(ms, sizeof ms, 1, fp) == 1 &&
                    std::fread(reserved, sizeof reserved, 1, fp) == 1;
    if (!ok || std::memcmp(magic, kDnbMagic, 4) != 0 || version != kDnbVersion || vb != 4 ||
        ib != 4 || nm == 0 || nm > DGPU_MAX_MODES || nnz == 0) {
        std::fclose(fp);
        set_error("%s: not a valid DNB1 file", path);
        return DGPU_ERR_IO;
    }
    int rc = coo_alloc(out, (int)nm, nnz);
    if (rc == DGPU_OK) {
        for (uint32_t n = 0; n < nm; ++n) out->mode_size[n] = ms[n];
        if (std::fread(out->vals, 4, nnz, fp) != nnz) rc = DGPU_ERR_IO;
        for (uint32_t n = 0; n < nm && rc == DGPU_OK; ++n)
            if (std::fread(out->idx[n], 4, nnz, fp) != nnz) rc = DGPU_ERR_IO;
        if (rc == DGPU_ERR_IO) set_error("%s: truncated DNB1 payload", path);
    }
    std::fclose(fp);
    return rc;
}

}  // namespace

extern "C" {

void dgpu_coo_free(dgpu_coo* c) {
    if (!c) return;
    std::free(c->vals);
    for (int n = 0; n < DGPU_MAX_MODES; ++n) std::free(c->idx[n]);
    coo_reset(c);
}

int dgpu_load_tns(const char* path, dgpu_coo* out) {
    if (!path || !out) { set_error("dgpu_load_tns: null argument"); return DGPU_ERR_ARG; }
    coo_reset(out);
    const int rc = parse_tns(path, out);
    if (rc != DGPU_OK) dgpu_coo_free(out);
    return rc;
}

int dgpu_load_dnb(const char* path, dgpu_coo* out) {
    if (!path || !out) { set_error("dgpu_load_dnb: null argument"); return DGPU_ERR_ARG; }
    coo_reset(out);
    const int rc = read_dnb(path, out);
    if (rc != DGPU_OK) dgpu_coo_free(out);
    return rc;
}

int dgpu_save_dnb(const char* path, const dgpu_coo* t) {
    if (!path || !t || !t->vals || t->nnz == 0 || t->num_modes <= 0 ||
        t->num_modes > DGPU_MAX_MODES) {
        set_error("dgpu_save_dnb: bad argument");
        return DGPU_ERR_ARG;
    }
    const std::string tmp = std::string(path) + ".tmp";
    std::FILE* fp = std::fopen(tmp.c_str(), "wb");
    if (!fp) { set_error("cannot write '%s'", tmp.c_str()); return DGPU_ERR_IO; }
    const uint32_t version = kDnbVersion, vb = 4, ib = 4, nm = (uint32_t)t->num_modes;
    const uint64_t nnz = t->nnz;
    uint32_t ms[DGPU_MAX_MODES] = {0};
    for (int n = 0; n < t->num_modes; ++n) ms[n] = t->mode_size[n];
    const uint32_t reserved[7] = {0};
    bool ok = std::fwrite(kDnbMagic, 4, 1, fp) == 1 && std::fwrite(&version, 4, 1, fp) == 1 &&
              std::fwrite(&vb, 4, 1, fp) == 1 && std::fwrite(&ib, 4, 1, fp) == 1 &&
              std::fwrite(&nm, 4, 1, fp) == 1 && std::fwrite(&nnz, 8, 1, fp) == 1 &&
              std::fwrite(ms, sizeof ms, 1, fp) == 1 &&
              std::fwrite(reserved, sizeof reserved, 1, fp) == 1 &&
              std::fwrite(t->vals, 4, nnz, fp) == nnz;
    for (int n = 0; ok && n < t->num_modes; ++n)
        ok = t->idx[n] && std::fwrite(t->idx[n], 4, nnz, fp) == nnz;
    std::fclose(fp);
    if (!ok) {
        std::remove(tmp.c_str());
        set_error("dgpu_save_dnb: write failed for '%s'", path);
        return DGPU_ERR_IO;
    }
    std::remove(path);
    if (std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        set_error("dgpu_save_dnb: rename to '%s' failed", path);
        return DGPU_ERR_IO;
    }
    return DGPU_OK;
}

int dgpu_load_coo_tensor(const char* path, int use_cache, dgpu_coo* out) {
    if (!path || !out) { set_error("dgpu_load_coo_tensor: null argument"); return DGPU_ERR_ARG; }
    coo_reset(out);
    const std::string dnb = std::string(path) + ".dnb";
    if (use_cache && dnb_is_fresh(path, dnb)) {
        if (read_dnb(dnb.c_str(), out) == DGPU_OK) return DGPU_OK;
        dgpu_coo_free(out);
        std::fprintf(stderr, "[io] WARN: stale or invalid binary cache '%s', reparsing text\n",
                     dnb.c_str());
    }
    int rc = parse_tns(path, out);
    if (rc != DGPU_OK) {
        dgpu_coo_free(out);
        return rc;
    }
    if (use_cache) dgpu_save_dnb(dnb.c_str(), out);   // best effort, as the reference
    return DGPU_OK;
}

int dgpu_dump_factor_bin(const char* path, const float* data, uint32_t rows, int rank,
                         int rank_padded) {
    if (!path || !data || rank <= 0 || rank_padded < rank) {
        set_error("dgpu_dump_factor_bin: bad argument");
        return DGPU_ERR_ARG;
    }
    std::FILE* fp = std::fopen(path, "wb");
    if (!fp) { set_error("cannot write '%s'", path); return DGPU_ERR_IO; }
    const char magic[4] = {'D', 'Y', 'F', 'M'};
    const uint32_t version = 1, vb = 4, r = (uint32_t)rank;
    const uint64_t rw = rows;
    bool ok = std::fwrite(magic, 4, 1, fp) == 1 && std::fwrite(&version, 4, 1, fp) == 1 &&
              std::fwrite(&vb, 4, 1, fp) == 1 && std::fwrite(&r, 4, 1, fp) == 1 &&
              std::fwrite(&rw, 8, 1, fp) == 1;
    for (uint32_t i = 0; ok && i < rows; ++i)
        ok = std::fwrite(data + (size_t)i * rank_padded, 4, (size_t)rank, fp) == (size_t)rank;
    std::fclose(fp);
    if (!ok) {
        std::remove(path);
        set_error("dgpu_dump_factor_bin: write failed");
        return DGPU_ERR_IO;
    }
    return DGPU_OK;
}

}  // extern "C"
