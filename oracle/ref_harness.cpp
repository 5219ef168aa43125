// ============================================================================
//  ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
//  A thin extern "C" shim over the UNMODIFIED Dynasor+ reference sources
//  (compiled from the reference tree by oracle/Makefile into oracle/_ref/).
//  It lets the pytest suite and bench.py's CPU-baseline leg drive the
//  reference's own code path through ctypes:
//
//    * build_flycoo            (src/dynasor_preprocess.cpp:2013-2163)
//    * SpmttkrpSweep::process  (src/dynasor.cpp:352-539)
//    * spmttkrp_reference      (src/dynasor_reference.cpp:18-50)
//    * cpals                   (src/dynasor_cpals.cpp:120-396)
//    * save_dnp_tensor / load_dnp_tensor (src/dynasor_dnp.cpp:639-803)
//    * build_morton_layout / spmttkrp_all_modes_morton
//                              (src/dynasor_morton.cpp:143-352, 612-784)
//
//  and to read back the FLYCOO plan tables and the SoA slab after each
//  process(n), which is what the bit-exact remap parity tests compare.
//
//  Nothing in the product library links or loads this file.
// ============================================================================
#include "dynasor_common.h"
#include "dynasor_cpals.h"
#include "dynasor_dnp.h"
#include "dynasor_morton.h"
#include "dynasor_linalg.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <unistd.h>
#include <fcntl.h>

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace dynasor;

namespace {

// Scoped redirect of stdout to /dev/null: the reference prints banners on
// every call; tests only need the data.
struct Quiet {
    int saved = -1;
    explicit Quiet(bool on) {
        if (!on) return;
        std::fflush(stdout);
        saved = dup(1);
        int fd = open("/dev/null", O_WRONLY);
        if (fd >= 0) { dup2(fd, 1); close(fd); }
    }
    ~Quiet() {
        if (saved < 0) return;
        std::fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

struct RefHandle {
    Tensor          T;
    FactorMatrices  F;
    SpmttkrpSweep*  sweep = nullptr;
    int             threads = 1;
    bool            quiet = true;
    ~RefHandle() { delete sweep; F.free_all(); }
};

void set_env(const char* k, const char* v) {
    if (v && *v) setenv(k, v, 1);
    else unsetenv(k);
}

} // namespace

extern "C" {

// Create a tensor from 0-based COO arrays (host copies are taken).
void* ref_create(int N, uint64_t nnz, const uint32_t* dims,
                 const float* vals, const uint32_t* const* idx, int quiet)
{
    auto* h = new RefHandle();
    h->quiet = quiet != 0;
    h->T.allocate_elements(nnz, N);
    for (int n = 0; n < N; ++n) h->T.mode_size[n] = dims[n];
    std::memcpy(h->T.vals, vals, nnz * sizeof(float));
    for (int n = 0; n < N; ++n)
        std::memcpy(h->T.idx_buf[n], idx[n], nnz * sizeof(uint32_t));
    return h;
}

void ref_destroy(void* hp) { delete static_cast<RefHandle*>(hp); }

// build_flycoo with a forced layout ("pingpong" | "ncopy" | "inplace").
// CSR compaction is disabled so every NCopy copy keeps all index columns.
int ref_build_flycoo(void* hp, int threads, const char* layout)
{
    auto* h = static_cast<RefHandle*>(hp);
    h->threads = threads;
#ifdef _OPENMP
    omp_set_num_threads(threads);
#endif
    set_env("DYN_LAYOUT", layout);
    set_env("DYN_NCOPY_CSR_COMPACT", "0");
    Quiet q(h->quiet);
    build_flycoo(h->T, threads, nullptr, 16);
    return (int)h->T.layout;
}

// Plan scalars per mode: mn_shift, shards_per_mode, kernel_class.
void ref_plan_modes(void* hp, int* mn_shift, uint32_t* shards, int* kclass,
                    double* avg_fiber)
{
    auto* h = static_cast<RefHandle*>(hp);
    for (int n = 0; n < h->T.num_modes; ++n) {
        mn_shift[n]  = h->T.mn_shift[n];
        shards[n]    = h->T.shards_per_mode[n];
        kclass[n]    = (int)h->T.kernel_class[n];
        avg_fiber[n] = h->T.avg_fiber_len[n];
    }
}

// shard_begin / shard_end of mode n (K entries each).
void ref_plan_shards(void* hp, int n, uint64_t* begin, uint64_t* end)
{
    auto* h = static_cast<RefHandle*>(hp);
    const size_t K = h->T.shard_begin[n].size();
    std::memcpy(begin, h->T.shard_begin[n].data(), K * sizeof(uint64_t));
    std::memcpy(end,   h->T.shard_end[n].data(),   K * sizeof(uint64_t));
}

// LPT schedule of mode n flattened: counts[tid] then the concatenated
// shard lists.  Returns the total number of listed shards.
int ref_plan_schedule(void* hp, int n, uint32_t* counts, uint32_t* flat)
{
    auto* h = static_cast<RefHandle*>(hp);
    int k = 0;
    const auto& L = h->T.ss_list[n];
    for (size_t t = 0; t < L.size(); ++t) {
        counts[t] = (uint32_t)L[t].size();
        for (sid_t s : L[t]) flat[k++] = s;
    }
    return k;
}

// Cursor table precomp_thr_off[n] (threads * stride entries) and stride.
size_t ref_plan_cursors(void* hp, int n, uint64_t* out)
{
    auto* h = static_cast<RefHandle*>(hp);
    const auto& v = h->T.precomp_thr_off[n];
    if (out) std::memcpy(out, v.data(), v.size() * sizeof(uint64_t));
    return v.size();
}

// Current primary slab (what the next process(n) reads in PingPong).
void ref_get_slab(void* hp, float* vals, uint32_t* const* idx)
{
    auto* h = static_cast<RefHandle*>(hp);
    const uint64_t nnz = h->T.nnz;
    std::memcpy(vals, h->T.vals, nnz * sizeof(float));
    for (int n = 0; n < h->T.num_modes; ++n)
        std::memcpy(idx[n], h->T.idx_buf[n], nnz * sizeof(uint32_t));
}

// NCopy copy k (valid after a build with layout "ncopy").
int ref_get_ncopy(void* hp, int k, float* vals, uint32_t* const* idx)
{
    auto* h = static_cast<RefHandle*>(hp);
    if (h->T.layout != Layout::NCopy || !h->T.ncopy_vals[k]) return -1;
    const uint64_t nnz = h->T.nnz;
    std::memcpy(vals, h->T.ncopy_vals[k], nnz * sizeof(float));
    for (int n = 0; n < h->T.num_modes; ++n) {
        if (!h->T.ncopy_idx[k][n]) return -2;
        std::memcpy(idx[n], h->T.ncopy_idx[k][n], nnz * sizeof(uint32_t));
    }
    return h->T.ncopy_fiber_sorted[k] ? 1 : 0;
}

// Run the reference's fiber sort of mode n on the current primary slab.
void ref_fiber_sort(void* hp, int n)
{
    auto* h = static_cast<RefHandle*>(hp);
    Quiet q(h->quiet);
    fiber_sort_shards(h->T, n);
}

// Allocate factors at rank R.  Returns rank_padded.
int ref_factors(void* hp, int R)
{
    auto* h = static_cast<RefHandle*>(hp);
    h->F.allocate(h->T.num_modes, h->T.mode_size, R);
    return h->F.rank_padded;
}

void ref_set_Y(void* hp, int n, const float* Y)
{
    auto* h = static_cast<RefHandle*>(hp);
    std::memcpy(h->F.Y[n], Y,
                (size_t)h->T.mode_size[n] * h->F.rank_padded * sizeof(float));
}

void ref_get_Y(void* hp, int n, float* Y)
{
    auto* h = static_cast<RefHandle*>(hp);
    std::memcpy(Y, h->F.Y[n],
                (size_t)h->T.mode_size[n] * h->F.rank_padded * sizeof(float));
}

void ref_get_Yhat(void* hp, int n, float* out)
{
    auto* h = static_cast<RefHandle*>(hp);
    std::memcpy(out, h->F.Yhat[n],
                (size_t)h->T.mode_size[n] * h->F.rank_padded * sizeof(float));
}

// SpmttkrpSweep with DYN_FIBER_OFF set from `fiber_off`.
void ref_sweep_begin(void* hp, int fiber_off)
{
    auto* h = static_cast<RefHandle*>(hp);
    delete h->sweep;
    set_env("DYN_FIBER_OFF", fiber_off ? "1" : nullptr);
    Quiet q(h->quiet);
    h->sweep = new SpmttkrpSweep(h->T, h->F, h->threads, false);
}

double ref_sweep_process(void* hp, int n)
{
    auto* h = static_cast<RefHandle*>(hp);
    Quiet q(h->quiet);
    const double t0 = h->sweep->elapsed_s();
    h->sweep->process(n);
    return h->sweep->elapsed_s() - t0;
}

// Single-thread textbook MTTKRP over the current slab (all modes).
void ref_reference_mttkrp(void* hp)
{
    auto* h = static_cast<RefHandle*>(hp);
    Quiet q(h->quiet);
    spmttkrp_reference(h->T, h->F);
}

// CP-ALS.  kernel: 0 = Gauss-Seidel, 1 = Jacobi.  fit_hist must hold
// max_iters doubles; lambda_out rank floats.  Returns iters done.
int ref_cpals(void* hp, int max_iters, double tol, uint64_t seed,
              int kernel, float ridge, int fiber_off,
              double* fit_hist, float* lambda_out,
              double* total_s, double* mttkrp_s)
{
    auto* h = static_cast<RefHandle*>(hp);
    set_env("DYN_FIBER_OFF", fiber_off ? "1" : nullptr);
    CpOptions opt;
    opt.max_iters   = max_iters;
    opt.tol         = tol;
    opt.seed        = seed;
    opt.num_threads = h->threads;
    opt.ridge       = ridge;
    opt.verbose     = !h->quiet;
    opt.kernel      = kernel ? CpKernel::Jacobi : CpKernel::GaussSeidel;
    CpResult r;
    {
        Quiet q(h->quiet);
        r = cpals(h->T, h->F, opt);
    }
    for (int i = 0; i < r.iters_done; ++i) fit_hist[i] = r.fit_history[i];
    for (size_t i = 0; i < r.lambda.size(); ++i) lambda_out[i] = r.lambda[i];
    if (total_s)  *total_s  = r.total_time_s;
    if (mttkrp_s) *mttkrp_s = r.mttkrp_time_s;
    return r.iters_done;
}

// One full sweep through the reference's legacy driver, timed by the
// reference itself (the `[summary] dynasor = t s` figure).
double ref_spmttkrp_dynasor(void* hp)
{
    auto* h = static_cast<RefHandle*>(hp);
    Quiet q(h->quiet);
    return spmttkrp_dynasor(h->T, h->F, h->threads);
}

int ref_simd_width_hint(void) {
#if defined(__AVX512F__)
    return 16;
#elif defined(__AVX2__)
    return 8;
#else
    return 4;
#endif
}

// build_morton_layout on a built (PingPong / InPlace) tensor; 0 on success.
int ref_build_morton(void* hp)
{
    auto* h = static_cast<RefHandle*>(hp);
    Quiet q(h->quiet);
    return build_morton_layout(h->T, h->threads) ? 0 : -1;
}

// Morton masks / bits and (when not null) the sorted keys and values.
int ref_morton_get(void* hp, uint64_t* mask, uint8_t* bits, uint64_t* keys, float* vals)
{
    auto* h = static_cast<RefHandle*>(hp);
    if (h->T.layout != Layout::Morton || !h->T.morton_keys) return -1;
    for (int n = 0; n < h->T.num_modes; ++n) {
        mask[n] = h->T.morton_mask[n];
        bits[n] = h->T.morton_bits[n];
    }
    if (keys) std::memcpy(keys, h->T.morton_keys, h->T.nnz * sizeof(uint64_t));
    if (vals) std::memcpy(vals, h->T.morton_vals, h->T.nnz * sizeof(float));
    return 0;
}

// spmttkrp_all_modes_morton into F.Yhat; returns its seconds.
double ref_all_modes_morton(void* hp)
{
    auto* h = static_cast<RefHandle*>(hp);
    Quiet q(h->quiet);
    return spmttkrp_all_modes_morton(h->T, h->F, h->threads);
}

// The reference's .dnp writer on the built tensor; 0 on success.
int ref_save_dnp(void* hp, const char* path)
{
    auto* h = static_cast<RefHandle*>(hp);
    Quiet q(h->quiet);
    return save_dnp_tensor(path, h->T, h->threads) ? 0 : -1;
}

// A tensor loaded by the reference's .dnp reader (runtime-only mode), or
// null when the reader rejects the file.
void* ref_load_dnp(const char* path, int threads, int quiet)
{
    auto* h = new RefHandle();
    h->quiet = quiet != 0;
    h->threads = threads;
#ifdef _OPENMP
    omp_set_num_threads(threads);
#endif
    bool ok;
    {
        Quiet q(h->quiet);
        ok = load_dnp_tensor(path, h->T, threads);
    }
    if (!ok) { delete h; return nullptr; }
    // The reference's PingPong loader (load_soa_slab, src/dynasor_dnp.cpp:
    // 497-504) materialises only the primary slab; its first remap then
    // writes through the unallocated scratch slab.  Materialise it here, as
    // build_flycoo does (src/dynasor_preprocess.cpp:2029).
    if (h->T.layout == Layout::PingPong || h->T.layout == Layout::InPlace) h->T.ensure_scratch();
    return h;
}

// dyn_build_compute_plan on the built tensor (src/dynasor_preprocess.cpp:
// 1179-1363): the CP-ALS kernel it picks (0 GS, 1 Jacobi), its reason and
// the per-mode kernel class (0 Element, 1 Fiber, 2 FiberCSR).  layout is
// the layout the tensor was built with ("pingpong" | "ncopy").
int ref_compute_plan(void* hp, int rank_padded, int threads, const char* layout,
                     const char* kernel_cli, char* reason, int reason_cap, int* per_mode)
{
    auto* h = static_cast<RefHandle*>(hp);
    ComputePlan p;
    {
        Quiet q(h->quiet);
        p = dyn_build_compute_plan(h->T, rank_padded, threads, layout ? layout : "",
                                   "off", kernel_cli ? kernel_cli : "");
    }
    if (reason && reason_cap > 0) std::snprintf(reason, (size_t)reason_cap, "%s", p.kernel_reason);
    for (int n = 0; n < h->T.num_modes; ++n) per_mode[n] = (int)p.per_mode[n];
    return p.kernel_enum;
}

} // extern "C"
