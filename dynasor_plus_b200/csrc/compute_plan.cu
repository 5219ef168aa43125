// ============================================================================
//  compute_plan.cu -- the run-time decisions of a plan in one record
//  (host code only).
//
//  Replaces ComputePlan / dyn_build_compute_plan / dyn_print_compute_plan
//  (include/dynasor_common.h:244-320, src/dynasor_preprocess.cpp:1179-1399).
//  The reference collects its scattered dispatch rules there: Jacobi
//  (all-modes) or Gauss-Seidel for CP-ALS, the per-mode kernel class, and
//  two CPU tuning switches (far prefetch, JIT) that have no device meaning.
//
//  The CP-ALS kernel rule is the reference's, clause for clause, so a
//  caller who leaves the kernel on "auto" gets the algorithm the reference
//  would run for the same tensor, worker count and host (the all-modes
//  memory clause is the reference's host-RAM budget for its per-thread
//  output copies, evaluated the same way):
//    * Morton layout                          -> Jacobi (only driver there)
//    * nnz < 1,000,000                        -> Gauss-Seidel
//    * (N == 3 and Rp >= 64) or Rp >= 128     -> Gauss-Seidel
//    * T * sum_n round64(I_n * Rp * 4) >= min(MemAvailable / 4, 8 GiB)
//                                             -> Gauss-Seidel
//    * otherwise                              -> Jacobi
//  DYN_CP_KERNEL (the reference's variable) overrides the caller's choice.
//  The per-mode class is the reference's (FiberCSR on fiber-sorted NCopy
//  copies, Fiber on DenseFiber modes or average fiber length >= 32, else
//  Element); beside it the record carries what this engine runs for the
//  mode: the accumulation scheme and the rank tile.
// ============================================================================
#include "dgpu_internal.h"

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

namespace dgpu {

int mttkrp_scheme(const Plan& p, int n);

namespace {

std::string lower(const char* s) {
    std::string out = s ? s : "";
    for (char& c : out) c = (char)std::tolower((unsigned char)c);
    return out;
}

bool is_jacobi_word(const std::string& k) {
    return k == "jacobi" || k == "all-modes" || k == "all_modes" || k == "js";
}

bool is_gs_word(const std::string& k) {
    return k == "gauss-seidel" || k == "gs" || k == "classical" || k == "per-mode" ||
           k == "per_mode";
}

// MemAvailable of /proc/meminfo in bytes (0 when absent), as the reference's
// dyn_memory_available_bytes (src/dynasor_io.cpp:93-115) reads it.
uint64_t host_available_bytes() {
    FILE* fp = std::fopen("/proc/meminfo", "r");
    if (!fp) return 0;
    char line[256];
    uint64_t avail = 0;
    while (std::fgets(line, sizeof(line), fp)) {
        unsigned long long kb = 0;
        if (std::sscanf(line, "MemAvailable: %llu kB", &kb) == 1) {
            avail = (uint64_t)kb * 1024ull;
            break;
        }
    }
    std::fclose(fp);
    return avail;
}

void copy_str(char* dst, size_t cap, const char* src) {
    std::snprintf(dst, cap, "%s", src);
}

}  // namespace

int compute_plan_decide(const dgpu_compute_plan_input& in, const char* kernel_cli,
                        dgpu_compute_plan& cp) {
    if (in.num_modes < 1 || in.num_modes > kMaxModes) {
        set_error("compute plan: %d modes (1..%d)", in.num_modes, kMaxModes);
        return DGPU_ERR_ARG;
    }
    if (in.rank_padded < 1 || in.threads < 1) {
        set_error("compute plan: rank_padded %d / threads %d must be >= 1", in.rank_padded,
                  in.threads);
        return DGPU_ERR_ARG;
    }
    std::memset(&cp, 0, sizeof(cp));
    const int N = in.num_modes, Rp = in.rank_padded;
    cp.layout = in.layout;
    cp.num_modes = N;
    cp.rank_padded = Rp;
    cp.threads = in.threads;
    cp.precision = DGPU_PREC_FP32;
    uint64_t per_thread = 0, factors = 0;
    for (int n = 0; n < N; ++n) {
        const uint64_t b = (uint64_t)in.mode_size[n] * (uint64_t)Rp * 4ull;
        per_thread += (b + 63ull) & ~63ull;
        factors += 2ull * b;
    }
    cp.ofibs_bytes = per_thread * (uint64_t)in.threads;
    cp.factor_bytes = factors;
    const uint64_t avail = in.host_avail_bytes ? in.host_avail_bytes : host_available_bytes();
    cp.budget_bytes = std::min<uint64_t>(avail / 4, 8ull << 30);

    const bool forced_jacobi = in.layout == DGPU_LAYOUT_MORTON;
    auto pick_auto = [&]() -> int {
        if (forced_jacobi) { copy_str(cp.kernel_reason, sizeof(cp.kernel_reason), "forced-jacobi-by-layout"); return DGPU_CP_JACOBI; }
        if (in.nnz < 1000000ull) { copy_str(cp.kernel_reason, sizeof(cp.kernel_reason), "nnz<1M (linalg-dominated)"); return DGPU_CP_GAUSS_SEIDEL; }
        if ((N == 3 && Rp >= 64) || Rp >= 128) { copy_str(cp.kernel_reason, sizeof(cp.kernel_reason), "all-modes-fallback-shape"); return DGPU_CP_GAUSS_SEIDEL; }
        if (cp.ofibs_bytes >= cp.budget_bytes) { copy_str(cp.kernel_reason, sizeof(cp.kernel_reason), "ofibs>budget"); return DGPU_CP_GAUSS_SEIDEL; }
        copy_str(cp.kernel_reason, sizeof(cp.kernel_reason), "all-modes fits");
        return DGPU_CP_JACOBI;
    };

    std::string k = lower(kernel_cli);
    const char* env = std::getenv("DYN_CP_KERNEL");
    const char* src = "auto";
    if (env && env[0]) { k = lower(env); src = "env-kernel"; }
    else if (!k.empty() && k != "auto") src = "cli-kernel";
    if (is_jacobi_word(k)) {
        cp.kernel = DGPU_CP_JACOBI;
        copy_str(cp.kernel_reason, sizeof(cp.kernel_reason), "user-forced-jacobi");
    } else if (is_gs_word(k)) {
        cp.kernel = DGPU_CP_GAUSS_SEIDEL;
        copy_str(cp.kernel_reason, sizeof(cp.kernel_reason), "user-forced-gs");
        if (forced_jacobi) {
            cp.kernel = DGPU_CP_JACOBI;
            copy_str(cp.kernel_reason, sizeof(cp.kernel_reason),
                     "user-wanted-gs-but-layout-forces-jacobi");
        }
    } else {
        if (!k.empty() && k != "auto")
            std::fprintf(stderr, "warning: dgpu compute plan: unknown kernel '%s'; "
                                 "falling back to auto.\n", k.c_str());
        cp.kernel = pick_auto();
    }
    copy_str(cp.kernel_source, sizeof(cp.kernel_source), src);

    for (int n = 0; n < N; ++n) {
        int impl = DGPU_IMPL_ELEMENT;
        if (in.layout == DGPU_LAYOUT_NCOPY && in.fiber && in.kernel_class[n] == 2)
            impl = DGPU_IMPL_FIBERCSR;
        else if (in.kernel_class[n] == 2 || in.avg_fiber_len[n] >= 32.0)
            impl = DGPU_IMPL_FIBER;
        cp.per_mode[n] = impl;
    }
    return DGPU_OK;
}

}  // namespace dgpu

using namespace dgpu;

extern "C" {

int dgpu_compute_plan_decide(const dgpu_compute_plan_input* in, const char* kernel_cli,
                             dgpu_compute_plan* out) {
    if (!in || !out) { set_error("dgpu_compute_plan_decide: null argument"); return DGPU_ERR_ARG; }
    return compute_plan_decide(*in, kernel_cli, *out);
}

int dgpu_build_compute_plan(const dgpu_plan* plan, const char* kernel_cli,
                            dgpu_compute_plan* out) {
    const Plan* p = reinterpret_cast<const Plan*>(plan);
    if (!p || !out) { set_error("dgpu_build_compute_plan: null argument"); return DGPU_ERR_ARG; }
    dgpu_compute_plan_input in{};
    in.num_modes = p->N;
    in.nnz = p->nnz;
    in.rank_padded = p->Rp;
    in.threads = p->T;
    in.layout = p->layout;
    in.fiber = p->fiber;
    for (int n = 0; n < p->N; ++n) {
        in.mode_size[n] = p->dims[n];
        in.kernel_class[n] = p->kclass[n];
        in.avg_fiber_len[n] = p->afl[n];
    }
    DGPU_TRY(compute_plan_decide(in, kernel_cli, *out));
    out->precision = p->precision;
    out->device_bytes = p->device_bytes;
    for (int n = 0; n < p->N; ++n) {
        if (p->layout == DGPU_LAYOUT_MORTON) {
            out->accum[n] = 0;          // all-modes pass only
            out->rank_tile[n] = p->Rp;
            continue;
        }
        out->accum[n] = mttkrp_scheme(*p, n);
        const bool fixed = p->rank_tile > 0 && p->rank_tile <= p->Rp && p->Rp % p->rank_tile == 0 &&
                           p->rank_tile % 16 == 0;
        out->rank_tile[n] = fixed ? p->rank_tile
                                  : (p->tile_for[n] ? p->tile_for[n] : (p->Rp <= 64 ? p->Rp : 0));
    }
    return DGPU_OK;
}

int dgpu_format_compute_plan(const dgpu_compute_plan* cp, const char* prefix, char* buf,
                             size_t cap) {
    if (!cp || !buf || cap == 0) { set_error("dgpu_format_compute_plan: null argument"); return DGPU_ERR_ARG; }
    if (!prefix) prefix = "[plan]";
    const int N = std::max(0, std::min(cp->num_modes, kMaxModes));
    std::string per_mode = "[", accum = "[", tiles = "[";
    for (int n = 0; n < N; ++n) {
        const char* sep = n ? "," : "";
        per_mode += sep;
        per_mode += cp->per_mode[n] == DGPU_IMPL_FIBERCSR ? "FiberCSR"
                    : cp->per_mode[n] == DGPU_IMPL_FIBER  ? "Fiber" : "Element";
        accum += sep;
        accum += cp->accum[n] == DGPU_ACCUM_PRIVATE ? "private"
                 : cp->accum[n] == DGPU_ACCUM_ROWRUN ? "rowrun" : "all-modes";
        tiles += sep;
        tiles += cp->rank_tile[n] ? std::to_string(cp->rank_tile[n]) : std::string("tuned");
    }
    per_mode += "]";
    accum += "]";
    tiles += "]";
    const char* lay = cp->layout == DGPU_LAYOUT_NCOPY    ? "NCopy"
                      : cp->layout == DGPU_LAYOUT_MORTON ? "Morton" : "PingPong";
    auto mib = [](uint64_t b) { return (double)b / (1024.0 * 1024.0); };
    const int len = std::snprintf(
        buf, cap,
        "%s layout : %s  (device)\n"
        "%s kernel : %s  (reason=%s; src=%s)\n"
        "%s per-mode : %s  (only used under GS)\n"
        "%s device : accum=%s  rank_tile=%s  gathers=%s\n"
        "%s tuning : Rp=%d  threads=%d\n"
        "%s budgets : ofibs=%.2f MiB  factors=%.2f MiB  device=%.2f MiB\n",
        prefix, lay,
        prefix, cp->kernel == DGPU_CP_JACOBI ? "Jacobi" : "GaussSeidel", cp->kernel_reason,
        cp->kernel_source,
        prefix, per_mode.c_str(),
        prefix, accum.c_str(), tiles.c_str(), cp->precision == DGPU_PREC_BF16 ? "bf16" : "fp32",
        prefix, cp->rank_padded, cp->threads,
        prefix, mib(cp->ofibs_bytes), mib(cp->factor_bytes), mib(cp->device_bytes));
    if (len < 0 || (size_t)len >= cap) {
        set_error("dgpu_format_compute_plan: buffer of %zu bytes too small (%d needed)", cap,
                  len + 1);
        return DGPU_ERR_ARG;
    }
    return DGPU_OK;
}

}  // extern "C"
