// ============================================================================
//  dynasor_b200_dropin.hpp -- header-only C++ shim that maps the B200
//  engine's C ABI (dynasor_b200.h) onto the reference's host API, so a
//  Dynasor+ driver (main.cpp's MTTKRP benchmark with --verify, or a CP-ALS
//  caller) switches to the GPU by changing the names it calls:
//
//    dynasor::SpmttkrpSweep  (include/dynasor_common.h:760-786)
//        -> dgpu_dropin::GpuSweep      same constructor and process(n)
//    dynasor::spmttkrp_dynasor (include/dynasor_common.h:699)
//        -> dgpu_dropin::spmttkrp_gpu  same arguments, same return value
//    dynasor::cpals          (include/dynasor_cpals.h:121)
//        -> dgpu_dropin::cpals_gpu     same arguments, same CpResult
//
//  Include it after the reference's headers are on the include path; link
//  libdynasor_b200.so.  The reference's types are used as they are: a
//  Tensor (loaded, before or after build_flycoo) and an allocated
//  FactorMatrices.
//
//  Semantics kept from the reference:
//    * process(n) reads the host factors F.Y[w] (w != n) as they are at the
//      call, so host-side factor updates between modes are seen, and writes
//      F.Yhat[n]; modes must be called in order 0, 1, ..., N-1, 0, ...;
//    * the FLYCOO plan depends on num_threads as the reference's does: built
//      from a freshly loaded tensor, the device slab after process(n) is the
//      reference's slab after SpmttkrpSweep::process(n) with the same
//      thread count.  (Given a tensor that build_flycoo has already ordered,
//      the device builds its plan over that order instead; Yhat is the same
//      up to FP32 summation order.)  The host tensor is not modified;
//    * cpals_gpu starts from the reference's seeded N(0,1) factors, applies
//      the same stop rule and returns the same CpResult fields.
//  Differences: errors throw std::runtime_error carrying dgpu_last_error()
//  (the reference's kernels return void and its drivers exit()); the
//  Cholesky solve is FP64; <T, M> in the fit stays FP64.
// ============================================================================
#ifndef DYNASOR_B200_DROPIN_HPP
#define DYNASOR_B200_DROPIN_HPP

#include "dynasor_common.h"
#include "dynasor_cpals.h"
#include "dynasor_b200.h"

#include <chrono>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace dgpu_dropin {

inline void check(int rc, const char* what) {
    if (rc != DGPU_OK) {
        const char* msg = dgpu_last_error();
        throw std::runtime_error(std::string(what) + ": " + (msg ? msg : "") + " (status " +
                                 std::to_string(rc) + ")");
    }
}

// Device plan of a reference Tensor's nonzeros (the work build_flycoo does).
inline dgpu_plan* make_plan(const dynasor::Tensor& T, int rank, int num_threads, int device = 0) {
    dgpu_tensor_desc d{};
    d.num_modes = T.num_modes;
    d.nnz = T.nnz;
    d.mode_size = T.mode_size;
    d.vals = T.vals;
    d.idx = T.idx_buf;                  // idx_t is uint32_t
    dgpu_plan_opts o;
    dgpu_plan_opts_default(&o);
    o.threads = num_threads > 0 ? num_threads : 1;
    o.rank = rank;
    o.layout = DGPU_LAYOUT_PINGPONG;
    o.device = device;
    dgpu_plan* p = nullptr;
    check(dgpu_plan_create(&d, &o, &p), "dgpu_plan_create");
    return p;
}

// SpmttkrpSweep on the GPU.
class GpuSweep {
public:
    GpuSweep(dynasor::Tensor& T, dynasor::FactorMatrices& F, int num_threads,
             bool print_banner = false, int device = 0)
        : T_(T), F_(F), threads_(num_threads) {
        if (F.num_modes != T.num_modes)
            throw std::runtime_error("GpuSweep: factor and tensor mode counts differ");
        plan_ = make_plan(T, F.rank, num_threads, device);
        dgpu_plan_info info;
        check(dgpu_plan_get_info(plan_, &info), "dgpu_plan_get_info");
        if (info.rank_padded != F.rank_padded) {
            dgpu_plan_destroy(plan_);
            throw std::runtime_error("GpuSweep: factor rank_padded differs from the plan's");
        }
        if (print_banner)
            std::printf("[gpu-sweep] %d modes, %llu nnz, rank %d (Rp %d), plan threads %d, "
                        "%.2f GiB on device %d\n",
                        T.num_modes, (unsigned long long)T.nnz, F.rank, F.rank_padded,
                        num_threads, (double)info.device_bytes / (1u << 30), device);
    }
    GpuSweep(const GpuSweep&) = delete;
    GpuSweep& operator=(const GpuSweep&) = delete;
    ~GpuSweep() { if (plan_) dgpu_plan_destroy(plan_); }

    // Mode n: upload the other modes' host factors, run the MTTKRP (and the
    // device remap for mode (n+1) % N), copy Yhat[n] back to F.Yhat[n].
    void process(int n) {
        const auto t0 = std::chrono::steady_clock::now();
        for (int w = 0; w < T_.num_modes; ++w)
            if (w != n) check(dgpu_upload_factor(plan_, w, F_.Y[w]), "dgpu_upload_factor");
        check(dgpu_mttkrp_mode(plan_, n), "dgpu_mttkrp_mode");
        check(dgpu_download_yhat(plan_, n, F_.Yhat[n]), "dgpu_download_yhat");
        elapsed_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    double elapsed_s() const { return elapsed_; }
    int num_threads() const { return threads_; }
    dynasor::Tensor& tensor() { return T_; }
    dynasor::FactorMatrices& factors() { return F_; }
    dgpu_plan* plan() { return plan_; }

private:
    dynasor::Tensor& T_;
    dynasor::FactorMatrices& F_;
    int threads_;
    dgpu_plan* plan_ = nullptr;
    double elapsed_ = 0.0;
};

// spmttkrp_dynasor on the GPU: one sweep over all modes, Yhat[n] for every
// n in F; returns the sweep's seconds.
inline double spmttkrp_gpu(dynasor::Tensor& T, dynasor::FactorMatrices& F, int num_threads) {
    GpuSweep s(T, F, num_threads);
    for (int n = 0; n < T.num_modes; ++n) s.process(n);
    return s.elapsed_s();
}

// cpals on the GPU (Gauss-Seidel or Jacobi per opt.kernel).  F must be
// allocated with the wanted rank; on return F.Y holds the normalised
// factors and the result carries lambda and the fit history.
inline dynasor::CpResult cpals_gpu(dynasor::Tensor& T, dynasor::FactorMatrices& F,
                                   const dynasor::CpOptions& opt, int device = 0) {
    const int threads = opt.num_threads > 0 ? opt.num_threads : 1;
    dgpu_plan* p = make_plan(T, F.rank, threads, device);
    dgpu_cp_options o;
    dgpu_cp_options_default(&o);
    o.max_iters = opt.max_iters;
    o.tol = opt.tol;
    o.seed = opt.seed;
    o.ridge = opt.ridge;
    o.kernel = opt.kernel == dynasor::CpKernel::Jacobi ? DGPU_CP_JACOBI : DGPU_CP_GAUSS_SEIDEL;
    o.verbose = opt.verbose ? 1 : 0;
    dgpu_cp_result r{};
    std::vector<double> hist((size_t)(opt.max_iters > 0 ? opt.max_iters : 1));
    const int rc = dgpu_cpals(p, &o, &r, hist.data());
    dynasor::CpResult out;
    if (rc == DGPU_OK) {
        out.iters_done = r.iters_done;
        out.final_fit = r.final_fit;
        out.final_residual = r.final_residual;
        out.tensor_norm = r.tensor_norm;
        out.total_time_s = r.total_time_s;
        out.mttkrp_time_s = r.mttkrp_time_s;
        out.linalg_time_s = r.linalg_time_s;
        out.fit_history.assign(hist.begin(), hist.begin() + r.iters_done);
        std::vector<float> lam((size_t)F.rank_padded);
        int rc2 = dgpu_download_lambda(p, lam.data());
        for (int n = 0; rc2 == DGPU_OK && n < T.num_modes; ++n)
            rc2 = dgpu_download_factor(p, n, F.Y[n]);
        if (rc2 != DGPU_OK) {
            dgpu_plan_destroy(p);
            check(rc2, "cpals_gpu: download");
        }
        out.lambda.assign(lam.begin(), lam.begin() + F.rank);
    }
    dgpu_plan_destroy(p);
    check(rc, "dgpu_cpals");
    return out;
}

}  // namespace dgpu_dropin

#endif  // DYNASOR_B200_DROPIN_HPP
