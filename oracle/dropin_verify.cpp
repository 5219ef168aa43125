// ============================================================================
//  dropin_verify.cpp -- TEST INFRASTRUCTURE ONLY.
//
//  The reference's MTTKRP benchmark with --verify (src/main.cpp:896-968) and
//  a CP-ALS run, written against the reference's own host API (Tensor,
//  FactorMatrices, load_coo_tensor, spmttkrp_reference,
//  compare_factors_detail, cpals) with the GPU shim
//  (include/dynasor_b200_dropin.hpp) in place of SpmttkrpSweep and cpals:
//  the code a Dynasor+ maintainer would write to switch a driver to the
//  B200 engine.  Built by oracle/Makefile against the reference headers and
//  the compiled reference library (oracle/_ref), linked with
//  libdynasor_b200.so.
//
//    dropin_verify <tensor.tns|.dnb> <rank> <threads> <seed> [cpals_iters]
//
//  1. load the tensor twice (one copy for the reference's CP-ALS);
//  2. U(0,1) inputs from one std::mt19937_64(seed) across the modes in
//     order (src/main.cpp:326-337, 903-907);
//  3. spmttkrp_reference into F_ref; a GpuSweep (process(0..N-1)) into F_gpu;
//  4. compare_factors_detail: PASS within 1e-4, else exit code 3 (the
//     reference's --verify failure code, src/main.cpp:957-965);
//  5. cpals_gpu and the reference's cpals from seed 42 on the same tensor,
//     tol 0: fit histories within 1e-4, else exit code 9.
// ============================================================================
#include "dynasor_b200_dropin.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

using namespace dynasor;

static void uniform_inputs(FactorMatrices& F, const Tensor& T, uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> U(0.0f, 1.0f);
    for (int n = 0; n < T.num_modes; ++n)
        for (idx_t i = 0; i < T.mode_size[n]; ++i) {
            for (int r = 0; r < F.rank; ++r) F.Y[n][(size_t)i * F.rank_padded + r] = U(rng);
            for (int r = F.rank; r < F.rank_padded; ++r) F.Y[n][(size_t)i * F.rank_padded + r] = 0.f;
        }
}

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <tensor.tns|.dnb> <rank> <threads> <seed> [cpals_iters]\n",
                     argv[0]);
        return 2;
    }
    const std::string path = argv[1];
    const int rank = std::atoi(argv[2]);
    const int threads = std::atoi(argv[3]);
    const uint64_t seed = std::strtoull(argv[4], nullptr, 10);
    const int iters = argc > 5 ? std::atoi(argv[5]) : 5;

    Tensor T;
    if (!load_coo_tensor(path, T, false)) {
        std::fprintf(stderr, "[dropin] cannot load %s\n", path.c_str());
        return 2;
    }
    FactorMatrices F_gpu, F_ref;
    F_gpu.allocate(T.num_modes, T.mode_size, rank);
    F_ref.allocate(T.num_modes, T.mode_size, rank);
    uniform_inputs(F_gpu, T, seed);
    for (int n = 0; n < T.num_modes; ++n)
        std::memcpy(F_ref.Y[n], F_gpu.Y[n],
                    (size_t)T.mode_size[n] * F_gpu.rank_padded * sizeof(value_t));

    spmttkrp_reference(T, F_ref);
    double secs = 0.0;
    try {
        dgpu_dropin::GpuSweep sweep(T, F_gpu, threads, true);
        for (int n = 0; n < T.num_modes; ++n) sweep.process(n);
        secs = sweep.elapsed_s();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[dropin] GPU sweep failed: %s\n", e.what());
        return 2;
    }
    int rc = 0;
    const double err = compare_factors_detail(F_gpu, F_ref, T.mode_size);
    if (err > 1e-4) {
        std::printf("FAIL: Frobenius relative error %.3e exceeds %.1e\n", err, 1e-4);
        rc = 3;
    } else {
        std::printf("PASS: Frobenius relative error %.3e within %.1e\n", err, 1e-4);
    }
    std::printf("[summary] gpu sweep = %.6f s (%.3f Mnnz/s, host copies included)\n", secs,
                (double)T.nnz / 1e6 / std::max(secs, 1e-12));

    // CP-ALS through the shim against the reference's cpals
    CpOptions opt;
    opt.max_iters = iters;
    opt.tol = 0.0;
    opt.seed = 42;
    opt.num_threads = threads;
    opt.verbose = false;
    FactorMatrices G_gpu;
    G_gpu.allocate(T.num_modes, T.mode_size, rank);
    CpResult rg;
    try {
        rg = dgpu_dropin::cpals_gpu(T, G_gpu, opt);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[dropin] cpals_gpu failed: %s\n", e.what());
        return 2;
    }
    Tensor T2;
    if (!load_coo_tensor(path, T2, false)) return 2;
    build_flycoo(T2, threads, nullptr, 16);
    FactorMatrices G_ref;
    G_ref.allocate(T2.num_modes, T2.mode_size, rank);
    const CpResult rr = cpals(T2, G_ref, opt);
    double dmax = 0.0;
    const size_t k = std::min(rg.fit_history.size(), rr.fit_history.size());
    for (size_t i = 0; i < k; ++i)
        dmax = std::max(dmax, std::fabs(rg.fit_history[i] - rr.fit_history[i]));
    const bool fit_ok = rg.iters_done == rr.iters_done && dmax < 1e-4;
    std::printf("%s: cpals_gpu %d iterations, final fit %.8f; reference %d, %.8f; "
                "max |fit difference| %.3e\n",
                fit_ok ? "PASS" : "FAIL", rg.iters_done, rg.final_fit, rr.iters_done,
                rr.final_fit, dmax);
    if (!fit_ok && rc == 0) rc = 9;

    F_gpu.free_all();
    F_ref.free_all();
    G_gpu.free_all();
    G_ref.free_all();
    return rc;
}
