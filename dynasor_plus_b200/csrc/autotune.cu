// ============================================================================
//  autotune.cu -- dgpu_plan_autotune: picks a plan's partition chunk sizes,
//  LSD digit widths and MTTKRP grid target by timing whole sweeps.
//
//  The reference fixes its chunking when it is compiled (the rows per shard
//  come from pick_mn, src/dynasor_preprocess.cpp:87-99; the thread count
//  does the rest).  On the device the costs move with the tensor: a
//  64.7M-nonzero Zipf tensor wants few, large partition chunks and 8-bit
//  digits, a tensor of a few hundred thousand nonzeros wants its MTTKRP
//  tiles split over more CTAs.  The knobs, none of which changes a
//  permutation (the remap and fiber sort are stable counting sorts whatever
//  their chunks and digits) or a result beyond FP32 summation order:
//    * fiber_digit_bits    bits per LSD pass of the per-shard fiber sort
//    * sort_digit_bits     bits per LSD pass of the remap
//    * chunks_per_sm       chunks per SM of the remap's partition
//    * seg_chunk_tiles     4096-nonzero tiles per chunk of the fiber sort
//    * mttkrp_ctas_per_sm  CTAs per SM the MTTKRP's tiles are split to
//    * mttkrp_kernel       factor rows by per-lane loads or by the TMA
//                          engine (tile::gather4), where the shape has both
//  Coordinate descent: each knob in turn, the others held, one warm-up
//  sweep and `sweeps` timed sweeps (CUDA events on the plan stream) per
//  candidate, the fastest kept.  The rank tile of wide factors is tuned by
//  the first sweep of each mode as before (mttkrp.cu).
// ============================================================================
#include "dgpu_internal.h"

#include <algorithm>
#include <vector>

namespace dgpu {

int mode_pingpong(Plan& p, int n);
int mode_ncopy(Plan& p, int n);

namespace {

int sweep_once(Plan& p) {
    for (int n = 0; n < p.N; ++n)
        DGPU_TRY(p.layout == DGPU_LAYOUT_NCOPY ? mode_ncopy(p, n) : mode_pingpong(p, n));
    return pingpong_drain(p);
}

// Average ms of `reps` sweeps after one warm-up sweep.
int time_sweeps(Plan& p, int reps, double* ms) {
    DGPU_TRY(sweep_once(p));
    cudaEvent_t a = nullptr, b = nullptr;
    DGPU_CUDA(cudaEventCreate(&a));
    DGPU_CUDA(cudaEventCreate(&b));
    struct E { cudaEvent_t a, b; ~E() { cudaEventDestroy(a); cudaEventDestroy(b); } } eg{a, b};
    DGPU_CUDA(cudaEventRecord(a, p.stream));
    for (int r = 0; r < reps; ++r) DGPU_TRY(sweep_once(p));
    DGPU_CUDA(cudaEventRecord(b, p.stream));
    DGPU_TRY(sync_checked(p));
    float t = 0.f;
    DGPU_CUDA(cudaEventElapsedTime(&t, a, b));
    *ms = (double)t / reps;
    return DGPU_OK;
}

struct Knob {
    int* field;
    std::vector<int> cands;
    bool rebuild;                 // partition lists depend on it
};

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" int dgpu_plan_autotune(dgpu_plan* plan, int sweeps, dgpu_tune_result* out) {
    Plan* pp = reinterpret_cast<Plan*>(plan);
    if (!pp || !out) { set_error("dgpu_plan_autotune: null argument"); return DGPU_ERR_ARG; }
    Plan& p = *pp;
    DGPU_CUDA(cudaSetDevice(p.device));
    if (p.layout == DGPU_LAYOUT_MORTON) {
        set_error("dgpu_plan_autotune: a Morton plan runs the all-modes pass only (nothing to tune)");
        return DGPU_ERR_ARG;
    }
    if (p.layout == DGPU_LAYOUT_PINGPONG && p.next_mode != 0) {
        set_error("dgpu_plan_autotune: the slab is ordered for mode %d; tune between sweeps",
                  p.next_mode);
        return DGPU_ERR_ORDER;
    }
    const int reps = std::max(1, std::min(sweeps, 50));
    bool any_fiber = false;
    for (int n = 0; n < p.N; ++n) any_fiber = any_fiber || (p.fiber && p.kclass[n] == 2);
    const bool pingpong = p.layout == DGPU_LAYOUT_PINGPONG;

    std::vector<Knob> knobs;
    if (pingpong && any_fiber) knobs.push_back({&p.fiber_digit_bits, {5, 6, 7, 8}, false});
    if (pingpong) knobs.push_back({&p.sort_digit_bits, {6, 7, 8}, false});
    if (pingpong) knobs.push_back({&p.chunks_per_sm, {2, 4, 8}, true});
    if (pingpong && any_fiber) knobs.push_back({&p.seg_chunk_tiles, {4, 8, 16}, true});
    knobs.push_back({&p.mttkrp_ctas_per_sm, {2, 4, 8}, false});
    if (gather_supported(p, p.Rp)) knobs.push_back({&p.mttkrp_kernel, {0, 1}, false});

    dgpu_tune_result r{};
    double best = 0.0;
    DGPU_TRY(time_sweeps(p, reps, &best));
    r.default_ms = best;
    r.candidates = 1;
    for (Knob& k : knobs) {
        const int keep = *k.field;
        int chosen = keep;
        for (int c : k.cands) {
            if (c == keep) continue;
            *k.field = c;
            if (k.rebuild) DGPU_TRY(plan_rebuild_partlists(p));
            double ms = 0.0;
            DGPU_TRY(time_sweeps(p, reps, &ms));
            ++r.candidates;
            if (ms < best) { best = ms; chosen = c; }
        }
        *k.field = chosen;
        if (k.rebuild) DGPU_TRY(plan_rebuild_partlists(p));
    }
    // the digit and grid knobs are baked into captured graphs too
    ++p.tables_gen;
    r.tuned_ms = best;
    r.fiber_digit_bits = p.fiber_digit_bits;
    r.sort_digit_bits = p.sort_digit_bits;
    r.chunks_per_sm = p.chunks_per_sm;
    r.seg_chunk_tiles = p.seg_chunk_tiles;
    r.mttkrp_ctas_per_sm = p.mttkrp_ctas_per_sm;
    r.mttkrp_gather = p.mttkrp_kernel;
    *out = r;
    return DGPU_OK;
}
