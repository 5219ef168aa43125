// ============================================================================
//  mttkrp_tma.cu -- mode-n MTTKRP with the factor-row gathers issued to the
//  tensor memory accelerator (sm_100a tile::gather4), row runs as in
//  mttkrp.cu's ROWRUN kernel.
//
//  The row-run kernel gathers every factor row with per-lane loads: a lane
//  group keeps one nonzero's N-1 rows in flight and waits, so the kernel is
//  bound by the latency of those loads (long-scoreboard stalls, DRAM at
//  32-45% of peak, L1 and L2 pipes at 20-30%).  Here lane 0 of every warp
//  asks the TMA engine for the rows ahead of the warp's lanes: one
//  cp.async.bulk.tensor ... tile::gather4 copies four factor rows (the rows
//  of the warp's four lane groups, or two groups' rows of two steps) into a
//  per-warp shared-memory ring of D stages, each stage completing on its own
//  mbarrier.  The lanes read the rows of the stage they work on from shared
//  memory and accumulate row runs in registers exactly as ROWRUN does; lane
//  0 refills the stage they left.  The rows in flight are bounded by the
//  ring (8 KB per warp), not by registers.
//
//  Per CTA: a sub-tile of <= 2048 consecutive slab positions, its
//  nonzeros' values and indices staged in shared memory (columns), 8 warps,
//  warp w the w-th contiguous slice, lane group g the g-th sub-slice of it.
//  Arithmetic per nonzero is the reference's (src/dynasor_kernel.cpp:158-202
//  order: val * Y[w0], middle factors, last factor fused into the FMA).
//  Waits are bounded; a wait that gives up raises the plan's fault flag and
//  the CTA drains the copies it issued before it exits.
// ============================================================================
#include "dgpu_internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <mutex>

namespace dgpu {

namespace {

constexpr int kGatThreads = 256;
constexpr int kGatWarps = kGatThreads / 32;
constexpr uint32_t kGatSub = 2048;             // nonzeros per CTA
constexpr int kGatRingWarpBytes = 8192;        // ring bytes per warp
constexpr int kErrGatherWait = 0x400;          // a gather did not complete in time
constexpr int kErrGatherShape = 0x800;         // sub-tile too long or ring misaligned (nothing done)

struct GatherMaps {
    CUtensorMap m[kMaxModes];
};

template <int N, int G, bool BF>
struct GatShape {
    static constexpr int NG = 32 / G;                      // lane groups per warp
    static constexpr int S = NG >= 4 ? 1 : 4 / NG;         // steps per stage
    static constexpr int RPS = NG * S;                     // rows per stage per gathered mode
    static constexpr int NQ = RPS / 4;                     // gather4 per gathered mode per stage
    static constexpr int ELEM = BF ? 2 : 4;
    static constexpr int RowBytes = 4 * G * ELEM;          // Rp = 4G columns
    static constexpr int StageBytes = (N - 1) * RPS * RowBytes;
    static constexpr int D0 = kGatRingWarpBytes / StageBytes;
    static constexpr int D = D0 < 2 ? 2 : (D0 > 16 ? 16 : D0);   // stages per warp
    static constexpr int SW = 1 + N;                       // staged columns
    static constexpr size_t smem() {
        return (size_t)kGatWarps * D * StageBytes + (size_t)SW * kGatSub * 4 +
               (size_t)kGatWarps * D * 8;
    }
    static_assert(RPS % 4 == 0, "a stage is whole gather4 copies");
    static_assert((4 * RowBytes) % 128 == 0 && StageBytes % 128 == 0, "128-byte aligned copies");
};

__device__ __forceinline__ uint32_t saddr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void g_mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(saddr(bar)));
}
__device__ __forceinline__ void g_mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool g_mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(saddr(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait: false after ~2^22 polls.
__device__ __forceinline__ bool g_mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < (1u << 22); ++i)
        if (g_mbar_try_wait(bar, parity)) return true;
    return false;
}
// Four rows (r0..r3) of a 2-D tensor map whose box is one row high and the
// row's columns wide, to consecutive rows at dst; completes on bar.
__device__ __forceinline__ void gather4(void* dst, const CUtensorMap* map, uint32_t r0,
                                        uint32_t r1, uint32_t r2, uint32_t r3, uint64_t* bar) {
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4"
                 ".mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
                 :: "r"(saddr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(0),
                    "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(saddr(bar))
                 : "memory");
}

template <bool BF>
__device__ __forceinline__ float4 row4(const unsigned char* p) {
    if constexpr (BF) {
        const uint2 raw = *reinterpret_cast<const uint2*>(p);
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.y));
        return make_float4(a.x, a.y, b.x, b.y);
    } else {
        return *reinterpret_cast<const float4*>(p);
    }
}

template <int N, int G, bool BF, int TN>
__global__ void __launch_bounds__(kGatThreads, 2)
k_mttkrp_gather(const __grid_constant__ SlabPtrs in, const Tile* __restrict__ tiles,
                const __grid_constant__ GatherMaps maps, float* __restrict__ Yhat, int n_rt,
                int wl_rt, int ld, int rows_contiguous, int* __restrict__ err)
{
    using Sh = GatShape<N, G, BF>;
    constexpr int NG = Sh::NG, S = Sh::S, RPS = Sh::RPS, D = Sh::D;
    constexpr int RB = Sh::RowBytes, SB = Sh::StageBytes;
    const int n = TN >= 0 ? TN : n_rt;
    const int wl = TN >= 0 ? (N == 2 ? -1 : (TN == N - 1 ? N - 2 : N - 1)) : wl_rt;
    extern __shared__ __align__(1024) unsigned char gsm[];
    unsigned char* ring = gsm;
    uint32_t* meta = reinterpret_cast<uint32_t*>(gsm + (size_t)kGatWarps * D * SB);
    uint64_t* bars = reinterpret_cast<uint64_t*>(meta + (size_t)Sh::SW * kGatSub);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;

    Tile tl = tiles[blockIdx.x];
    {
        const uint32_t a = (uint32_t)(((uint64_t)tl.count * blockIdx.y) / gridDim.y);
        const uint32_t b = (uint32_t)(((uint64_t)tl.count * (blockIdx.y + 1)) / gridDim.y);
        tl.begin += a;
        tl.count = b - a;
    }
    const uint32_t cnt = tl.count;
    // the launch keeps sub-tiles <= kGatSub; TMA destinations must be aligned
    if (cnt > kGatSub || (saddr(ring) & 127u) != 0u) {
        if (threadIdx.x == 0) atomicOr(err, kErrGatherShape);
        return;
    }
    // the sub-tile's values and indices, one column each (the slab is read
    // once per sweep: streaming loads)
    for (uint32_t i = threadIdx.x; i < cnt; i += kGatThreads) {
        meta[i] = __float_as_uint(__ldcs(in.vals + tl.begin + i));
#pragma unroll
        for (int w = 0; w < N; ++w) meta[(size_t)(1 + w) * kGatSub + i] = __ldcs(in.idx[w] + tl.begin + i);
    }
    uint64_t* wbar = bars + warp * D;
    unsigned char* wring = ring + (size_t)warp * D * SB;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < D; ++k) g_mbar_init(&wbar[k]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();                                // metadata staged, barriers initialised

    const uint32_t per_w = (cnt + kGatWarps - 1) / kGatWarps;
    const uint32_t wb = min(cnt, (uint32_t)warp * per_w);
    const uint32_t we = min(cnt, wb + per_w);
    if (we <= wb) return;                           // no work for this warp
    const uint32_t span = we - wb;
    const uint32_t per_g = (span + NG - 1) / NG;    // steps of every group
    const uint32_t nst = (per_g + S - 1) / S;       // stages of the warp
    const uint32_t* midx = meta + kGatSub;          // idx[w] column at midx + w * kGatSub

    // lane 0: the rows of stage k into ring slot k % D
    auto issue = [&](uint32_t k) {
        const uint32_t slot = k % D;
        uint64_t* b = &wbar[slot];
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        g_mbar_expect_tx(b, (uint32_t)SB);
        unsigned char* dst = wring + (size_t)slot * SB;
        int wi = 0;
#pragma unroll
        for (int w = 0; w < N; ++w) {
            if (w == n) continue;
            const uint32_t* col = midx + (size_t)w * kGatSub;
#pragma unroll
            for (int q = 0; q < Sh::NQ; ++q) {
                uint32_t r[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int j = q * 4 + t;                   // row j of the stage
                    const uint32_t e = k * S + j / NG;          // its step
                    const uint32_t rel = (uint32_t)(j % NG) * per_g + e;
                    // finished groups fetch the warp's first row (in range)
                    r[t] = col[wb + ((e < per_g && rel < span) ? rel : 0u)];
                }
                gather4(dst + (size_t)(wi * RPS + q * 4) * RB, &maps.m[w], r[0], r[1], r[2], r[3], b);
            }
            ++wi;
        }
    };
    if (lane == 0)
        for (uint32_t k = 0; k < nst && k < (uint32_t)D; ++k) issue(k);
    __syncwarp();

    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t cur = 0xffffffffu;
    bool first_run = true;
    bool fail = false;
    uint32_t k = 0;
    for (; k < nst; ++k) {
        const uint32_t slot = k % D;
        const bool ok = g_mbar_wait(&wbar[slot], (k / D) & 1u);
        if (__any_sync(0xffffffffu, !ok)) {
            fail = true;
            if (lane == 0) atomicOr(err, kErrGatherWait);
            break;
        }
        const unsigned char* st = wring + (size_t)slot * SB;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const uint32_t e = k * S + s;
            const uint32_t rel = (uint32_t)grp * per_g + e;
            if (e < per_g && rel < span) {
                const uint32_t i = wb + rel;
                const float val = __uint_as_float(meta[i]);
                const uint32_t row = midx[(size_t)n * kGatSub + i];
                float y[N][4];
                int wi = 0;
#pragma unroll
                for (int w = 0; w < N; ++w) {
                    float4 g4 = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (w != n) {
                        g4 = row4<BF>(st + (size_t)(wi * RPS + s * NG + grp) * RB +
                                      (size_t)gl * 4 * Sh::ELEM);
                        ++wi;
                    }
                    y[w][0] = g4.x; y[w][1] = g4.y; y[w][2] = g4.z; y[w][3] = g4.w;
                }
                if (row != cur) {
                    if (cur != 0xffffffffu) {
                        float4* out = reinterpret_cast<float4*>(Yhat + (size_t)cur * ld);
                        const float4 a4 = make_float4(acc[0], acc[1], acc[2], acc[3]);
                        // a run that neither starts nor ends the group's
                        // slice holds its row's every nonzero when rows are
                        // contiguous (fiber-sorted): store, no atomic
                        if (rows_contiguous && !first_run) out[gl] = a4;
                        else atomicAdd(out + gl, a4);
                        acc[0] = acc[1] = acc[2] = acc[3] = 0.f;
                        first_run = false;
                    }
                    cur = row;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float pr = val, yl = 1.f;
#pragma unroll
                    for (int w = 0; w < N; ++w) {
                        const float yy = y[w][q];
                        pr = (w != n && w != wl) ? pr * yy : pr;
                        yl = (w == wl) ? yy : yl;
                    }
                    acc[q] = (wl >= 0) ? __fmaf_rn(pr, yl, acc[q]) : acc[q] + pr;
                }
            }
        }
        __syncwarp();                               // the stage's rows are read
        if (lane == 0 && k + D < nst) issue(k + D);
    }
    if (!fail && cur != 0xffffffffu)
        atomicAdd(reinterpret_cast<float4*>(Yhat + (size_t)cur * ld) + gl,
                  make_float4(acc[0], acc[1], acc[2], acc[3]));
    if (fail && lane == 0) {
        // leave no copy in flight into this CTA's shared memory
        const uint32_t issued = std::min<uint32_t>(nst, k + D);
        for (uint32_t j = k; j < issued; ++j) g_mbar_wait(&wbar[j % D], (j / D) & 1u);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, []() {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Tensor maps of the gathered factors: rows x Rp elements, row stride Rp,
// box one row high and Rp columns wide (what tile::gather4 takes).
int build_maps(const Plan& p, int n, bool bf, GatherMaps& gm) {
    auto enc = encode_fn();
    if (!enc) {
        set_error("mttkrp: cuTensorMapEncodeTiled is not available from the driver");
        return DGPU_ERR_CUDA;
    }
    std::memset(&gm, 0, sizeof(gm));
    for (int w = 0; w < p.N; ++w) {
        if (w == n) continue;
        void* base = bf ? (void*)p.Yb[w] : (void*)p.Y[w];
        const cuuint64_t dim[2] = {(cuuint64_t)p.Rp, (cuuint64_t)p.dims[w]};
        const cuuint64_t stride[1] = {(cuuint64_t)p.Rp * (bf ? 2 : 4)};
        const cuuint32_t box[2] = {(cuuint32_t)p.Rp, 1u};
        const cuuint32_t es[2] = {1u, 1u};
        const CUresult rc = enc(&gm.m[w], bf ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                2, base, dim, stride, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (rc != CUDA_SUCCESS) {
            set_error("mttkrp: tensor map of factor %d failed (CUresult %d)", w, (int)rc);
            return DGPU_ERR_CUDA;
        }
    }
    return DGPU_OK;
}

template <int N, int G, bool BF, int TN>
int launch_gather_t(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles,
                    int wl, int rows_contiguous) {
    using Sh = GatShape<N, G, BF>;
    GatherMaps gm;
    DGPU_TRY(build_maps(p, n, BF, gm));
    auto k = k_mttkrp_gather<N, G, BF, TN>;
    const size_t smem = Sh::smem();
    DGPU_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // sub-tiles of <= kGatSub nonzeros; more when the tensor has few tiles
    const uint32_t want = (uint32_t)std::max(1, std::min(16, p.mttkrp_ctas_per_sm)) * (uint32_t)p.sms;
    uint32_t split = (kTile + kGatSub - 1) / kGatSub;
    if ((uint64_t)ntiles * split < want)
        split = std::min<uint32_t>(16u, std::max(split, (want + ntiles - 1) / std::max(1u, ntiles)));
    const dim3 grid(ntiles, split);
    k<<<grid, kGatThreads, smem, p.stream>>>(slab_in(in, p.N), tiles, gm, p.Yhat[n], n, wl, p.Rp,
                                             rows_contiguous, p.err_flag);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

template <int N, int G, bool BF>
int launch_gather_n(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles, int wl,
                    int rows_contiguous) {
    switch (n) {
        case 0: return launch_gather_t<N, G, BF, 0>(p, n, in, tiles, ntiles, wl, rows_contiguous);
        case 1: return launch_gather_t<N, G, BF, 1>(p, n, in, tiles, ntiles, wl, rows_contiguous);
        case 2: return launch_gather_t<N, G, BF, 2>(p, n, in, tiles, ntiles, wl, rows_contiguous);
        default:
            if constexpr (N == 4)
                return launch_gather_t<N, G, BF, 3>(p, n, in, tiles, ntiles, wl, rows_contiguous);
            set_error("mttkrp: gather kernel has no mode %d of %d", n, N);
            return DGPU_ERR_ARG;
    }
}

template <bool BF>
int launch_gather_bf(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles, int wl,
                     int rows_contiguous) {
    const int G = p.Rp / 4;
#define DGPU_GAT(NN, GG) \
    if (p.N == NN && G == GG) return launch_gather_n<NN, GG, BF>(p, n, in, tiles, ntiles, wl, rows_contiguous)
    DGPU_GAT(3, 4); DGPU_GAT(3, 8); DGPU_GAT(3, 16);
    DGPU_GAT(4, 4); DGPU_GAT(4, 8); DGPU_GAT(4, 16);
#undef DGPU_GAT
    set_error("mttkrp: gather kernel has no %d-mode rank-%d variant", p.N, p.Rp);
    return DGPU_ERR_ARG;
}

}  // namespace

bool gather_supported(const Plan& p, int cols) {
    return (p.N == 3 || p.N == 4) && cols == p.Rp && (p.Rp == 16 || p.Rp == 32 || p.Rp == 64) &&
           p.err_flag != nullptr;
}

int launch_mttkrp_gather(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles,
                         bool bf, int wl, int rows_contiguous) {
    if (bf) return launch_gather_bf<true>(p, n, in, tiles, ntiles, wl, rows_contiguous);
    return launch_gather_bf<false>(p, n, in, tiles, ntiles, wl, rows_contiguous);
}

}  // namespace dgpu
