// ============================================================================
//  mttkrp.cu -- mode-n sparse MTTKRP over a FLYCOO slab (sm_100a).
//
//  Replaces the reference's per-nnz kernels (src/dynasor_kernel.cpp:91-229,
//  fiber variant :365-489).  Arithmetic per nonzero is the reference's:
//      prod = val * Y[w0][i_w0, :]            (w0 = n==0 ? 1 : 0)
//      prod *= Y[w][i_w, :]                   (every other w except w_last)
//      Yhat[n][i_n, :] += prod * Y[w_last][i_wl, :]
//  (for N == 2 the last factor is absent).  Gathers are FP32 or BF16 widened
//  to FP32; accumulation is FP32.  This is a gather, not a contraction: no
//  tensor cores.
//
//  Two accumulation schemes (dgpu_plan_opts.accum):
//
//  PRIVATE  (k_mttkrp_priv) -- the Yhat block of the current super-shard
//      (m_n rows x Rp) is held in shared memory.  Each nonzero adds its row
//      contribution with shared-memory atomics (lane c owns columns c,
//      c+32, ..., so the 32 lanes of a warp hit 32 distinct banks).  Slab
//      order inside a shard is irrelevant.  A persistent CTA walks a
//      contiguous run of tiles in processing order and flushes the block to
//      global Yhat (vector atomics, touched rows only) when the shard
//      changes and at the end, so global atomics scale with rows, not with
//      nonzeros.
//
//  ROWRUN   (k_mttkrp_rowrun) -- a lane group (G lanes, float4 columns)
//      walks a contiguous run of a tile and keeps the current row's partial
//      sum in registers, flushing with one vector atomic per row segment.
//      Ideal on fiber-sorted slabs (rows contiguous); any order is correct.
//
//  Both read the slab exactly once.  Metadata of 32 consecutive nonzeros
//  is fetched by the 32 lanes of a warp with coalesced loads; factor rows
//  are gathered with one warp-coalesced load per row.
// ============================================================================
#include "dgpu_internal.h"

#include <algorithm>

namespace dgpu {

namespace {

struct FacPtrs {
    const float*         Y[kMaxModes];
    const __nv_bfloat16* Yb[kMaxModes];
};

template <bool BF>
__device__ __forceinline__ float4 gather4(const FacPtrs& F, int w, uint32_t row, int Rp, int c4) {
    if constexpr (BF) {
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(F.Yb[w] + (size_t)row * Rp) + c4);
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.y));
        return make_float4(a.x, a.y, b.x, b.y);
    } else {
        return __ldg(reinterpret_cast<const float4*>(F.Y[w] + (size_t)row * Rp) + c4);
    }
}

// Compile-time loop: f(integral_constant<int, 0..K-1>) so register arrays
// indexed by the loop variable stay in registers.
template <int I, int K, typename Fn>
__device__ __forceinline__ void static_for(Fn&& f) {
    if constexpr (I < K) {
        f(std::integral_constant<int, I>{});
        static_for<I + 1, K>(f);
    }
}

template <bool BF>
__device__ __forceinline__ float gather1(const FacPtrs& F, int w, uint32_t row, int RP, int c) {
    if constexpr (BF) return __bfloat162float(F.Yb[w][(size_t)row * RP + c]);
    else return __ldg(F.Y[w] + (size_t)row * RP + c);
}

// Products of the two BF16 values in each half of words a and b, exact in
// FP32 (two 8-bit significands), by sm_100's mixed-precision FMA
// (fma.rn.f32.bf16: BF16 multiplicands, FP32 addend and result) with a zero
// addend: no conversion instructions.  .x = low halves, .y = high halves.
__device__ __forceinline__ float2 bf16x2_products(uint32_t a, uint32_t b) {
    float lo, hi;
    asm("{\n\t.reg .b16 a0, a1, b0, b1;\n\t"
        "mov.b32 {a0, a1}, %2;\n\t"
        "mov.b32 {b0, b1}, %3;\n\t"
        "fma.rn.f32.bf16 %0, a0, b0, 0f00000000;\n\t"
        "fma.rn.f32.bf16 %1, a1, b1, 0f00000000;\n\t}"
        : "=f"(lo), "=f"(hi) : "r"(a), "r"(b));
    return make_float2(lo, hi);
}
// BF16 half h (0 low, 1 high) of word w as FP32 (exact).
__device__ __forceinline__ float bf16_half(uint32_t w, int h) {
    return __uint_as_float(h ? (w & 0xffff0000u) : (w << 16));
}

// ===========================================================================
//  ROWRUN
// ===========================================================================
constexpr int kRunThreads = 256;
constexpr int kRunWarps = kRunThreads / 32;

// Nonzeros whose gathers a lane group keeps in flight together (U) and the
// CTAs per SM the kernel is compiled for.  The kernel is bound by gather
// latency, so occupancy (40-64 registers, 4-6 CTAs of 256 threads) pays more
// than a deeper batch, for BF16 rows as well.
template <int N, int V, bool BF>
struct RunBatch {
    static constexpr int kWork = (N - 1) * V;
    // measured on the 3-mode rank-32 Zipf tensor (MTTKRP ms per sweep):
    //   FP32 4 CTAs/U=2 3.68, 5/1 3.60, 6/1 3.45, 8/1 3.66 (spills), 4/1 4.03;
    //   BF16 4/4 3.65, 6/2 3.70, 6/1 3.08
    // and on the 4-mode rank-64 tensor (NCopy CP-ALS iterations/s):
    //   FP32 4/2 34.3, 3/2 32.8, 3/3 29.8, 5/1 36.0, 6/1 33.2 (spills);
    //   BF16 4/2 31.2, 4/4 22.4, 3/3 28.8, 5/1 35.8, 6/1 36.9
    // and, BF16 rows as raw pairs with mixed-precision products (MTTKRP ms
    // per sweep, 3-mode / 4-mode): 6/1 2.71 / 20.65, 4/2 3.15 / 25.58
    // and, FP32 3-mode with cp.async metadata: 6/1 3.30, 5/2 3.44
    static constexpr bool kQuad = (N == 4 && V == 1);
    static constexpr int U = kWork <= 2 ? 1 : (kQuad ? 1 : (kWork <= 4 ? 2 : 1));
    static constexpr int kMinBlocks = kWork <= 2 ? 6 : (kQuad ? (BF ? 6 : 5) : (N <= 4 ? 4 : 2));
};

// One CTA per tile.  Warp w owns the w-th contiguous slice of the tile and
// lane group g (G lanes) the g-th contiguous sub-slice of that, so a group
// sees every row run of its sub-slice in order.  Per chunk of CH nonzeros
// the group's lanes load the metadata with coalesced loads into a small
// shared slot array (prefetching the next chunk into registers), then walk
// the chunk U nonzeros at a time: U x (N-1) float4 gathers in flight per
// lane, products in registers, one vector atomic per finished row run.
// Rp columns starting at the factor pointers are processed; ld is the row
// stride (a rank tile of a wider factor has Rp < ld).
// TN >= 0 pins the target mode at compile time (the reference's TGT
// specialisation, src/dynasor_kernel.cpp:247-265), so only the N-1 gathered
// rows occupy registers; TN = -1 takes the mode at run time.
template <int N, int G, int V, bool BF, int TN>
__global__ void __launch_bounds__(kRunThreads, (RunBatch<N, V, BF>::kMinBlocks))
k_mttkrp_rowrun(const __grid_constant__ SlabPtrs in, const Tile* __restrict__ tiles,
                const __grid_constant__ FacPtrs F, float* __restrict__ Yhat,
                int n_rt, int w0_rt, int wl_rt, int Rp, int ld, int rows_contiguous)
{
    // the first gathered mode (w0) starts the product by position: only the
    // target and the fused last mode (wl) need names
    const int n = TN >= 0 ? TN : n_rt;
    (void)w0_rt;
    const int wl = TN >= 0 ? (N == 2 ? -1 : (TN == N - 1 ? N - 2 : N - 1)) : wl_rt;
    constexpr int U = RunBatch<N, V, BF>::U;
    // BF16 rows with the target pinned (3 and 4 modes): rows kept as raw
    // BF16 pairs; the first two gathered modes (MA < MB) multiply by the
    // mixed-precision FMA, a third (MC, 4 modes) is widened
    constexpr bool kMix = BF && TN >= 0 && V == 1 && (N == 3 || N == 4);
    constexpr int MA = TN == 0 ? 1 : 0;
    constexpr int MB = (MA + 1 == TN) ? MA + 2 : MA + 1;
    constexpr int MC = N == 4 ? 6 - TN - MA - MB : 0;
    constexpr int NG = 32 / G;                    // groups per warp
    constexpr int CH = G >= 16 ? G : ((1 + N + 3) / 4 * 4 > 8 ? 8 : 16);  // staged per group
    constexpr int LPE = CH / G;                   // nonzeros loaded per lane per chunk
    constexpr int SW = (1 + N + 3) / 4 * 4;       // words per slot (16-byte multiple)
    // Group slot areas are CH*SW + 4 words apart so the NG groups' 16-byte
    // slot reads of one instruction land in distinct banks.
    constexpr int GS = CH * SW + 4;
    // kAsync: the next chunk's metadata streams into a second slot buffer
    // with cp.async instead of through registers, which frees the registers
    // (and the spill) of the 3-mode FP32 kernel: sweep 7.39 -> 7.25 ms on
    // the 64.7M-nonzero tensor.  Measured slower for BF16 rows (2.70 ->
    // 2.78 ms) and 4 modes (27.3 -> 27.7 ms), and at 8 CTAs per SM, where
    // no room is left for the remap beside the MTTKRP.
    constexpr bool kAsync = N == 3 && !BF && 2u * kRunWarps * NG * GS * 4u <= 48u * 1024u;
    __shared__ __align__(16) uint32_t slots[kAsync ? 2 : 1][kRunWarps * NG * GS];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;
    const int C4 = Rp >> 2;

    // a tile may be split over gridDim.y CTAs (small tensors: more CTAs);
    // row runs cut at a split point are flushed with atomics like any other
    Tile tl = tiles[blockIdx.x];
    if (gridDim.y > 1) {
        const uint32_t a = (uint32_t)(((uint64_t)tl.count * blockIdx.y) / gridDim.y);
        const uint32_t b = (uint32_t)(((uint64_t)tl.count * (blockIdx.y + 1)) / gridDim.y);
        tl.begin += a;
        tl.count = b - a;
    }
    const uint32_t per_w = (tl.count + kRunWarps - 1) / kRunWarps;
    const uint32_t wb = min(tl.count, (uint32_t)warp * per_w);
    const uint32_t we = min(tl.count, wb + per_w);
    const uint32_t per_g = (we - wb + NG - 1) / NG;          // warp-uniform
    const uint32_t gb = min(we, wb + grp * per_g);
    const uint32_t ge = min(we, gb + per_g);
    const uint32_t nchunks = (per_g + CH - 1) / CH;          // warp-uniform
    uint32_t* const gs0 = slots[0] + (warp * NG + grp) * GS;
    uint32_t* const gs1 = slots[kAsync ? 1 : 0] + (warp * NG + grp) * GS;

    float acc[V][4];
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[v][q] = 0.f;
    uint32_t cur = 0xffffffffu;
    bool first_run = true;                 // the run at the start of this group's slice

    // the next chunk's metadata: in registers (stored to the slot buffer
    // when its chunk starts), or, kAsync, copied by cp.async into the other
    // slot buffer (no registers held for it)
    uint32_t pf[kAsync ? 1 : LPE][SW];
    auto prefetch = [&](uint32_t ch) {
#pragma unroll
        for (int k = 0; k < LPE; ++k) {
            const uint32_t e = gb + ch * CH + gl + k * G;
            const uint32_t p = tl.begin + (e < ge ? e : gb);
            if constexpr (kAsync) {
                uint32_t* dst = ((ch & 1u) ? gs1 : gs0) + (gl + k * G) * SW;
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;"
                             :: "r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(in.vals + p)
                             : "memory");
#pragma unroll
                for (int w = 0; w < N; ++w)
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;"
                                 :: "r"((uint32_t)__cvta_generic_to_shared(dst + 1 + w)),
                                    "l"(in.idx[w] + p)
                                 : "memory");
            } else {
                // the slab is read once per sweep: streaming loads (evict
                // first) keep L2 for the factor rows the gathers reuse
                // (plain __ldg measured: 3-mode BF16 2.71 -> 2.83 ms per
                // sweep, 4-mode within 0.5%)
                pf[k][0] = __float_as_uint(__ldcs(in.vals + p));
#pragma unroll
                for (int w = 0; w < N; ++w) pf[k][1 + w] = __ldcs(in.idx[w] + p);
#pragma unroll
                for (int f = 1 + N; f < SW; ++f) pf[k][f] = 0u;
            }
        }
        if constexpr (kAsync) asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (nchunks) prefetch(0);

    for (uint32_t ch = 0; ch < nchunks; ++ch) {
        const uint32_t* gs;
        if constexpr (kAsync) {
            if (ch + 1 < nchunks) {
                prefetch(ch + 1);
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            }
            __syncwarp();
            gs = (ch & 1u) ? gs1 : gs0;
        } else {
#pragma unroll
            for (int k = 0; k < LPE; ++k)
#pragma unroll
                for (int f = 0; f < SW; f += 4)
                    *reinterpret_cast<uint4*>(gs0 + (gl + k * G) * SW + f) =
                        make_uint4(pf[k][f], pf[k][f + 1], pf[k][f + 2], pf[k][f + 3]);
            __syncwarp();
            if (ch + 1 < nchunks) prefetch(ch + 1);
            gs = gs0;
        }
        const uint32_t base = gb + ch * CH;
        const int cnt = base < ge ? (int)min((uint32_t)CH, ge - base) : 0;
        for (int e0 = 0; e0 < cnt; e0 += U) {
            float val[U];
            uint32_t row[U];
            float y[U][kMix ? 1 : N][V][4];
            uint32_t yr[U][kMix ? N : 1][2];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = e0 + u;
                uint32_t s[SW];
#pragma unroll
                for (int f = 0; f < SW; f += 4) {
                    const uint4 q = *reinterpret_cast<const uint4*>(gs + (e < cnt ? e : 0) * SW + f);
                    s[f] = q.x; s[f + 1] = q.y; s[f + 2] = q.z; s[f + 3] = q.w;
                }
                val[u] = e < cnt ? __uint_as_float(s[0]) : 0.f;
                row[u] = 0u;
#pragma unroll
                for (int w = 0; w < N; ++w) row[u] = (w == n) ? s[1 + w] : row[u];
                if constexpr (kMix) {
#pragma unroll
                    for (int w = 0; w < N; ++w) {
                        yr[u][w][0] = yr[u][w][1] = 0u;
                        if (w != TN) {
                            const uint2 raw = __ldg(reinterpret_cast<const uint2*>(
                                                        F.Yb[w] + (size_t)s[1 + w] * ld) + gl);
                            yr[u][w][0] = raw.x;
                            yr[u][w][1] = raw.y;
                        }
                    }
                } else {
#pragma unroll
                    for (int w = 0; w < N; ++w) {
                        const uint32_t id = s[1 + w];
#pragma unroll
                        for (int v = 0; v < V; ++v) {
                            const int c4 = gl + v * G;
                            float4 g4 = make_float4(0.f, 0.f, 0.f, 0.f);
                            if (w != n && (V == 1 || c4 < C4)) g4 = gather4<BF>(F, w, id, ld, c4);
                            y[u][w][v][0] = g4.x; y[u][w][v][1] = g4.y;
                            y[u][w][v][2] = g4.z; y[u][w][v][3] = g4.w;
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (e0 + u < cnt) {
                    if (row[u] != cur) {
                        if (cur != 0xffffffffu) {
                            float4* out = reinterpret_cast<float4*>(Yhat + (size_t)cur * ld);
                            // a run that neither starts nor ends this group's
                            // slice holds every nonzero of its row when rows
                            // are contiguous (fiber-sorted): store, no atomic
                            // (plain stores: evict-first ones, __stcs, measured
                            // slower, 3.31 -> 3.34 ms FP32 / 2.70 -> 2.74 ms
                            // BF16 per 3-mode sweep)
                            const bool own = rows_contiguous && !first_run;
#pragma unroll
                            for (int v = 0; v < V; ++v) {
                                const int c4 = gl + v * G;
                                const float4 a4 = make_float4(acc[v][0], acc[v][1], acc[v][2], acc[v][3]);
                                if (V == 1 || c4 < C4) {
                                    if (own) out[c4] = a4;
                                    else atomicAdd(out + c4, a4);
                                }
#pragma unroll
                                for (int q = 0; q < 4; ++q) acc[v][q] = 0.f;
                            }
                            first_run = false;
                        }
                        cur = row[u];
                    }
                    if constexpr (kMix) {
                        // rows MA x MB exact in FP32, times the value, times
                        // row MC (4 modes) in the accumulating FMA
                        const float2 p0 = bf16x2_products(yr[u][MA][0], yr[u][MB][0]);
                        const float2 p1 = bf16x2_products(yr[u][MA][1], yr[u][MB][1]);
                        const float t[4] = {p0.x, p0.y, p1.x, p1.y};
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            if constexpr (N == 3) {
                                acc[0][q] = __fmaf_rn(val[u], t[q], acc[0][q]);
                            } else {
                                const float yc = bf16_half(yr[u][MC][q >> 1], q & 1);
                                acc[0][q] = __fmaf_rn(val[u] * t[q], yc, acc[0][q]);
                            }
                        }
                        continue;
                    }
                    // non-target modes in increasing order: the first starts
                    // the product (w0), the middle ones multiply, the last
                    // (w_last) is fused into the accumulate (reference order)
#pragma unroll
                    for (int v = 0; v < V; ++v)
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            // select instead of index: w0/wl are runtime values
                            float pr = val[u], yl = 1.f;
#pragma unroll
                            for (int w = 0; w < N; ++w) {
                                const float yy = y[u][w][v][q];
                                pr = (w != n && w != wl) ? pr * yy : pr;
                                yl = (w == wl) ? yy : yl;
                            }
                            acc[v][q] = (wl >= 0) ? __fmaf_rn(pr, yl, acc[v][q]) : acc[v][q] + pr;
                        }
                }
            }
        }
        __syncwarp();
    }
    if (cur != 0xffffffffu) {
        float4* out = reinterpret_cast<float4*>(Yhat + (size_t)cur * ld);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int c4 = gl + v * G;
            if (V == 1 || c4 < C4)
                atomicAdd(out + c4, make_float4(acc[v][0], acc[v][1], acc[v][2], acc[v][3]));
        }
    }
}

// ===========================================================================
//  PRIVATE
// ===========================================================================
constexpr int kPrivThreads = 1024;
constexpr int kPrivWarps = kPrivThreads / 32;

template <int N>
struct Slot {
    static constexpr int kWords = (1 + N + 3) / 4 * 4;   // 16-byte multiple
};

template <int N, int C>
struct PrivBatch {
    static constexpr int kWork = (N - 1) * C;
    static constexpr int U = kWork <= 2 ? 8 : (kWork <= 4 ? 4 : (kWork <= 8 ? 2 : 1));
};

__host__ __device__ constexpr uint32_t priv_flag_words(uint32_t m) {
    return ((m + 31) / 32 + 3) / 4 * 4;
}

template <int N, int RP, bool BF>
__global__ void __launch_bounds__(kPrivThreads, 1)
k_mttkrp_priv(const __grid_constant__ SlabPtrs in, const Tile* __restrict__ tiles,
              uint32_t ntiles, uint32_t per_cta, const __grid_constant__ FacPtrs F,
              float* __restrict__ Yhat, int n, int w0, int wl, int shift_n, uint32_t dim_n)
{
    constexpr int G = RP < 32 ? RP : 32;          // lanes per nonzero
    constexpr int E = 32 / G;                     // nonzeros per warp step
    constexpr int C = RP / G;                     // columns per lane (stride G)
    constexpr int SW = Slot<N>::kWords;
    constexpr int U = PrivBatch<N, C>::U;

    extern __shared__ float sm[];
    const uint32_t m = 1u << shift_n;
    float* yb = sm;                                                        // m x RP
    uint32_t* touched = reinterpret_cast<uint32_t*>(yb + (size_t)m * RP);  // bit per row
    uint32_t* slots = touched + priv_flag_words(m);                        // warps x 32 x SW
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* ws = slots + (size_t)warp * 32 * SW;

    for (uint32_t i = threadIdx.x; i < m * RP; i += blockDim.x) yb[i] = 0.f;
    for (uint32_t i = threadIdx.x; i < priv_flag_words(m); i += blockDim.x) touched[i] = 0u;
    __syncthreads();

    const uint32_t t0 = blockIdx.x * per_cta;
    const uint32_t t1 = min(ntiles, t0 + per_cta);
    uint32_t cur_shard = 0xffffffffu;
    const int sub = lane / G;                 // which nonzero of a step this lane serves
    const int gl = lane % G;                  // lane within its group

    for (uint32_t t = t0; t <= t1; ++t) {
        const bool last = (t == t1);
        const uint32_t shard = last ? 0xfffffffeu : tiles[t].shard;
        if (shard != cur_shard && cur_shard != 0xffffffffu) {
            // flush the finished shard block: one warp per touched row
            __syncthreads();
            const uint32_t base = cur_shard << shift_n;
            for (uint32_t r = warp; r < m; r += kPrivWarps) {
                if (!(touched[r >> 5] & (1u << (r & 31)))) continue;
                const uint32_t grow = base + r;
                if (grow < dim_n)
                    for (int c = lane; c < RP; c += 32) {
                        atomicAdd(Yhat + (size_t)grow * RP + c, yb[(size_t)r * RP + c]);
                        yb[(size_t)r * RP + c] = 0.f;
                    }
            }
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < priv_flag_words(m); i += blockDim.x) touched[i] = 0u;
            __syncthreads();
        }
        if (last) break;
        cur_shard = shard;
        const Tile tl = tiles[t];
        const uint32_t rbase = tl.shard << shift_n;
        const uint32_t nbat = (tl.count + 31) / 32;
        for (uint32_t b = warp; b < nbat; b += kPrivWarps) {
            const uint32_t j = b * 32 + lane;
            if (j < tl.count) {
                const uint32_t pidx = tl.begin + j;
                ws[lane * SW] = __float_as_uint(__ldg(in.vals + pidx));
#pragma unroll
                for (int w = 0; w < N; ++w) ws[lane * SW + 1 + w] = __ldg(in.idx[w] + pidx);
            }
            __syncwarp();
            const int cnt = (int)min(32u, tl.count - b * 32);
            for (int e0 = 0; e0 < cnt; e0 += U * E) {
                float val[U];
                uint32_t rowl[U];
                float y[U][N][C];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int e = e0 + u * E + sub;
                    const bool ok = e < cnt;
                    const uint32_t* sl = ws + (ok ? e : 0) * SW;
                    val[u] = ok ? __uint_as_float(sl[0]) : 0.f;
                    rowl[u] = ok ? sl[1 + n] - rbase : 0xffffffffu;
#pragma unroll
                    for (int w = 0; w < N; ++w) {
                        if (w == n) continue;
                        const uint32_t id = sl[1 + w];
#pragma unroll
                        for (int c = 0; c < C; ++c) y[u][w][c] = gather1<BF>(F, w, id, RP, gl + c * G);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (rowl[u] == 0xffffffffu) continue;
                    float* dst = yb + (size_t)rowl[u] * RP + gl;
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        float pr = val[u];
#pragma unroll
                        for (int w = 0; w < N; ++w)
                            if (w != n) pr *= y[u][w][c];
                        atomicAdd(dst + c * G, pr);
                    }
                    if (gl == 0) atomicOr(touched + (rowl[u] >> 5), 1u << (rowl[u] & 31));
                }
            }
            __syncwarp();
        }
    }
}

size_t priv_smem_bytes(int N, uint32_t m, int RP) {
    const int sw = (1 + N + 3) / 4 * 4;
    return (size_t)m * RP * 4 + (size_t)priv_flag_words(m) * 4 + (size_t)kPrivWarps * 32 * sw * 4;
}

constexpr size_t kPrivMaxSmem = 200 * 1024;

template <int N, bool BF>
int launch_priv(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles,
                const FacPtrs& F, int w0, int wl)
{
    const uint32_t m = 1u << p.shift[n];
    const size_t smem = priv_smem_bytes(N, m, p.Rp);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device);
    const int per_sm = smem <= 100 * 1024 ? 2 : 1;
    const uint32_t want = std::max<uint32_t>(1, std::min<uint32_t>(ntiles, (uint32_t)(sms * per_sm)));
    const uint32_t per_cta = (ntiles + want - 1) / want;
    const uint32_t grid = (ntiles + per_cta - 1) / per_cta;
    const SlabPtrs sp = slab_in(in, p.N);
#define DGPU_PRIV(RPV)                                                                           \
    do {                                                                                         \
        auto k = k_mttkrp_priv<N, RPV, BF>;                                                      \
        DGPU_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
        k<<<grid, kPrivThreads, smem, p.stream>>>(sp, tiles, ntiles, per_cta, F, p.Yhat[n], n,    \
                                                  w0, wl, p.shift[n], p.dims[n]);               \
    } while (0)
    switch (p.Rp) {
        case 16: DGPU_PRIV(16); break;
        case 32: DGPU_PRIV(32); break;
        case 64: DGPU_PRIV(64); break;
        default: DGPU_PRIV(128); break;
    }
#undef DGPU_PRIV
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

template <int N, bool BF>
int launch_rowrun(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles,
                  const FacPtrs& F0, int w0, int wl, int c0, int cols)
{
    // columns [c0, c0 + cols) of every factor (a rank tile when cols < Rp)
    const int C4 = cols / 4;
    // every row's nonzeros are contiguous in the slab when the mode is
    // fiber-sorted (each row lies in one shard, sorted by row)
    const int contiguous = (p.fiber && p.kclass[n] == 2) ? 1 : 0;
    const SlabPtrs sp = slab_in(in, p.N);
    float* out = p.Yhat[n] + c0;
    FacPtrs F = F0;
    for (int w = 0; w < p.N; ++w) {
        if (F.Y[w]) F.Y[w] += c0;
        if (F.Yb[w]) F.Yb[w] += c0;
    }
    // at least ~mttkrp_ctas_per_sm (default 4) CTAs per SM: split tiles
    // when the tensor has few of them
    const uint32_t want = (uint32_t)std::max(1, std::min(16, p.mttkrp_ctas_per_sm)) * (uint32_t)p.sms;
    const uint32_t split = ntiles >= want ? 1u : std::min(16u, (want + ntiles - 1) / std::max(1u, ntiles));
    const dim3 grid(ntiles, split);
#define DGPU_RUNT(G, V, TN)                                                                      \
    k_mttkrp_rowrun<N, G, V, BF, TN><<<grid, kRunThreads, 0, p.stream>>>(sp, tiles, F, out, n, \
                                                                         w0, wl, cols, p.Rp,     \
                                                                         contiguous)
#define DGPU_RUN(G, V) DGPU_RUNT(G, V, -1)
    // target-mode specialisations for the common 3- and 4-mode, Rp <= 128 shapes
#define DGPU_RUN_TGT(G)                                                       \
    do {                                                                      \
        if constexpr (N == 3 || N == 4) {                                     \
            if (n == 0) DGPU_RUNT(G, 1, 0);                                   \
            else if (n == 1) DGPU_RUNT(G, 1, 1);                              \
            else if (n == 2) DGPU_RUNT(G, 1, 2);                              \
            else DGPU_RUNT(G, 1, (N == 4 ? 3 : -1));                          \
        } else {                                                              \
            DGPU_RUN(G, 1);                                                   \
        }                                                                     \
    } while (0)
    if (C4 == 4) DGPU_RUN_TGT(4);
    else if (C4 == 8) DGPU_RUN_TGT(8);
    else if (C4 == 16) DGPU_RUN_TGT(16);
    else if (C4 == 32) DGPU_RUN_TGT(32);
    else if (C4 <= 64) DGPU_RUN(32, 2);
    else if (C4 <= 96) DGPU_RUN(32, 3);
    else if (C4 <= 128) DGPU_RUN(32, 4);
    else if (C4 <= 256) DGPU_RUN(32, 8);
    else {
        set_error("mttkrp: rank tile %d exceeds the supported maximum 1024", cols);
        return DGPU_ERR_ARG;
    }
#undef DGPU_RUN_TGT
#undef DGPU_RUN
#undef DGPU_RUNT
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

}  // namespace

// Which accumulation scheme mode n uses under this plan.
int mttkrp_scheme(const Plan& p, int n) {
    const bool priv_ok = (p.Rp == 16 || p.Rp == 32 || p.Rp == 64 || p.Rp == 128) &&
                         priv_smem_bytes(p.N, 1u << p.shift[n], p.Rp) <= kPrivMaxSmem;
    if (p.accum == DGPU_ACCUM_ROWRUN) return DGPU_ACCUM_ROWRUN;
    if (p.accum == DGPU_ACCUM_PRIVATE) return priv_ok ? DGPU_ACCUM_PRIVATE : DGPU_ACCUM_ROWRUN;
    const bool sorted = p.fiber && p.kclass[n] == 2;
    if (!sorted && priv_ok) return DGPU_ACCUM_PRIVATE;
    return DGPU_ACCUM_ROWRUN;
}

namespace {

template <int N, bool BF>
int launch_n(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles,
             const FacPtrs& F, int w0, int wl)
{
    if (mttkrp_scheme(p, n) == DGPU_ACCUM_PRIVATE)
        return launch_priv<N, BF>(p, n, in, tiles, ntiles, F, w0, wl);
    if (p.mttkrp_kernel == 1 && gather_supported(p, p.Rp))
        return launch_mttkrp_gather(p, n, in, tiles, ntiles, BF, wl,
                                    (p.fiber && p.kclass[n] == 2) ? 1 : 0);
    // Rank tiles: one pass over the slab per tile of `rt` columns.  Wide
    // factors gather whole rows per nonzero, which spills the hot rows out
    // of L1; narrower tiles re-read the slab but keep gathers cached.  The
    // tile width is tuned once per mode: the first call times each candidate
    // width (Rp, 128, 64, 32 that divide Rp) and keeps the fastest
    // (DGPU_RANK_TILE fixes it instead).
    auto run = [&](int rt) -> int {
        for (int c0 = 0; c0 < p.Rp; c0 += rt) {
            const int rc = launch_rowrun<N, BF>(p, n, in, tiles, ntiles, F, w0, wl, c0, rt);
            if (rc != DGPU_OK) return rc;
        }
        return DGPU_OK;
    };
    if (p.rank_tile > 0 && p.rank_tile <= p.Rp && p.Rp % p.rank_tile == 0 && p.rank_tile % 16 == 0)
        return run(p.rank_tile);
    int& chosen = p.tile_for[n];
    if (chosen == 0) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        DGPU_CUDA(cudaStreamIsCapturing(p.stream, &cs));
        if (p.Rp <= 64 || cs != cudaStreamCaptureStatusNone || p.timing) return run(p.Rp);
        const size_t yb = (size_t)p.dims[n] * p.Rp * sizeof(float);
        cudaEvent_t a, b;
        DGPU_CUDA(cudaEventCreate(&a));
        DGPU_CUDA(cudaEventCreate(&b));
        float best = 0.f;
        int best_rt = p.Rp;
        const int cands[4] = {p.Rp, 128, 64, 32};
        for (int ci = 0; ci < 4; ++ci) {
            const int rt = cands[ci];
            bool seen = false;
            for (int cj = 0; cj < ci; ++cj) seen = seen || cands[cj] == rt;
            if (seen || rt > p.Rp || p.Rp % rt != 0) continue;
            DGPU_CUDA(cudaMemsetAsync(p.Yhat[n], 0, yb, p.stream));
            DGPU_CUDA(cudaEventRecord(a, p.stream));
            DGPU_TRY(run(rt));
            DGPU_CUDA(cudaEventRecord(b, p.stream));
            DGPU_CUDA(cudaEventSynchronize(b));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            if (best == 0.f || ms < best) { best = ms; best_rt = rt; }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        chosen = best_rt;
        DGPU_CUDA(cudaMemsetAsync(p.Yhat[n], 0, yb, p.stream));
    }
    return run(chosen);
}

template <bool BF>
int launch_modes(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles,
                 const FacPtrs& F, int w0, int wl)
{
    switch (p.N) {
        case 2: return launch_n<2, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 3: return launch_n<3, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 4: return launch_n<4, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 5: return launch_n<5, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 6: return launch_n<6, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 7: return launch_n<7, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 8: return launch_n<8, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        default:
            set_error("mttkrp: %d modes unsupported (2..8)", p.N);
            return DGPU_ERR_ARG;
    }
}

__global__ void k_to_bf16(const float* __restrict__ y, __nv_bfloat16* __restrict__ yb, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        yb[i] = __float2bfloat16_rn(y[i]);
}

}  // namespace

int launch_to_bf16(Plan& p, int n) {
    const size_t cnt = (size_t)p.dims[n] * p.Rp;
    const unsigned blocks = (unsigned)std::min<size_t>((cnt + 255) / 256, 148 * 16);
    k_to_bf16<<<blocks, 256, 0, p.stream>>>(p.Y[n], p.Yb[n], cnt);
    DGPU_CUDA(cudaGetLastError());
    p.yb_stale[n] = false;
    return DGPU_OK;
}

int launch_mttkrp(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles) {
    if (ntiles == 0) return DGPU_OK;
    const int w0 = (n == 0) ? 1 : 0;
    int wl = -1;
    for (int w = p.N - 1; w >= 0; --w)
        if (w != n && w != w0) { wl = w; break; }
    FacPtrs F{};
    for (int w = 0; w < p.N; ++w) { F.Y[w] = p.Y[w]; F.Yb[w] = p.Yb[w]; }
    const bool bf = (p.precision == DGPU_PREC_BF16) && n != p.fp32_gather_mode &&
                    !p.gather_fp32_all;
    if (bf)
        for (int w = 0; w < p.N; ++w)
            if (w != n && p.yb_stale[w]) DGPU_TRY(launch_to_bf16(p, w));
    // algorithmic bytes: the slab once, every other factor once, Yhat once
    double bytes = (double)p.nnz * (4.0 + 4.0 * p.N) + (double)p.dims[n] * p.R * 4.0;
    for (int w = 0; w < p.N; ++w)
        if (w != n) bytes += (double)p.dims[w] * p.R * (bf ? 2.0 : 4.0);
    LaunchTimer t(p, KK_MTTKRP, bytes);
    if (bf) return launch_modes<true>(p, n, in, tiles, ntiles, F, w0, wl);
    return launch_modes<false>(p, n, in, tiles, ntiles, F, w0, wl);
}

}  // namespace dgpu
