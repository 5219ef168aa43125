// ============================================================================
//  mttkrp.cu -- mode-n sparse MTTKRP over a FLYCOO slab (sm_100a).
//
//  Replaces the reference's per-nnz kernel (src/dynasor_kernel.cpp:91-229,
//  fiber variant :365-489).  Arithmetic per nonzero is the reference's:
//      prod = val * Y[w0][i_w0, :]            (w0 = n==0 ? 1 : 0)
//      prod *= Y[w][i_w, :]                   (every other w except w_last)
//      Yhat[n][i_n, :] = fma(prod, Y[w_last][i_wl, :], Yhat[n][i_n, :])
//  (for N == 2 the last step is an add).  Gathers and products are FP32 (or
//  BF16 gathers widened to FP32); accumulation is FP32.
//
//  GPU mapping.  One CTA per work tile (<= kTile consecutive slab positions
//  of one super-shard, tiles in the reference's processing order).  A
//  "lane group" of G lanes owns one nonzero at a time; lane g holds float4
//  column chunk g (+ v*G) of the rank, so one warp-wide LDG.128 gathers
//  32/G factor rows.  Each group walks a contiguous run of the tile and
//  keeps the current output row's partial sum in registers; the sum is
//  written with one vector atomic (red.global.add.v4.f32) when the row
//  changes.  On a fiber-sorted slab (rows contiguous, the reference's
//  DenseFiber layout) that is one atomic per row segment; on an unsorted
//  slab it degrades to one per nonzero, which stays correct.
// ============================================================================
#include "dgpu_internal.h"

#include <algorithm>

namespace dgpu {

namespace {

constexpr int kThreads = 256;

struct FacPtrs {
    const float*         Y[kMaxModes];
    const __nv_bfloat16* Yb[kMaxModes];
};

template <bool BF>
__device__ __forceinline__ float4 gather4(const FacPtrs& F, int w, uint32_t row, int Rp, int c4) {
    if constexpr (BF) {
        const uint2 raw = __ldg(reinterpret_cast<const uint2*>(F.Yb[w] + (size_t)row * Rp) + c4);
        const __nv_bfloat162 lo = *reinterpret_cast<const __nv_bfloat162*>(&raw.x);
        const __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162*>(&raw.y);
        const float2 a = __bfloat1622float2(lo), b = __bfloat1622float2(hi);
        return make_float4(a.x, a.y, b.x, b.y);
    } else {
        return __ldg(reinterpret_cast<const float4*>(F.Y[w] + (size_t)row * Rp) + c4);
    }
}

__device__ __forceinline__ float4 mul4(float4 a, float4 b) {
    return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
}
__device__ __forceinline__ float4 scale4(float4 a, float s) {
    return make_float4(s * a.x, s * a.y, s * a.z, s * a.w);
}
__device__ __forceinline__ float4 fma4(float4 a, float4 b, float4 c) {
    return make_float4(__fmaf_rn(a.x, b.x, c.x), __fmaf_rn(a.y, b.y, c.y),
                       __fmaf_rn(a.z, b.z, c.z), __fmaf_rn(a.w, b.w, c.w));
}
__device__ __forceinline__ float4 add4(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// Elements per batch: keeps (N-1)*V*U float4 gathers in flight per lane.
template <int N, int V>
struct Batch {
    static constexpr int kWork = (N - 1) * V;
    static constexpr int U = kWork <= 2 ? 4 : (kWork <= 4 ? 2 : 1);
};

template <int N, int G, int V, bool BF>
__global__ void __launch_bounds__(kThreads)
k_mttkrp_rowrun(SlabPtrs in, const uint32_t* __restrict__ rowcol,
                const Tile* __restrict__ tiles, FacPtrs F, float* __restrict__ Yhat,
                int n, int w0, int wl, int Rp)
{
    constexpr int U = Batch<N, V>::U;
    const int gl = threadIdx.x % G;
    const int grp = threadIdx.x / G;
    constexpr int kGroups = kThreads / G;
    const int C4 = Rp >> 2;

    const Tile tl = tiles[blockIdx.x];
    const uint32_t per = (tl.count + kGroups - 1) / kGroups;
    const uint32_t gb = min(tl.count, (uint32_t)grp * per);
    const uint32_t ge = min(tl.count, gb + per);

    float4 acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t cur = 0xffffffffu;

    auto flush = [&](uint32_t row) {
        float4* out = reinterpret_cast<float4*>(Yhat + (size_t)row * Rp);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int c4 = gl + v * G;
            if (V == 1 || c4 < C4) atomicAdd(out + c4, acc[v]);
            acc[v] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };

    for (uint32_t j0 = gb; j0 < ge; j0 += U) {
        float    val[U];
        uint32_t row[U];
        uint32_t id[U][N];
        bool     ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            ok[u] = (j0 + u) < ge;
            const uint32_t p = tl.begin + (ok[u] ? j0 + u : gb);
            val[u] = __ldg(in.vals + p);
            row[u] = __ldg(rowcol + p);
#pragma unroll
            for (int w = 0; w < N; ++w) id[u][w] = (w == n) ? 0u : __ldg(in.idx[w] + p);
        }
        float4 y[U][N][V];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int w = 0; w < N; ++w) {
                if (w == n) continue;
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int c4 = gl + v * G;
                    y[u][w][v] = (V == 1 || c4 < C4) ? gather4<BF>(F, w, id[u][w], Rp, c4)
                                                     : make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            if (row[u] != cur) {
                if (cur != 0xffffffffu) flush(cur);
                cur = row[u];
            }
            // Non-target modes in increasing order: the first starts the
            // product (w0), the middle ones multiply, the last (w_last) is
            // fused into the accumulate -- the reference's operation order.
#pragma unroll
            for (int v = 0; v < V; ++v) {
                float4 pr = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int w = 0; w < N; ++w) {
                    if (w == n) continue;
                    if (w == w0)      pr = scale4(y[u][w][v], val[u]);
                    else if (w == wl) acc[v] = fma4(pr, y[u][w][v], acc[v]);
                    else              pr = mul4(pr, y[u][w][v]);
                }
                if (wl < 0) acc[v] = add4(acc[v], pr);
            }
        }
    }
    if (cur != 0xffffffffu) flush(cur);
}

template <int N, bool BF>
int dispatch_rowrun(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles,
                    const FacPtrs& F, int w0, int wl)
{
    const int C4 = p.Rp / 4;
    const SlabPtrs sp = slab_in(in, p.N);
    float* out = p.Yhat[n];
#define DGPU_LAUNCH(G, V) \
    k_mttkrp_rowrun<N, G, V, BF><<<ntiles, kThreads, 0, p.stream>>>(sp, in.idx[n], tiles, F, out, n, w0, wl, p.Rp)
    if (C4 == 4) DGPU_LAUNCH(4, 1);
    else if (C4 == 8) DGPU_LAUNCH(8, 1);
    else if (C4 == 16) DGPU_LAUNCH(16, 1);
    else if (C4 == 32) DGPU_LAUNCH(32, 1);
    else if (C4 <= 64) DGPU_LAUNCH(32, 2);
    else if (C4 <= 96) DGPU_LAUNCH(32, 3);
    else if (C4 <= 128) DGPU_LAUNCH(32, 4);
    else if (C4 <= 256) DGPU_LAUNCH(32, 8);
    else {
        set_error("mttkrp: rank_padded %d exceeds the supported maximum 1024", p.Rp);
        return DGPU_ERR_ARG;
    }
#undef DGPU_LAUNCH
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

template <bool BF>
int dispatch_modes(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles,
                   const FacPtrs& F, int w0, int wl)
{
    switch (p.N) {
        case 2: return dispatch_rowrun<2, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 3: return dispatch_rowrun<3, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 4: return dispatch_rowrun<4, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 5: return dispatch_rowrun<5, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 6: return dispatch_rowrun<6, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 7: return dispatch_rowrun<7, BF>(p, n, in, tiles, ntiles, F, w0, wl);
        case 8: return dispatch_rowrun<8, BF>(p, n, in, tiles, ntiles, F, w0, wl);
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
    const bool bf = (p.precision == DGPU_PREC_BF16);
    if (bf)
        for (int w = 0; w < p.N; ++w)
            if (w != n && p.yb_stale[w]) DGPU_TRY(launch_to_bf16(p, w));
    // algorithmic bytes: the slab once, every other factor once, Yhat once
    double bytes = (double)p.nnz * (4.0 + 4.0 * p.N) + (double)p.dims[n] * p.R * 4.0;
    for (int w = 0; w < p.N; ++w)
        if (w != n) bytes += (double)p.dims[w] * p.R * (bf ? 2.0 : 4.0);
    LaunchTimer t(p, KK_MTTKRP, bytes);
    if (bf) return dispatch_modes<true>(p, n, in, tiles, ntiles, F, w0, wl);
    return dispatch_modes<false>(p, n, in, tiles, ntiles, F, w0, wl);
}

}  // namespace dgpu
