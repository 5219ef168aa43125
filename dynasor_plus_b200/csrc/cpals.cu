// ============================================================================
//  cpals.cu -- CP-ALS on the device (replaces cpals, src/dynasor_cpals.cpp:
//  120-396, and la::*, src/dynasor_linalg.cpp:47-402).
//
//  Per Gauss-Seidel mode update (after the mode-n MTTKRP):
//    k_build_solve_map  one CTA: V = Hadamard_{m!=n} G[m] (FP64), relative
//                       ridge, right-looking Cholesky, and the linear map W
//                       with  y = yhat * W  equal to the reference's forward
//                       + backward substitution (zero pivot -> component 0,
//                       negative pivot clamped, linalg.cpp:181-245).  FP64
//                       by default; FP32 for the plain-FP32 path.
//    k_apply_map        Y[n] = Yhat[n] * W, FP64 (or FP32) accumulation.
//    k_gram_partial     per-chunk partial Grams of Y[n] (FP32 in-chunk sums,
//                       FP64 partials).
//    k_finalize_mode    one CTA: G_un = sum of partials, lambda_r =
//                       sqrt(G_un[r,r]), G[n] = G_un / (lambda lambda^T),
//                       i.e. the Gram of the column-normalised factor.
//    k_scale_cols       Y[n][:, r] /= lambda_r (lambda <= 1e-20 -> 0), and
//                       on the last mode the per-column <Y, Yhat> partials
//                       of the fit.
//    k_fit              one CTA: <T,M> = sum_r lambda_r <Y_r, Yhat_r>,
//                       ||M||^2 = lambda^T (Hadamard_n G[n]) lambda, all
//                       FP64 (the reference truncates <T,M> to FP32,
//                       linalg.cpp:365; this keeps FP64 throughout).
//  Grams are kept in FP64 between modes.
// ============================================================================
#include <functional>
#include "dgpu_internal.h"
#include "la_warp.cuh"
#include "apply_map.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <vector>

namespace dgpu {

int mode_pingpong(Plan& p, int n);
int mode_pingpong_then(Plan& p, int n, const std::function<int()>& after);
int mode_ncopy(Plan& p, int n);

namespace {

constexpr int kLaThreads = 256;
#ifndef DGPU_SMALL_THREADS
#define DGPU_SMALL_THREADS 1024
#endif
constexpr int kSmallThreads = DGPU_SMALL_THREADS;   // threads of the one-CTA factor update
constexpr int kGramTile = 32;
constexpr int kGramChunks = 296;           // 2 per SM

// ---------------------------------------------------------------------------
template <typename Real>
__global__ void __launch_bounds__(1024)
k_build_solve_map(const double* __restrict__ Gd, int N, int n, int R, double ridge,
                  Real* __restrict__ A, double* __restrict__ Wd, float* __restrict__ W32)
{
    // A: R x R work matrix (global scratch, L1/L2 resident).
    const int tid = threadIdx.x, nt = blockDim.x;
    const size_t RR = (size_t)R * R;
    for (size_t e = tid; e < RR; e += nt) {
        double v = 1.0;
        for (int m = 0; m < N; ++m)
            if (m != n) v *= Gd[(size_t)m * RR + e];
        A[e] = (Real)v;
    }
    __syncthreads();
    __shared__ Real s_eps;
    if (tid == 0) {
        Real dmax = 0;
        for (int r = 0; r < R; ++r) dmax = max(dmax, A[(size_t)r * R + r]);
        s_eps = max((Real)ridge * dmax, (Real)0);
    }
    __syncthreads();
    for (int r = tid; r < R; r += nt) A[(size_t)r * R + r] += s_eps;
    __syncthreads();

    // Right-looking Cholesky (lower), column by column.
    for (int j = 0; j < R; ++j) {
        __shared__ Real s_d, s_inv;
        if (tid == 0) {
            Real s = A[(size_t)j * R + j];
            if (s < (Real)0) s = 0;
            const Real d = sqrt(s);
            A[(size_t)j * R + j] = d;
            s_d = d;
            s_inv = d > (Real)0 ? (Real)1 / d : (Real)0;
        }
        __syncthreads();
        for (int i = j + 1 + tid; i < R; i += nt) A[(size_t)i * R + j] *= s_inv;
        __syncthreads();
        // trailing update of the lower triangle: A[i][k] -= A[i][j]*A[k][j]
        const int m = R - j - 1;
        const long tot = (long)m * (m + 1) / 2;
        for (long e = tid; e < tot; e += nt) {
            // map e -> (i, k) with k <= i in the trailing block
            int i = (int)((sqrt(8.0 * (double)e + 1.0) - 1.0) * 0.5);
            while ((long)(i + 1) * (i + 2) / 2 <= e) ++i;
            while ((long)i * (i + 1) / 2 > e) --i;
            const int k = (int)(e - (long)i * (i + 1) / 2);
            const int ii = j + 1 + i, kk = j + 1 + k;
            A[(size_t)ii * R + kk] -= A[(size_t)ii * R + j] * A[(size_t)kk * R + j];
        }
        __syncthreads();
    }

    // W: row c of the map is the solve applied to unit vector e_c, i.e.
    // x = solve(e_c); y_row = yhat_row * W with W[c][:] = x.
    for (int c = tid; c < R; c += nt) {
        double* x = Wd + (size_t)c * R;
        for (int r = 0; r < R; ++r) x[r] = (r == c) ? 1.0 : 0.0;
        for (int r = 0; r < R; ++r) {                       // L z = b
            Real s = (Real)x[r];
            for (int k = 0; k < r; ++k) s -= A[(size_t)r * R + k] * (Real)x[k];
            const Real d = A[(size_t)r * R + r];
            x[r] = d > (Real)0 ? (double)(s / d) : 0.0;
        }
        for (int r = R - 1; r >= 0; --r) {                  // L^T x = z
            Real s = (Real)x[r];
            for (int k = r + 1; k < R; ++k) s -= A[(size_t)k * R + r] * (Real)x[k];
            const Real d = A[(size_t)r * R + r];
            x[r] = d > (Real)0 ? (double)(s / d) : 0.0;
        }
        for (int r = 0; r < R; ++r) W32[(size_t)c * R + r] = (float)x[r];
    }
}

// Y[i][c] = sum_k Yhat[i][k] * W[k][c]   (padding columns written as 0)
template <typename Real>
__global__ void __launch_bounds__(kLaThreads)
k_apply_map(const float* __restrict__ Yhat, uint32_t rows, int R, int Rp,
            const Real* __restrict__ W, float* __restrict__ Y)
{
    extern __shared__ unsigned char smem_raw[];
    Real* Ws = reinterpret_cast<Real*>(smem_raw);            // R x R
    for (int e = threadIdx.x; e < R * R; e += blockDim.x) Ws[e] = W[e];
    __syncthreads();
    // a thread takes one row and four columns: each Yhat entry is loaded
    // once per four outputs (16-byte loads), each output keeps its single
    // k-ordered sum
    const int groups = Rp >> 2;
    const size_t items = (size_t)rows * groups;
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < items;
         w += (size_t)gridDim.x * blockDim.x) {
        const size_t i = w / groups;
        const int c0 = (int)(w - i * groups) * 4;
        const float4* yh = reinterpret_cast<const float4*>(Yhat + i * Rp);
        Real s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int k4 = 0; k4 < R; k4 += 4) {
            const float4 h4 = __ldg(yh + (k4 >> 2));
            const float hv[4] = {h4.x, h4.y, h4.z, h4.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k4 + u;
                if (k >= R) break;
                const Real h = (Real)hv[u];
                const Real* wr = Ws + (size_t)k * R + c0;
                if (c0 < R) s0 += h * wr[0];
                if (c0 + 1 < R) s1 += h * wr[1];
                if (c0 + 2 < R) s2 += h * wr[2];
                if (c0 + 3 < R) s3 += h * wr[3];
            }
        }
        float4 out;
        out.x = c0 < R ? (float)s0 : 0.f;
        out.y = c0 + 1 < R ? (float)s1 : 0.f;
        out.z = c0 + 2 < R ? (float)s2 : 0.f;
        out.w = c0 + 3 < R ? (float)s3 : 0.f;
        reinterpret_cast<float4*>(Y + i * Rp)[c0 >> 2] = out;
    }
}

// The same map for Rp = RP in {16, 32}: lane c of a warp (c = lane % RP)
// owns output column c with column c of W in registers; a warp stages 8
// rows of Yhat (converted to Real) in its own shared-memory slice and reads
// them back as broadcasts, so each Yhat entry is converted once and each
// loaded pair of entries feeds a multiply-add in every lane.  The next 8
// rows are loaded while the current ones are multiplied.  Each output is the
// same k-ordered fused multiply-add chain as in k_apply_map.
template <typename Real, int RP>
__global__ void __launch_bounds__(kLaThreads, 2)
k_apply_map_lanes(const float* __restrict__ Yhat, uint32_t rows, int R,
                  const Real* __restrict__ W, float* __restrict__ Y)
{
    static_assert(RP == 16 || RP == 32, "one or two rows per warp pass");
    constexpr int RW = 32 / RP;                          // rows per warp pass
    constexpr int V4 = kMapRows * RP / 4 / 32;            // float4 loads per lane per block
    __shared__ __align__(16) Real hs[kLaThreads / 32][kMapRows][RP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c = lane % RP, sub = lane / RP;
    Real w[RP];
#pragma unroll
    for (int k = 0; k < RP; ++k) w[k] = (k < R && c < R) ? W[(size_t)k * R + c] : (Real)0;
    const uint32_t nblocks = (rows + kMapRows - 1) / kMapRows;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const float4* src = reinterpret_cast<const float4*>(Yhat);
    const size_t n4 = (size_t)rows * RP / 4;
    float4 pf[V4];
    auto load = [&](uint32_t b) {
#pragma unroll
        for (int v = 0; v < V4; ++v) {
            const size_t q = (size_t)b * (kMapRows * RP / 4) + v * 32 + lane;
            pf[v] = q < n4 ? __ldg(src + q) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };
    uint32_t b = gw;
    if (b < nblocks) load(b);
    for (; b < nblocks; b += nw) {
        Real* hw = &hs[warp][0][0];
#pragma unroll
        for (int v = 0; v < V4; ++v) {
            const int e = (v * 32 + lane) * 4;               // element within the block
            hw[e] = (Real)pf[v].x; hw[e + 1] = (Real)pf[v].y;
            hw[e + 2] = (Real)pf[v].z; hw[e + 3] = (Real)pf[v].w;
        }
        __syncwarp();
        if (b + nw < nblocks) load(b + nw);
#pragma unroll
        for (int r0 = 0; r0 < kMapRows; r0 += RW) {
            const int r = r0 + sub;
            const Real* h = &hs[warp][r][0];
            Real acc = 0;
#pragma unroll
            for (int k = 0; k < RP; k += 2) {
                Real h0, h1;
                if constexpr (sizeof(Real) == 8) {
                    const double2 hv = *reinterpret_cast<const double2*>(h + k);
                    h0 = hv.x; h1 = hv.y;
                } else {
                    const float2 hv = *reinterpret_cast<const float2*>(h + k);
                    h0 = hv.x; h1 = hv.y;
                }
                if constexpr (sizeof(Real) == 8) {
                    if (k < R) acc = fma(h0, w[k], acc);
                    if (k + 1 < R) acc = fma(h1, w[k + 1], acc);
                } else {
                    if (k < R) acc = fmaf(h0, w[k], acc);
                    if (k + 1 < R) acc = fmaf(h1, w[k + 1], acc);
                }
            }
            const uint32_t i = b * kMapRows + r;
            if (i < rows) Y[(size_t)i * RP + c] = c < R ? (float)acc : 0.f;
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;"
                 :: "r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))), "l"(src),
                    "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }

// Rows a partial-Gram CTA stages per step, and steps in flight.
constexpr int kGramRows = 64;
constexpr int kGramStages = 4;
constexpr size_t kGramSmem = 2 * (size_t)kGramStages * kGramRows * kGramTile * sizeof(float);

// Partial Grams: grid (chunks, tilesA, tilesB), 32 x 32 output tile per CTA,
// 16 outputs per thread.  partial[(chunk * R + a) * R + b] (FP64).
__global__ void __launch_bounds__(kLaThreads, 2)
k_gram_partial(const float* __restrict__ Y, uint32_t rows, int R, int Rp,
               double* __restrict__ partial)
{
    // A block sums one chunk of rows for one (a, b) pair of 32-column tiles.
    // Thread = (row group g of 4, a-block ta of 8, b-block tb of 8) with a
    // 4 x 4 register tile: per row it reads two 16-byte vectors from shared
    // memory for 16 FMAs.  The four row groups take interleaved rows; their
    // sums are added in a fixed order at the end.  Rows stream into a
    // kGramStages-deep ring of shared-memory stages with 16-byte cp.async
    // copies (zero fill past the chunk and past Rp), so three steps of loads
    // are in flight while one is multiplied.  Columns >= R only reach Gram
    // entries that are not stored.
    static_assert(kLaThreads == 256 && kGramTile == 32, "4 row groups x 8 x 8 threads");
    extern __shared__ __align__(16) float gsm[];
    typedef float Stage[kGramRows][kGramTile];
    Stage* sa = reinterpret_cast<Stage*>(gsm);
    Stage* sb = sa + kGramStages;
    const int a0 = blockIdx.y * kGramTile, b0 = blockIdx.z * kGramTile;
    const bool same = (a0 == b0);
    const int g = threadIdx.x >> 6, u = threadIdx.x & 63;
    const int ta = u & 7, tb = u >> 3;
    const uint32_t chunk = (rows + gridDim.x - 1) / gridDim.x;
    const uint32_t r0 = min(rows, blockIdx.x * chunk), r1 = min(rows, r0 + chunk);
    const uint32_t nsteps = (r1 - r0 + kGramRows - 1) / kGramRows;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    auto issue = [&](uint32_t st) {
        const uint32_t base = r0 + st * kGramRows;
        const uint32_t nr = min((uint32_t)kGramRows, r1 - base);
        Stage& da = sa[st % kGramStages];
        Stage& db = sb[st % kGramStages];
#pragma unroll
        for (int k = 0; k < kGramRows * (kGramTile / 4) / kLaThreads; ++k) {
            const int q = threadIdx.x + k * kLaThreads;
            const int rr = q >> 3, c4 = q & 7;
            const bool rowok = (uint32_t)rr < nr;
            const float* row = Y + (size_t)(base + (rowok ? rr : 0)) * Rp;
            const int ca = a0 + 4 * c4;
            const bool oka = rowok && ca + 4 <= Rp;
            cp_async16(&da[rr][4 * c4], oka ? row + ca : Y, oka ? 16 : 0);
            if (!same) {
                const int cb = b0 + 4 * c4;
                const bool okb = rowok && cb + 4 <= Rp;
                cp_async16(&db[rr][4 * c4], okb ? row + cb : Y, okb ? 16 : 0);
            }
        }
    };
#pragma unroll
    for (int st = 0; st < kGramStages - 1; ++st) {
        if ((uint32_t)st < nsteps) issue(st);
        cp_async_commit();
    }
    for (uint32_t st = 0; st < nsteps; ++st) {
        cp_async_wait<kGramStages - 2>();
        __syncthreads();           // step st landed for every thread; step st-1 consumed
        if (st + kGramStages - 1 < nsteps) issue(st + kGramStages - 1);
        cp_async_commit();
        const uint32_t nr = min((uint32_t)kGramRows, r1 - (r0 + st * kGramRows));
        const float (*A)[kGramTile] = sa[st % kGramStages];
        const float (*B)[kGramTile] = same ? A : sb[st % kGramStages];
#pragma unroll 4
        for (uint32_t rr = g; rr < nr; rr += 4) {
            const float4 av = *reinterpret_cast<const float4*>(&A[rr][4 * ta]);
            const float4 bv = *reinterpret_cast<const float4*>(&B[rr][4 * tb]);
            const float x[4] = {av.x, av.y, av.z, av.w};
            const float y[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(x[i], y[j], acc[i][j]);
        }
    }
    cp_async_wait<0>();
    __syncthreads();               // every stage consumed: reuse it for the row-group sums
    float (*red)[kGramTile][kGramTile + 1] = reinterpret_cast<float (*)[kGramTile][kGramTile + 1]>(gsm);
    if (g > 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) red[g - 1][4 * ta + i][4 * tb + j] = acc[i][j];
    }
    __syncthreads();
    if (g == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int a = a0 + 4 * ta + i, b = b0 + 4 * tb + j;
                const double v = (double)acc[i][j] + (double)red[0][4 * ta + i][4 * tb + j] +
                                 (double)red[1][4 * ta + i][4 * tb + j] +
                                 (double)red[2][4 * ta + i][4 * tb + j];
                if (a < R && b < R) partial[((size_t)blockIdx.x * R + a) * R + b] = v;
            }
    }
}

// Launches k_gram_partial (its shared memory is above the 48 KB default).
int launch_gram_partial(dim3 grid, cudaStream_t st, const float* Y, uint32_t rows, int R, int Rp,
                        double* partial) {
    // once per device (function attributes are per context); batched runs
    // set up several plans on parallel host threads
    static std::mutex mu;
    static bool attr_set[64] = {};
    int dev = 0;
    DGPU_CUDA(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!attr_set[dev & 63]) {
            DGPU_CUDA(cudaFuncSetAttribute(k_gram_partial,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kGramSmem));
            attr_set[dev & 63] = true;
        }
    }
    k_gram_partial<<<grid, kLaThreads, kGramSmem, st>>>(Y, rows, R, Rp, partial);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

// Sums the `chunks` partial Grams into partial[0 .. RR) (in place): a CTA
// takes 32 entries, its 8 warps take 8 consecutive runs of chunks and the
// 8 run sums are added in run order, so the result does not depend on
// timing.  Spreading the 2.4 MB of partials of a large mode over many SMs
// replaces one CTA reading all of them.
__global__ void __launch_bounds__(256)
k_reduce_partials(double* __restrict__ partial, int chunks, int RR)
{
    __shared__ double run[8][32];
    const int el = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int e = blockIdx.x * 32 + el;
    const int per = (chunks + 7) / 8;
    const int c0 = min(chunks, w * per), c1 = min(chunks, c0 + per);
    double s = 0.0;
    if (e < RR) {
#pragma unroll 4
        for (int c = c0; c < c1; ++c) s += partial[(size_t)c * RR + e];
    }
    run[w][el] = s;
    __syncthreads();
    if (w == 0 && e < RR) {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) t += run[k][el];
        partial[e] = t;
    }
}

// Reduce partial Grams; if `normalise`, lambda = sqrt(diag) and the Gram of
// the column-normalised factor is stored; else the raw Gram.
__global__ void __launch_bounds__(1024)
k_finalize_mode(const double* __restrict__ partial, int chunks, int R, int ldo, int normalise,
                double* __restrict__ Gd_n, float* __restrict__ G32_n,
                float* __restrict__ lambda, double* __restrict__ lam64)
{
    const size_t RR = (size_t)R * R;
    for (size_t e = threadIdx.x; e < RR; e += blockDim.x) {
        double s = 0;
        // in chunk order; unrolled so that the loads are in flight together
#pragma unroll 8
        for (int c = 0; c < chunks; ++c) s += partial[(size_t)c * RR + e];
        Gd_n[e] = s;
    }
    __syncthreads();
    if (normalise) {
        for (int r = threadIdx.x; r < R; r += blockDim.x) {
            const double l = sqrt(max(Gd_n[(size_t)r * R + r], 0.0));
            lam64[r] = l;
            lambda[r] = (float)l;
        }
        __syncthreads();
        for (size_t e = threadIdx.x; e < RR; e += blockDim.x) {
            const int a = (int)(e / R), b = (int)(e % R);
            const double la = lam64[a], lb = lam64[b];
            const double ia = la > 1e-20 ? 1.0 / la : 0.0, ib = lb > 1e-20 ? 1.0 / lb : 0.0;
            Gd_n[e] = Gd_n[e] * ia * ib;
        }
        __syncthreads();
    }
    for (size_t e = threadIdx.x; e < RR; e += blockDim.x)
        G32_n[(e / R) * ldo + e % R] = (float)Gd_n[e];
}

// Y[:, r] *= 1/lambda_r; with Yhat != null also per-CTA partial sums of
// Y_norm[:, r] * Yhat[:, r] (FP64) for the fit.
__global__ void __launch_bounds__(kLaThreads)
k_scale_cols(float* __restrict__ Y, const float* __restrict__ Yhat, uint32_t rows, int R, int Rp,
             const double* __restrict__ lam64, double* __restrict__ dot_partial)
{
    extern __shared__ double sdot[];   // [R], then R floats: 1 / lambda per column
    float* invs = reinterpret_cast<float*>(sdot + R);
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        sdot[r] = 0.0;
        const double l = lam64[r];
        invs[r] = l > 1e-20 ? (float)(1.0 / l) : 0.f;
    }
    __syncthreads();
    const size_t total = (size_t)rows * Rp;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t first = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int C4 = Rp >> 2;
    if ((Rp & 3) == 0 && stride % C4 == 0) {
        // float4 per thread, every float4 this thread visits in one group of
        // four columns; four float4 of Y (and of Yhat) in flight at once
        constexpr int U = 4;
        const int c0 = (int)(first % C4) * 4;
        float inv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) inv[j] = c0 + j < R ? invs[c0 + j] : 0.f;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        float4* Y4 = reinterpret_cast<float4*>(Y);
        const float4* H4 = reinterpret_cast<const float4*>(Yhat);
        const size_t total4 = total >> 2;
        for (size_t q = first; q < total4; q += U * stride) {
            float4 y[U], h[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const size_t qq = q + u * stride;
                y[u] = qq < total4 ? Y4[qq] : make_float4(0.f, 0.f, 0.f, 0.f);
                h[u] = (Yhat && qq < total4) ? __ldg(H4 + qq) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const size_t qq = q + u * stride;
                if (qq >= total4) break;
                const float4 v = make_float4(y[u].x * inv[0], y[u].y * inv[1], y[u].z * inv[2],
                                             y[u].w * inv[3]);
                Y4[qq] = v;
                if (Yhat) {
                    acc[0] += (double)v.x * (double)h[u].x;
                    acc[1] += (double)v.y * (double)h[u].y;
                    acc[2] += (double)v.z * (double)h[u].z;
                    acc[3] += (double)v.w * (double)h[u].w;
                }
            }
        }
        if (Yhat) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (c0 + j < R) atomicAdd(&sdot[c0 + j], acc[j]);
        }
    } else if (Yhat && stride % Rp == 0) {
        // every element this thread visits is in one column: one atomic
        const int c = (int)(first % Rp);
        double acc = 0.0;
        if (c < R) {
            const float inv = invs[c];
            for (size_t e = first; e < total; e += stride) {
                const float y = Y[e] * inv;
                Y[e] = y;
                acc += (double)y * (double)Yhat[e];
            }
            atomicAdd(&sdot[c], acc);
        }
    } else {
        for (size_t e = first; e < total; e += stride) {
            const int c = (int)(e % Rp);
            if (c >= R) continue;
            const float y = Y[e] * invs[c];
            Y[e] = y;
            if (Yhat) atomicAdd(&sdot[c], (double)y * (double)Yhat[e]);
        }
    }
    __syncthreads();
    if (Yhat)
        for (int r = threadIdx.x; r < R; r += blockDim.x)
            dot_partial[(size_t)blockIdx.x * R + r] = sdot[r];
}

__global__ void __launch_bounds__(1024)
k_fit(const double* __restrict__ Gd, int N, int R, const double* __restrict__ lam64,
      const double* __restrict__ dot_partial, int nblk, double tnorm2,
      double* __restrict__ out /* [inner, mnrm2, fit, resid] */)
{
    __shared__ double red[1024];
    const size_t RR = (size_t)R * R;
    double s_in = 0;
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        double d = 0;
        for (int b = 0; b < nblk; ++b) d += dot_partial[(size_t)b * R + r];
        s_in += lam64[r] * d;
    }
    double s_m = 0;
    for (size_t e = threadIdx.x; e < RR; e += blockDim.x) {
        double h = 1.0;
        for (int m = 0; m < N; ++m) h *= Gd[(size_t)m * RR + e];
        s_m += lam64[e / R] * lam64[e % R] * h;
    }
    red[threadIdx.x] = s_in;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double inner = red[0];
    __syncthreads();
    red[threadIdx.x] = s_m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double m2 = max(0.0, red[0]);
        double r2 = tnorm2 - 2.0 * inner + m2;
        if (r2 < 0.0) r2 = 0.0;
        const double resid = sqrt(r2);
        out[0] = inner;
        out[1] = m2;
        out[2] = 1.0 - resid / max(sqrt(tnorm2), 1e-30);
        out[3] = resid;
    }
}

// The solve map of mode n alone (one warp): V = Hadamard of the other
// modes' Grams, ridge, Cholesky, W -> Wout (FP64, entry (r, c) at
// Wout[r * R + c]).  It depends only on the other modes' Grams, so it runs
// on a side stream while mode n's MTTKRP runs.
template <typename Real>
__global__ void __launch_bounds__(32)
k_small_solve(const double* __restrict__ Gd, int N, int n, int R, double ridge,
              double* __restrict__ Wout)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const int RR = R * R, LDA = R + 1;
    double* Wx = reinterpret_cast<double*>(smraw);
    Real* A = reinterpret_cast<Real*>(Wx + RR);
    Real* invd = A + R * LDA;
    // Hadamard of the other modes' Grams, eight entries per lane at a time
    // with every mode's loads issued before the products
    for (int e0 = threadIdx.x; e0 < RR; e0 += 32 * 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = 1.0;
        for (int m = 0; m < N; ++m) {
            if (m == n) continue;
            double g[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = e0 + 32 * u;
                g[u] = e < RR ? __ldg(Gd + (size_t)m * RR + e) : 1.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] *= g[u];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + 32 * u;
            if (e < RR) A[(e / R) * LDA + e % R] = (Real)v[u];
        }
    }
    __syncwarp();
    // R <= 16: factor and map in registers (a 32-wide register version does
    // not stay unrolled); wider ranks use the shared-memory solve
    if (R <= 16) {
        warp_ridge<Real>(A, LDA, R, ridge);
        warp_chol_solve_map_reg<Real, 16>(A, LDA, R, invd, Wx);
    } else {
        warp_chol_solve_map<Real>(A, LDA, R, invd, Wx, ridge);
    }
    for (int e = threadIdx.x; e < RR; e += 32) Wout[e] = Wx[e];
}

// The whole factor update of a small mode in one CTA (rows * Rp <= 8192,
// R <= 64; the new factor is built in shared memory): Hadamard of the other Grams + relative ridge, Cholesky, the
// solve map W, Y = Yhat W, the Gram of Y, lambda from its diagonal, the
// normalised Gram, column scaling and, for the last mode, the fit.  The same
// arithmetic as the multi-kernel path (k_build_solve_map, k_apply_map,
// k_gram_partial, k_finalize_mode, k_scale_cols, k_fit) except that the
// Gram is summed in FP64 throughout; one launch instead of six keeps small
// tensors from being bound by launch latency.
template <typename Real>
__global__ void __launch_bounds__(1024)
k_update_small(double* __restrict__ Gd, float* __restrict__ G32, int N, int n, int R, int Rp,
               double ridge, const float* __restrict__ Yhat, float* __restrict__ Y, uint32_t rows,
               float* __restrict__ lambda, double* __restrict__ lam64, int last, double tnorm2,
               double* __restrict__ fitout, const double* __restrict__ Wpre)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const int RR = R * R;
    double* Wx = reinterpret_cast<double*>(smraw);         // R x R solve map (FP64)
    double* G = Wx + RR;                                    // R x R Gram
    double* lam = G + RR;                                   // R
    double* dot = lam + R;                                  // R
    const int LDA = R + 1;                                  // padded: lanes own rows
    Real* A = reinterpret_cast<Real*>(dot + R);             // R x LDA Cholesky work
    Real* invd = A + R * LDA;                               // R: 1 / pivot (0 for a zero pivot)
    float* Ys = reinterpret_cast<float*>(invd + R);         // rows x Rp: the new factor
    float* Hs = Ys + (size_t)rows * Rp;                     // rows x Rp: Yhat
    __shared__ double red[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    const uint32_t total = rows * (uint32_t)Rp;
    for (uint32_t e = tid; e < total; e += nt) Hs[e] = __ldg(Yhat + e);

    for (int e = tid; e < RR; e += nt) {
        if (Wpre) {
            Wx[e] = Wpre[e];
        } else {
            double v = 1.0;
            for (int m = 0; m < N; ++m)
                if (m != n) v *= Gd[(size_t)m * RR + e];
            A[(e / R) * LDA + e % R] = (Real)v;
        }
        G[e] = 0.0;
    }
    for (int r = tid; r < R; r += nt) dot[r] = 0.0;
    __syncthreads();
    // ridge, Cholesky and the solve map in warp 0 alone (warp barriers
    // only); the other warps wait at the next block barrier.  With Wpre the
    // map was built by k_small_solve while this mode's MTTKRP ran.
    if (!Wpre && tid < 32) warp_chol_solve_map<Real>(A, LDA, R, invd, Wx, ridge);
    __syncthreads();
    // Y = Yhat W (padding columns zero): a thread takes one row and four
    // columns, so each Yhat entry is read once per four outputs; every
    // output keeps its even-k / odd-k partial sums
    {
        const int groups = Rp >> 2;
        for (uint32_t w = tid; w < rows * (uint32_t)groups; w += nt) {
            const uint32_t i = w / groups;
            const int c0 = (int)(w - i * groups) * 4;
            const float* yh = Hs + (size_t)i * Rp;
            Real a0[4] = {0, 0, 0, 0}, a1[4] = {0, 0, 0, 0};
            int k = 0;
            for (; k + 2 <= R; k += 2) {
                const Real h0 = (Real)yh[k], h1 = (Real)yh[k + 1];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (c0 + q >= R) continue;
                    a0[q] += h0 * (Real)Wx[k * R + c0 + q];
                    a1[q] += h1 * (Real)Wx[(k + 1) * R + c0 + q];
                }
            }
            if (k < R) {
                const Real h0 = (Real)yh[k];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (c0 + q < R) a0[q] += h0 * (Real)Wx[k * R + c0 + q];
            }
            float* ys = Ys + (size_t)i * Rp + c0;
#pragma unroll
            for (int q = 0; q < 4; ++q) ys[q] = (c0 + q < R) ? (float)(a0[q] + a1[q]) : 0.f;
        }
    }
    __syncthreads();
    // Gram of Y in FP64 over the upper triangle (a <= b): thread = (pair,
    // row slice); the lower triangle is mirrored below
    {
        const int P = R * (R + 1) / 2;
        const int slices = max(1, nt / P);
        for (int t = tid; t < P * slices; t += nt) {
            const int pair = t % P, sl = t / P;
            int a = 0, rem = pair;
            while (rem >= R - a) { rem -= R - a; ++a; }
            const int b = a + rem;
            double acc = 0.0;
            for (uint32_t i = sl; i < rows; i += slices)
                acc += (double)Ys[(size_t)i * Rp + a] * (double)Ys[(size_t)i * Rp + b];
            atomicAdd(&G[a * R + b], acc);
        }
    }
    __syncthreads();
    // lambda from the diagonal; 1/lambda per column (FP32, for the scaling);
    // the Gram's lower triangle from its upper one
    float* invc = reinterpret_cast<float*>(invd);           // R (the solve is done)
    for (int r = tid; r < R; r += nt) {
        const double l = sqrt(max(G[r * R + r], 0.0));
        lam[r] = l;
        lam64[r] = l;
        lambda[r] = (float)l;
        invc[r] = l > 1e-20 ? (float)(1.0 / l) : 0.f;
    }
    for (int e = tid; e < RR; e += nt) {
        const int a = e / R, b = e % R;
        if (a > b) G[e] = G[b * R + a];
    }
    __syncthreads();
    for (int e = tid; e < RR; e += nt) {
        const double la = lam[e / R], lb = lam[e % R];
        const double ia = la > 1e-20 ? 1.0 / la : 0.0, ib = lb > 1e-20 ? 1.0 / lb : 0.0;
        const double g = G[e] * ia * ib;
        Gd[(size_t)n * RR + e] = g;
        G32[(size_t)n * RR + e] = (float)g;
    }
    for (uint32_t e = tid; e < total; e += nt) {
        const int c = (int)(e % Rp);
        Y[e] = c < R ? Ys[e] * invc[c] : 0.f;
    }
    if (last) {
        // <Y_c, Yhat_c> per column: thread = (column, row slice)
        const int slices = max(1, nt / R);
        for (int t = tid; t < R * slices; t += nt) {
            const int c = t % R, sl = t / R;
            double acc = 0.0;
            for (uint32_t i = sl; i < rows; i += slices) {
                const size_t e = (size_t)i * Rp + c;
                acc += (double)(Ys[e] * invc[c]) * (double)Hs[e];
            }
            atomicAdd(&dot[c], acc);
        }
    }
    __syncthreads();
    if (!last) return;
    // fit: <T,M> = sum_r lambda_r <Y_r, Yhat_r>, ||M||^2 from the Grams
    double s_in = 0.0, s_m = 0.0;
    for (int r = tid; r < R; r += nt) s_in += lam[r] * dot[r];
    for (int e = tid; e < RR; e += nt) {
        double h = 1.0;
        for (int m = 0; m < N; ++m) h *= Gd[(size_t)m * RR + e];
        s_m += lam[e / R] * lam[e % R] * h;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s_in += __shfl_xor_sync(0xffffffffu, s_in, o);
        s_m += __shfl_xor_sync(0xffffffffu, s_m, o);
    }
    const int lane = tid & 31, warp = tid >> 5;
    __shared__ double red2[32];
    if (lane == 0) { red[warp] = s_in; red2[warp] = s_m; }
    __syncthreads();
    if (tid == 0) {
        double inner = 0.0, m2 = 0.0;
        for (int w = 0; w < nt / 32; ++w) { inner += red[w]; m2 += red2[w]; }
        m2 = max(0.0, m2);
        double r2 = tnorm2 - 2.0 * inner + m2;
        if (r2 < 0.0) r2 = 0.0;
        const double resid = sqrt(r2);
        fitout[0] = inner;
        fitout[1] = m2;
        fitout[2] = 1.0 - resid / max(sqrt(tnorm2), 1e-30);
        fitout[3] = resid;
    }
}

// Device-side loop control of graph-replayed CP-ALS: records the iteration's
// fit and residual and keeps the WHILE condition set until the reference's
// stop rule (|fit_i - fit_{i-1}| < tol after the first iteration,
// src/dynasor_cpals.cpp:371-379) or max_iters ends the loop.
__global__ void k_loop_ctl(cudaGraphConditionalHandle h, const double* __restrict__ fitout,
                           double* __restrict__ st, double* __restrict__ fit_hist,
                           double* __restrict__ resid_hist, double tol, int max_iters)
{
    if (threadIdx.x != 0) return;
    const int it = (int)st[0];
    const double fit = fitout[2];
    fit_hist[it] = fit;
    resid_hist[it] = fitout[3];
    const bool stop = (it > 0 && fabs(fit - st[1]) < tol) || (it + 1 >= max_iters);
    st[1] = fit;
    st[0] = (double)(it + 1);
    cudaGraphSetConditional(h, stop ? 0u : 1u);
}

__global__ void k_sumsq(const float* __restrict__ v, uint64_t n, double* __restrict__ out) {
    __shared__ double red[256];
    double s = 0;
    // float4 loads, four in flight per thread (v is 16-byte aligned: a slab
    // column), then the scalar tail
    const float4* v4 = reinterpret_cast<const float4*>(v);
    const uint64_t n4 = n >> 2, stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += 4 * stride) {
        float4 x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            x[u] = q + u * stride < n4 ? __ldg(v4 + q + u * stride) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            s += (double)x[u].x * x[u].x + (double)x[u].y * x[u].y + (double)x[u].z * x[u].z +
                 (double)x[u].w * x[u].w;
    }
    for (uint64_t i = 4 * n4 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = v[i];
        s += x * x;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// ---------------------------------------------------------------------------
//  Scratch layout inside p.la_work (FP64):
//    Gd       N * R * R     Grams (FP64)
//    partial  kGramChunks * R * R
//    Wd       R * R
//    A        R * R         Cholesky work (FP64 or reinterpreted FP32)
//    lam64    R
//    dot      kGramChunks * R
//    fitout   4
//    misc     kGramChunks
// ---------------------------------------------------------------------------
struct LaLayout {
    double *Gd, *partial, *Wd, *A, *lam64, *dot, *fitout, *misc;
    float *G32, *W32;
};

int la_ensure(Plan& p, LaLayout& L) {
    const size_t R = p.R, RR = R * R;
    const size_t need = (size_t)p.N * RR + (size_t)kGramChunks * RR + 2 * RR + R +
                        (size_t)kGramChunks * R + 4 + kGramChunks + 64;
    if (need > p.la_work_cap) {
        dev_free(p.la_work);
        p.la_work = nullptr;
        DGPU_TRY(dev_alloc(p, (void**)&p.la_work, need * sizeof(double)));
        p.la_work_cap = need;
    }
    const size_t need32 = (size_t)p.N * RR + RR + 64;
    if (need32 > p.la_f32_cap) {
        dev_free(p.la_f32);
        p.la_f32 = nullptr;
        DGPU_TRY(dev_alloc(p, (void**)&p.la_f32, need32 * sizeof(float)));
        p.la_f32_cap = need32;
    }
    double* w = p.la_work;
    L.Gd = w;        w += (size_t)p.N * RR;
    L.partial = w;   w += (size_t)kGramChunks * RR;
    L.Wd = w;        w += RR;
    L.A = w;         w += RR;
    L.lam64 = w;     w += R;
    L.dot = w;       w += (size_t)kGramChunks * R;
    L.fitout = w;    w += 4;
    L.misc = w;
    L.G32 = p.la_f32;
    L.W32 = p.la_f32 + (size_t)p.N * RR;
    return DGPU_OK;
}

int gram_into(Plan& p, const LaLayout& L, int n, int normalise) {
    const int tiles = (p.R + kGramTile - 1) / kGramTile;
    const int chunks = (int)std::min<uint32_t>(kGramChunks, std::max<uint32_t>(1u, (p.dims[n] + 63) / 64));
    dim3 grid(chunks, tiles, tiles);
    DGPU_TRY(launch_gram_partial(grid, p.stream, p.Y[n], p.dims[n], p.R, p.Rp, L.partial));
    const size_t RR = (size_t)p.R * p.R;
    int fin_chunks = chunks;
    if (chunks > 8) {
        k_reduce_partials<<<(unsigned)((RR + 31) / 32), 256, 0, p.stream>>>(L.partial, chunks, (int)RR);
        fin_chunks = 1;
    }
    k_finalize_mode<<<1, 1024, 0, p.stream>>>(L.partial, fin_chunks, p.R, p.R, normalise,
                                              L.Gd + (size_t)n * RR, L.G32 + (size_t)n * RR,
                                              p.lambda, L.lam64);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

unsigned grid_for(size_t work, unsigned cap = 148 * 8) {
    return (unsigned)std::max<size_t>(1, std::min<size_t>((work + kLaThreads - 1) / kLaThreads, cap));
}

size_t small_update_smem(int R, int Rp, uint32_t rows, bool fp64) {
    const size_t RR = (size_t)R * R;
    return (2 * RR + 2 * (size_t)R) * sizeof(double) +
           (size_t)R * (R + 2) * (fp64 ? sizeof(double) : sizeof(float)) +
           2 * (size_t)rows * Rp * sizeof(float);
}

// One ALS factor update of mode n from Yhat[n] (cpals.cpp:290-321).  For the
// last mode *fit_done reports whether the fit was computed with it.
bool small_mode(const Plan& p, int n) {
    const uint64_t RR = (uint64_t)p.R * p.R;
    return p.R <= 64 && (uint64_t)p.dims[n] * p.Rp <= 8192 && (uint64_t)p.dims[n] * RR <= (1ull << 21);
}

// The solve map of small mode n into L.Wd on stream `st` (k_small_solve).
int launch_small_solve(Plan& p, const LaLayout& L, int n, int solve_fp64, double ridge,
                       cudaStream_t st) {
    const size_t RR = (size_t)p.R * p.R;
    const size_t sm = RR * sizeof(double) + (size_t)p.R * (p.R + 2) * (solve_fp64 ? 8 : 4);
    if (solve_fp64) {
        if (sm > 48 * 1024)
            DGPU_CUDA(cudaFuncSetAttribute(k_small_solve<double>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_small_solve<double><<<1, 32, sm, st>>>(L.Gd, p.N, n, p.R, ridge, L.Wd);
    } else {
        if (sm > 48 * 1024)
            DGPU_CUDA(cudaFuncSetAttribute(k_small_solve<float>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_small_solve<float><<<1, 32, sm, st>>>(L.Gd, p.N, n, p.R, ridge, L.Wd);
    }
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

// The large-mode solve map (FP64 Wd and its FP32 copy W32) on stream st.
int launch_large_solve(Plan& p, const LaLayout& L, int n, int solve_fp64, double ridge,
                       cudaStream_t st) {
    if (solve_fp64)
        k_build_solve_map<double><<<1, 1024, 0, st>>>(L.Gd, p.N, n, p.R, ridge, L.A, L.Wd, L.W32);
    else
        k_build_solve_map<float><<<1, 1024, 0, st>>>(L.Gd, p.N, n, p.R, ridge,
                                                      reinterpret_cast<float*>(L.A), L.Wd, L.W32);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

// Wpre != nullptr: the mode's solve map was already built (on the side
// stream, while its MTTKRP ran) into L.Wd / L.W32.
int update_mode(Plan& p, const LaLayout& L, int n, int solve_fp64, double ridge, bool last,
                double tn2, bool* fit_done, const double* Wpre = nullptr) {
    const size_t RR = (size_t)p.R * p.R;
    *fit_done = false;
    if (small_mode(p, n)) {
        const size_t sm = small_update_smem(p.R, p.Rp, p.dims[n], solve_fp64 != 0);
        if (solve_fp64) {
            if (sm > 48 * 1024)
                DGPU_CUDA(cudaFuncSetAttribute(k_update_small<double>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            k_update_small<double><<<1, kSmallThreads, sm, p.stream>>>(
                L.Gd, L.G32, p.N, n, p.R, p.Rp, ridge, p.Yhat[n], p.Y[n], p.dims[n], p.lambda,
                L.lam64, last ? 1 : 0, tn2, L.fitout, Wpre);
        } else {
            if (sm > 48 * 1024)
                DGPU_CUDA(cudaFuncSetAttribute(k_update_small<float>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            k_update_small<float><<<1, kSmallThreads, sm, p.stream>>>(
                L.Gd, L.G32, p.N, n, p.R, p.Rp, ridge, p.Yhat[n], p.Y[n], p.dims[n], p.lambda,
                L.lam64, last ? 1 : 0, tn2, L.fitout, Wpre);
        }
        DGPU_CUDA(cudaGetLastError());
        p.yb_stale[n] = true;
        *fit_done = last;
        return DGPU_OK;
    }
    if (!Wpre) DGPU_TRY(launch_large_solve(p, L, n, solve_fp64, ridge, p.stream));
    if (p.Rp == 16 || p.Rp == 32) {
        const unsigned gm = grid_for((size_t)p.dims[n] * p.Rp / 4);
        if (solve_fp64 && p.Rp == 16)
            k_apply_map_dmma<16><<<gm, kApplyThreads, 0, p.stream>>>(p.Yhat[n], p.dims[n], p.R, p.Rp,
                                                                     L.Wd, 0, nullptr, p.Y[n]);
        else if (solve_fp64)
            k_apply_map_dmma<32><<<gm, kApplyThreads, 0, p.stream>>>(p.Yhat[n], p.dims[n], p.R, p.Rp,
                                                                     L.Wd, 0, nullptr, p.Y[n]);
        else if (p.Rp == 16)
            k_apply_map_lanes<float, 16><<<gm, kLaThreads, 0, p.stream>>>(p.Yhat[n], p.dims[n], p.R, L.W32, p.Y[n]);
        else
            k_apply_map_lanes<float, 32><<<gm, kLaThreads, 0, p.stream>>>(p.Yhat[n], p.dims[n], p.R, L.W32, p.Y[n]);
    } else if (solve_fp64) {
        const size_t sm = RR * sizeof(double);
        if (sm > 48 * 1024)
            DGPU_CUDA(cudaFuncSetAttribute(k_apply_map<double>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_apply_map<double><<<grid_for((size_t)p.dims[n] * p.Rp), kLaThreads, sm, p.stream>>>(
            p.Yhat[n], p.dims[n], p.R, p.Rp, L.Wd, p.Y[n]);
    } else {
        const size_t sm = RR * sizeof(float);
        if (sm > 48 * 1024)
            DGPU_CUDA(cudaFuncSetAttribute(k_apply_map<float>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_apply_map<float><<<grid_for((size_t)p.dims[n] * p.Rp), kLaThreads, sm, p.stream>>>(
            p.Yhat[n], p.dims[n], p.R, p.Rp, L.W32, p.Y[n]);
    }
    DGPU_CUDA(cudaGetLastError());
    DGPU_TRY(gram_into(p, L, n, 1));
    const unsigned g = grid_for((size_t)p.dims[n] * p.Rp, kGramChunks);
    k_scale_cols<<<g, kLaThreads, (size_t)p.R * (sizeof(double) + sizeof(float)), p.stream>>>(
        p.Y[n], last ? p.Yhat[n] : nullptr, p.dims[n], p.R, p.Rp, L.lam64, L.dot);
    DGPU_CUDA(cudaGetLastError());
    p.yb_stale[n] = true;
    return DGPU_OK;
}

// N(0,1) initial factors exactly as the reference draws them
// (src/dynasor_cpals.cpp:42-69): a splitmix64 step of (seed, n) seeds a
// std::mt19937_64, entries from std::normal_distribution<float>(0, 1),
// row-major, padding zero.  Generated on the host, uploaded once.
// skip_mode >= 0: that mode's factor is zeroed instead of drawn.  Each mode
// has its own generator, so the other modes' draws are unchanged;
// Gauss-Seidel never reads mode 0's initial factor (mode 0 is solved first,
// from the other modes' Grams, and its Gram is recomputed from the result),
// so a Gauss-Seidel run skips the draw of mode 0 -- on the 1M-row rank-32
// factor, 32M normal draws.
// One mode's factor (rows x Rp, row-major, padding zero) into host memory.
void draw_factor(uint64_t seed, int n, uint32_t rows, int R, int Rp, float* y) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (uint64_t)(n + 1);
    z ^= z >> 30; z *= 0xBF58476D1CE4E5B9ULL;
    z ^= z >> 27; z *= 0x94D049BB133111EBULL;
    z ^= z >> 31;
    std::mt19937_64 rng(z);
    std::normal_distribution<float> g(0.0f, 1.0f);
    for (uint32_t i = 0; i < rows; ++i) {
        for (int r = 0; r < R; ++r) y[(size_t)i * Rp + r] = g(rng);
        for (int r = R; r < Rp; ++r) y[(size_t)i * Rp + r] = 0.f;
    }
}

int init_factors_host(Plan& p, uint64_t seed, int skip_mode) {
    // one independent generator per mode: draw the modes on parallel host
    // threads (large factors take seconds to draw serially)
    std::vector<std::vector<float>> Y(p.N);
    std::vector<std::thread> th;
    size_t total = 0;
    for (int n = 0; n < p.N; ++n) total += n == skip_mode ? 0 : (size_t)p.dims[n] * p.R;
    const bool par = total >= (1u << 20);       // small factors: no thread start-up
    for (int n = 0; n < p.N; ++n) {
        if (n == skip_mode) continue;
        auto draw = [&, n]() {
            Y[n].assign((size_t)p.dims[n] * p.Rp, 0.f);
            draw_factor(seed, n, p.dims[n], p.R, p.Rp, Y[n].data());
        };
        if (par) th.emplace_back(draw);
        else draw();
    }
    for (auto& t : th) t.join();
    for (int n = 0; n < p.N; ++n) {
        if (n == skip_mode)
            DGPU_CUDA(cudaMemsetAsync(p.Y[n], 0, (size_t)p.dims[n] * p.Rp * sizeof(float), p.stream));
        else
            DGPU_CUDA(cudaMemcpyAsync(p.Y[n], Y[n].data(), Y[n].size() * sizeof(float),
                                      cudaMemcpyHostToDevice, p.stream));
        p.yb_stale[n] = true;
    }
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    return DGPU_OK;
}

}  // namespace

int cp_tensor_norm(Plan& p, const float* vals, double* out) {
    const unsigned blocks = 296;
    double* tmp = nullptr;
    DGPU_TRY(dev_alloc(p, (void**)&tmp, blocks * sizeof(double)));
    k_sumsq<<<blocks, 256, 0, p.stream>>>(vals, p.nnz, tmp);
    std::vector<double> h(blocks);
    DGPU_CUDA(cudaMemcpyAsync(h.data(), tmp, blocks * sizeof(double), cudaMemcpyDeviceToHost, p.stream));
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    dev_free(tmp);
    p.device_bytes -= blocks * sizeof(double);
    double s = 0;
    for (double x : h) s += x;
    *out = s;
    return DGPU_OK;
}

// One CP-ALS run on a plan, in phases so that several runs can share one
// graph launch (cpals_batch_run).  Iteration 0 runs eagerly (it allocates,
// times the MTTKRP / update split and fixes tuned kernel choices); later
// iterations run either as a device-side WHILE loop captured into a graph
// (when an iteration leaves the live slab where it found it) or from the
// host, replaying per-iteration graphs.
struct CpSession {
    using clk = std::chrono::steady_clock;
    Plan& p;
    dgpu_cp_options o;
    dgpu_cp_result& res;
    double* fit_history;
    LaLayout L{};
    double tn2 = 0.0;
    bool jacobi = false;
    // kept on the plan across calls (created on first use)
    std::vector<cudaEvent_t>& ev;            // iteration timing
    std::vector<cudaEvent_t>& fork;          // side-stream solve of each mode
    std::vector<cudaEvent_t>& join;
    double*& fit_host;                       // pinned: the per-iteration graphs' D2H target
    double*& st;                             // device loop: [it, fit_prev] + fit/residual histories
    size_t& st_bytes;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int cur_after[2] = {0, 0};
    double fit_prev = 0.0;
    int cur_start = 0;
    int it = 0;                              // next iteration index
    bool done = false;
    bool graphs = false;
    clk::time_point t_start;
    clk::time_point t_it;                    // start of the iteration in flight
    // host plan state saved around a capture (a capture advances it without
    // running the work)
    int cur0 = 0, nm0 = 0;
    uint64_t pp0 = 0;
    bool stale0[kMaxModes] = {};
    // iterations run eagerly before any capture: 2 when the first one left
    // PingPong partition passes without kept tables (the slab's first
    // cycle), so that the captured iterations use the kept tables
    int warm_iters = 1;
    bool self_map = true;                    // one iteration leaves the live slab in place

    CpSession(Plan& pl, const dgpu_cp_options& op, dgpu_cp_result& r, double* fh)
        : p(pl), o(op), res(r), fit_history(fh), ev(pl.cp_ev), fork(pl.cp_fork), join(pl.cp_join),
          fit_host(pl.cp_fit_host), st(pl.cp_st), st_bytes(pl.cp_st_bytes) {}
    ~CpSession() {
        for (int k = 0; k < 2; ++k) if (exec[k]) cudaGraphExecDestroy(exec[k]);
    }

    static int ensure_events(std::vector<cudaEvent_t>& v, size_t n, unsigned flags) {
        if (v.size() == n) return DGPU_OK;
        for (auto e : v) if (e) cudaEventDestroy(e);
        v.assign(n, nullptr);
        for (auto& e : v) DGPU_CUDA(cudaEventCreateWithFlags(&e, flags));
        return DGPU_OK;
    }

    int setup() {
        res = dgpu_cp_result{};
        DGPU_TRY(la_ensure(p, L));
        const bool gs = o.kernel != DGPU_CP_JACOBI && p.layout != DGPU_LAYOUT_MORTON;
        if (!o.use_init) DGPU_TRY(init_factors_host(p, o.seed, gs && o.max_iters > 0 ? 0 : -1));
        for (int n = 0; n < p.N; ++n) DGPU_TRY(gram_into(p, L, n, 0));
        // ||T||^2 of the plan's values, computed once per plan
        if (p.cp_tnorm2 < 0.0) DGPU_TRY(cp_tensor_norm(p, live_vals(p), &p.cp_tnorm2));
        tn2 = p.cp_tnorm2;
        res.tensor_norm = std::sqrt(tn2);
        if (o.verbose)
            std::printf("[cpals] modes=%d  rank=%d  padded=%d  nnz=%llu  ||T|| = %.6e  max_iters=%d  "
                        "tol=%.1e  seed=%llu\n", p.N, p.R, p.Rp, (unsigned long long)p.nnz,
                        res.tensor_norm, o.max_iters, o.tol, (unsigned long long)o.seed);
        // the Morton layout has only the all-modes pass: Gauss-Seidel runs
        // as Jacobi there, as the reference does (src/dynasor_cpals.cpp:232-240)
        jacobi = (o.kernel == DGPU_CP_JACOBI) || p.layout == DGPU_LAYOUT_MORTON;
        if (p.layout == DGPU_LAYOUT_MORTON && o.kernel != DGPU_CP_JACOBI && o.verbose)
            std::printf("[cpals] WARN: Morton layout has no Gauss-Seidel driver; running Jacobi\n");
        // ev[0] iteration start, ev[1 + 2n] end of mode n's MTTKRP (Jacobi:
        // ev[1] ends all MTTKRPs), ev[2 + 2n] end of mode n's factor update
        DGPU_TRY(ensure_events(ev, 2 * (size_t)p.N + 2, cudaEventDefault));
        DGPU_TRY(ensure_events(fork, p.N, cudaEventDisableTiming));
        DGPU_TRY(ensure_events(join, p.N, cudaEventDisableTiming));
        if (!p.side_stream)
            DGPU_CUDA(cudaStreamCreateWithFlags(&p.side_stream, cudaStreamNonBlocking));
        if (!fit_host) DGPU_CUDA(cudaMallocHost((void**)&fit_host, 4 * sizeof(double)));
        graphs = o.graphs != 0 && !p.timing;
        cur_start = p.cur;
        done = o.max_iters <= 0;
        t_start = clk::now();
        return DGPU_OK;
    }

    void save_state() {
        cur0 = p.cur;
        nm0 = p.next_mode;
        pp0 = p.pp_transitions;
        for (int n = 0; n < kMaxModes; ++n) stale0[n] = p.yb_stale[n];
    }
    void restore_state() {
        p.cur = cur0;
        p.next_mode = nm0;
        p.pp_transitions = pp0;
        for (int n = 0; n < kMaxModes; ++n) p.yb_stale[n] = stale0[n];
    }

    // One iteration's work on p.stream.  kind 0: eager; 1: captured for
    // per-iteration replay (event records become graph event nodes); 2: the
    // body of the device-side loop (no events, no host copy; the loop
    // control kernel follows).
    int enqueue(int kind) {
        auto rec = [&](int i) -> cudaError_t {
            if (kind == 2) return cudaSuccess;
            return kind == 1 ? cudaEventRecordWithFlags(ev[i], p.stream, cudaEventRecordExternal)
                             : cudaEventRecord(ev[i], p.stream);
        };
        DGPU_CUDA(rec(0));
        bool fit_done = false;
        // Jacobi: every MTTKRP from the iteration's starting factors
        // (src/dynasor_cpals.cpp:270-278).  The N mode passes on the FLYCOO
        // layout accumulate each output row in registers; the all-modes
        // kernel (dgpu_mttkrp_all_modes) computes the same outputs in one slab
        // pass but with a vector atomic per nonzero and mode, which on the
        // 4-mode, 200M-nonzero, rank-64 tensor ran at 3.9 iterations/s against
        // 18.6 for the mode passes.
        if (jacobi && p.layout == DGPU_LAYOUT_MORTON)
            DGPU_TRY(launch_mttkrp_all_modes(p));
        else if (jacobi)
            for (int n = 0; n < p.N; ++n)
                DGPU_TRY(p.layout == DGPU_LAYOUT_NCOPY ? mode_ncopy(p, n) : mode_pingpong(p, n));
        for (int n = 0; n < p.N; ++n) {
            // Gauss-Seidel: a mode's solve map depends only on the other
            // modes' Grams, so it is built on the side stream while this
            // mode's MTTKRP runs (fork after the previous update, join
            // before this one)
            const bool ovl = !jacobi;
            if (ovl) {
                // the previous update may still run on the PingPong overlap
                // stream: fork from there
                const cudaStream_t from = p.ovl_pending ? p.ovl_stream : p.stream;
                DGPU_CUDA(cudaEventRecord(fork[n], from));
                DGPU_CUDA(cudaStreamWaitEvent(p.side_stream, fork[n], 0));
                if (small_mode(p, n))
                    DGPU_TRY(launch_small_solve(p, L, n, o.solve_fp64, o.ridge, p.side_stream));
                else
                    DGPU_TRY(launch_large_solve(p, L, n, o.solve_fp64, o.ridge, p.side_stream));
                DGPU_CUDA(cudaEventRecord(join[n], p.side_stream));
            }
            // the factor update (on the stream that ran the MTTKRP)
            auto update = [&]() -> int {
                DGPU_CUDA(rec(1 + 2 * n));
                if (ovl) DGPU_CUDA(cudaStreamWaitEvent(p.stream, join[n], 0));
                DGPU_TRY(update_mode(p, L, n, o.solve_fp64, o.ridge, n == p.N - 1, tn2, &fit_done,
                                     ovl ? L.Wd : nullptr));
                DGPU_CUDA(rec(2 + 2 * n));
                return DGPU_OK;
            };
            if (jacobi) {
                DGPU_TRY(update());
            } else if (p.layout == DGPU_LAYOUT_NCOPY) {
                DGPU_TRY(mode_ncopy(p, n));
                DGPU_TRY(update());
            } else {
                // PingPong: the update needs this mode's Yhat, not the
                // remapped slab, so it runs beside the remap and the next
                // mode's fiber sort
                DGPU_TRY(mode_pingpong_then(p, n, update));
            }
        }
        DGPU_TRY(pingpong_drain(p));
        if (!fit_done) {
            const int nblk = (int)grid_for((size_t)p.dims[p.N - 1] * p.Rp, kGramChunks);
            k_fit<<<1, 1024, 0, p.stream>>>(L.Gd, p.N, p.R, L.lam64, L.dot, nblk, tn2, L.fitout);
            DGPU_CUDA(cudaGetLastError());
        }
        if (kind != 2)
            DGPU_CUDA(cudaMemcpyAsync(fit_host, L.fitout, 4 * sizeof(double),
                                      cudaMemcpyDeviceToHost, p.stream));
        return DGPU_OK;
    }

    // One host-driven iteration: eager, or (after the first) a replay of the
    // per-iteration graph keyed by the live slab (PingPong alternates slabs,
    // so at most two graphs), then the fit bookkeeping and the stop rule.
    int step_host() {
        DGPU_TRY(launch_iteration());
        return collect_iteration();
    }

    // The iteration's work on p.stream, not waited for (a batch launches the
    // first iterations of all its plans before it collects any).
    int launch_iteration() {
        t_it = clk::now();
        const int key = (p.layout == DGPU_LAYOUT_NCOPY) ? 0 : (p.cur & 1);
        if (graphs && it >= warm_iters && exec[key]) {
            DGPU_CUDA(cudaGraphLaunch(exec[key], p.stream));
            p.cur = cur_after[key];
            p.next_mode = 0;
        } else if (graphs && it >= warm_iters) {
            save_state();
            cudaGraph_t g = nullptr;
            cudaError_t ec = cudaStreamBeginCapture(p.stream, cudaStreamCaptureModeRelaxed);
            int rc = DGPU_OK;
            if (ec == cudaSuccess) {
                rc = enqueue(1);
                ec = cudaStreamEndCapture(p.stream, &g);
            }
            cudaError_t ei = cudaErrorUnknown;
            if (rc == DGPU_OK && ec == cudaSuccess && g)
                ei = cudaGraphInstantiate(&exec[key], g, 0);
            if (g) cudaGraphDestroy(g);
            if (rc == DGPU_OK && ec == cudaSuccess && ei == cudaSuccess) {
                cur_after[key] = p.cur;
                DGPU_CUDA(cudaGraphLaunch(exec[key], p.stream));
            } else {
                // this stream cannot be captured (e.g. the legacy default
                // stream): iterate eagerly from here on
                cudaGetLastError();
                exec[key] = nullptr;
                graphs = false;
                restore_state();
                DGPU_TRY(enqueue(0));
            }
        } else {
            DGPU_TRY(enqueue(0));
        }
        return DGPU_OK;
    }

    // Waits for the launched iteration; fit bookkeeping and the stop rule.
    int collect_iteration() {
        DGPU_CUDA(cudaStreamSynchronize(p.stream));
        float mt_ms = 0.f, la_ms = 0.f;
        for (int n = 0; n < p.N; ++n) {
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, ev[n == 0 ? 0 : 2 * n], ev[1 + 2 * n]);
            cudaEventElapsedTime(&b, ev[1 + 2 * n], ev[2 + 2 * n]);
            mt_ms += a;
            la_ms += b;
        }
        const double fit = fit_host[2];
        res.mttkrp_time_s += mt_ms * 1e-3;
        res.linalg_time_s += la_ms * 1e-3;
        if (fit_history) fit_history[it] = fit;
        res.final_fit = fit;
        res.final_residual = fit_host[3];
        res.iters_done = it + 1;
        const double iter_s = std::chrono::duration<double>(clk::now() - t_it).count();
        if (o.verbose)
            std::printf("[cpals] iter %3d  fit = %.6f  dfit = %.2e  resid = %.3e  iter = %.3f s\n",
                        it, fit, it == 0 ? 0.0 : std::fabs(fit - fit_prev), fit_host[3], iter_s);
        if (it > 0 && std::fabs(fit - fit_prev) < o.tol) {
            if (o.verbose)
                std::printf("[cpals] converged after %d iterations (|dfit|=%.2e < %.1e)\n", it + 1,
                            std::fabs(fit - fit_prev), o.tol);
            done = true;
        }
        fit_prev = fit;
        ++it;
        if (it >= o.max_iters) done = true;
        return DGPU_OK;
    }

    // The remaining iterations can run as a device-side loop.
    bool loop_eligible() const {
        return graphs && !done && it == warm_iters && !o.verbose && self_map &&
               (p.layout == DGPU_LAYOUT_NCOPY || p.cur == cur_start);
    }

    // Captures one iteration + the loop control into `body` (the WHILE
    // node's graph).  DGPU_ERR_CUDA: capture not possible (state restored).
    // The loop state array (reallocated only to grow; a cached loop graph
    // that read the old one is dropped).
    int ensure_state() {
        const size_t need = (2 + 2 * (size_t)o.max_iters) * sizeof(double);
        if (st_bytes >= need) return DGPU_OK;
        if (p.cp_loop_exec) {
            cudaGraphExecDestroy(p.cp_loop_exec);
            p.cp_loop_exec = nullptr;
        }
        if (st) {
            dev_free(st);
            p.device_bytes -= st_bytes;
            st = nullptr;
            st_bytes = 0;
        }
        DGPU_TRY(dev_alloc(p, (void**)&st, need));
        st_bytes = need;
        return DGPU_OK;
    }
    // BF16 mirrors of every factor changed since its last conversion.  A
    // loop graph converts, per mode, the mirrors that were stale when it was
    // captured (the steady state of the capturing run: the factors updated
    // since the previous mode), so a graph kept from an earlier run assumes
    // the other mirrors current.  Fresh initial factors leave them stale:
    // convert them before such a graph runs.
    int refresh_mirrors() {
        if (p.precision != DGPU_PREC_BF16) return DGPU_OK;
        for (int n = 0; n < p.N; ++n)
            if (p.yb_stale[n]) DGPU_TRY(launch_to_bf16(p, n));
        return DGPU_OK;
    }
    int write_state() {
        const double init[2] = {(double)it, fit_prev};
        DGPU_CUDA(cudaMemcpyAsync(st, init, sizeof(init), cudaMemcpyHostToDevice, p.stream));
        DGPU_CUDA(cudaStreamSynchronize(p.stream));
        return DGPU_OK;
    }

    // What the captured loop body depends on: options, tensor norm, live
    // slab at the loop start and the device buffers it reads and writes.
    void loop_key(uint64_t (&k)[kLoopKeyWords]) const {
        auto bits = [](double v) { uint64_t u; std::memcpy(&u, &v, 8); return u; };
        k[0] = (uint64_t)o.kernel;
        k[1] = (uint64_t)o.solve_fp64;
        k[2] = bits(o.ridge);
        k[3] = bits(o.tol);
        k[4] = (uint64_t)o.max_iters;
        k[5] = bits(tn2);
        k[6] = (uint64_t)cur_start | ((uint64_t)p.layout << 8) | ((uint64_t)p.precision << 16);
        k[7] = (uint64_t)(uintptr_t)p.la_work;
        k[8] = (uint64_t)(uintptr_t)p.la_f32;
        k[9] = (uint64_t)(uintptr_t)st;
        k[10] = (uint64_t)(uintptr_t)p.lambda;
        k[11] = (uint64_t)(uintptr_t)p.Y[0];
        k[12] = p.tables_gen;                  // partition lists and launch knobs
    }

    int capture_body(cudaGraph_t body, cudaGraphConditionalHandle h) {
        DGPU_TRY(ensure_state());
        DGPU_TRY(write_state());
        save_state();
        if (cudaStreamBeginCaptureToGraph(p.stream, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed) != cudaSuccess) {
            cudaGetLastError();
            set_error("cpals: device loop capture not available; iterating from the host");
            return DGPU_ERR_CUDA;
        }
        int rc = enqueue(2);
        if (rc == DGPU_OK) {
            k_loop_ctl<<<1, 32, 0, p.stream>>>(h, L.fitout, st, st + 2, st + 2 + o.max_iters,
                                               o.tol, o.max_iters);
            if (cudaGetLastError() != cudaSuccess) rc = DGPU_ERR_CUDA;
        }
        cudaGraph_t cap = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(p.stream, &cap);
        if (rc != DGPU_OK || ec != cudaSuccess) {
            cudaGetLastError();
            restore_state();
            if (rc != DGPU_OK && rc != DGPU_ERR_CUDA) return rc;
            set_error("cpals: device loop graph not available; iterating from the host");
            return DGPU_ERR_CUDA;
        }
        return DGPU_OK;
    }

    // After the loop graph ran: iterations, fits and the time split (the
    // loop's device time `ms`, divided between MTTKRP and the factor updates
    // in the proportion measured on the eager first iteration).
    int finish_loop(float ms) {
        std::vector<double> hs(2 + 2 * (size_t)o.max_iters);
        DGPU_CUDA(cudaMemcpy(hs.data(), st, hs.size() * sizeof(double), cudaMemcpyDeviceToHost));
        const int last = (int)hs[0];
        const double tot = res.mttkrp_time_s + res.linalg_time_s;
        // split of the loop's device time: this run's eager iteration, else
        // the last measured one on this plan
        const double fm = tot > 0 ? res.mttkrp_time_s / tot : p.cp_mttkrp_frac;
        if (tot > 0) p.cp_mttkrp_frac = fm;
        res.mttkrp_time_s += fm * ms * 1e-3;
        res.linalg_time_s += (1.0 - fm) * ms * 1e-3;
        for (int i = it; i < last; ++i) {
            if (fit_history) fit_history[i] = hs[2 + i];
            res.final_fit = hs[2 + i];
            res.final_residual = hs[2 + o.max_iters + i];
        }
        res.iters_done = last;
        it = last;
        done = true;
        return DGPU_OK;
    }

    void finish() {
        res.total_time_s = std::chrono::duration<double>(clk::now() - t_start).count();
        if (o.verbose)
            std::printf("[cpals] done  iters=%d  final_fit=%.6f  resid=%.3e\n"
                        "[cpals] total = %.3f s   spMTTKRP = %.3f s (%.1f%%)   linalg  = %.3f s (%.1f%%)\n",
                        res.iters_done, res.final_fit, res.final_residual, res.total_time_s,
                        res.mttkrp_time_s, 100.0 * res.mttkrp_time_s / std::max(res.total_time_s, 1e-30),
                        res.linalg_time_s, 100.0 * res.linalg_time_s / std::max(res.total_time_s, 1e-30));
    }
};

// Key of a batch's loop graph: the plans (by serial, never reused) and each
// session's loop key, in batch order.
std::vector<uint64_t> batch_key(const std::vector<CpSession*>& ss) {
    std::vector<uint64_t> key{(uint64_t)ss.size()};
    for (CpSession* s : ss) {
        uint64_t k[kLoopKeyWords];
        s->loop_key(k);
        key.push_back(s->p.serial);
        key.insert(key.end(), k, k + kLoopKeyWords);
    }
    return key;
}

// Launches `gx` on `launch` and hands every session its share of the loop.
int launch_loops(std::vector<CpSession*>& in, cudaGraphExec_t gx, cudaStream_t launch) {
    cudaEvent_t a, b;
    DGPU_CUDA(cudaEventCreate(&a));
    DGPU_CUDA(cudaEventCreate(&b));
    struct E { cudaEvent_t a, b; ~E() { cudaEventDestroy(a); cudaEventDestroy(b); } } eg{a, b};
    DGPU_CUDA(cudaEventRecord(a, launch));
    DGPU_CUDA(cudaGraphLaunch(gx, launch));
    DGPU_CUDA(cudaEventRecord(b, launch));
    DGPU_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    for (CpSession* s : in) DGPU_TRY(s->finish_loop(ms));
    return DGPU_OK;
}

// Runs the device loops of `ss` (all eligible) as parallel WHILE nodes of one
// graph, launched once on `owner`'s stream.  Sessions whose capture is not
// possible are left to iterate from the host.  When every session is in the
// graph it is kept on `owner` with the batch key, for a later call on the
// same plans (cpals_batch_run).
int run_loops(std::vector<CpSession*>& ss, Plan& owner) {
    cudaGraph_t outer = nullptr;
    cudaGraphExec_t gx = nullptr;
    struct G { cudaGraph_t& g; cudaGraphExec_t& x;
               ~G() { if (x) cudaGraphExecDestroy(x); if (g) cudaGraphDestroy(g); } } gg{outer, gx};
    DGPU_CUDA(cudaGraphCreate(&outer, 0));
    std::vector<CpSession*> in;
    for (CpSession* s : ss) {
        cudaGraphConditionalHandle h;
        DGPU_CUDA(cudaGraphConditionalHandleCreate(&h, outer, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        DGPU_CUDA(cudaGraphAddNode(&node, outer, nullptr, 0, &np));
        const int rc = s->capture_body(np.conditional.phGraph_out[0], h);
        if (rc == DGPU_OK) { in.push_back(s); continue; }
        if (rc != DGPU_ERR_CUDA) return rc;
        s->graphs = false;                       // iterate this one from the host
        DGPU_CUDA(cudaGraphDestroyNode(node));
    }
    if (in.empty()) return DGPU_OK;
    if (cudaGraphInstantiate(&gx, outer, 0) != cudaSuccess) {
        cudaGetLastError();
        for (CpSession* s : in) { s->restore_state(); s->graphs = false; }
        return DGPU_OK;
    }
    if (in.size() == ss.size()) {
        if (owner.cp_batch_exec) cudaGraphExecDestroy(owner.cp_batch_exec);
        owner.cp_batch_exec = gx;
        owner.cp_batch_key = batch_key(in);
        gx = nullptr;                            // kept: not destroyed with the guard
        return launch_loops(in, owner.cp_batch_exec, owner.stream);
    }
    return launch_loops(in, gx, owner.stream);
}

// The device loop of one run, with its executable graph kept on the plan:
// a later run with the same loop key relaunches it (after writing the loop
// state) instead of capturing and instantiating it again.
int run_loop_cached(CpSession& s) {
    Plan& p = s.p;
    uint64_t key[kLoopKeyWords];
    DGPU_TRY(s.ensure_state());
    s.loop_key(key);
    if (!p.cp_loop_exec || std::memcmp(key, p.cp_loop_key, sizeof(key)) != 0) {
        if (p.cp_loop_exec) {
            cudaGraphExecDestroy(p.cp_loop_exec);
            p.cp_loop_exec = nullptr;
        }
        cudaGraph_t outer = nullptr;
        DGPU_CUDA(cudaGraphCreate(&outer, 0));
        struct G { cudaGraph_t g; ~G() { if (g) cudaGraphDestroy(g); } } gg{outer};
        cudaGraphConditionalHandle h;
        DGPU_CUDA(cudaGraphConditionalHandleCreate(&h, outer, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        DGPU_CUDA(cudaGraphAddNode(&node, outer, nullptr, 0, &np));
        const int rc = s.capture_body(np.conditional.phGraph_out[0], h);
        if (rc == DGPU_ERR_CUDA) {
            s.graphs = false;                    // iterate from the host
            return DGPU_OK;
        }
        DGPU_TRY(rc);
        if (cudaGraphInstantiate(&p.cp_loop_exec, outer, 0) != cudaSuccess) {
            cudaGetLastError();
            p.cp_loop_exec = nullptr;
            s.restore_state();
            s.graphs = false;
            return DGPU_OK;
        }
        std::memcpy(p.cp_loop_key, key, sizeof(key));
    } else {
        DGPU_TRY(s.refresh_mirrors());
        DGPU_TRY(s.write_state());
    }
    DGPU_CUDA(cudaEventRecord(s.ev[0], p.stream));
    DGPU_CUDA(cudaGraphLaunch(p.cp_loop_exec, p.stream));
    DGPU_CUDA(cudaEventRecord(s.ev[1], p.stream));
    DGPU_CUDA(cudaEventSynchronize(s.ev[1]));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s.ev[0], s.ev[1]);
    return s.finish_loop(ms);
}

int cpals_run(Plan& p, const dgpu_cp_options& o, dgpu_cp_result& res, double* fit_history) {
    CpSession s(p, o, res, fit_history);
    DGPU_TRY(s.setup());
    // A plan whose device-loop graph was captured for this run's key runs
    // every iteration, the first included, in that loop: the eager first
    // iteration's work (allocation, tuning, timing split) was done by the
    // run that captured it.
    bool replayed = false;
    if (s.graphs && !o.verbose && !s.done && p.cp_loop_exec) {
        DGPU_TRY(s.ensure_state());
        uint64_t key[kLoopKeyWords];
        s.loop_key(key);
        if (std::memcmp(key, p.cp_loop_key, sizeof(key)) == 0) {
            DGPU_TRY(run_loop_cached(s));
            replayed = true;
        }
    }
    if (!replayed && !s.done) {
        const uint64_t unc0 = p.pc_uncached;
        DGPU_TRY(s.step_host());
        s.self_map = p.layout == DGPU_LAYOUT_NCOPY || p.cur == s.cur_start;
        if (s.graphs && p.pc_uncached != unc0 && !s.done) {
            s.warm_iters = 2;
            DGPU_TRY(s.step_host());
        }
    }
    if (!replayed && s.loop_eligible()) DGPU_TRY(run_loop_cached(s));
    while (!s.done) DGPU_TRY(s.step_host());
    s.finish();
    return DGPU_OK;
}

// Independent CP-ALS runs on several plans (one per tensor).
//   * The set-up of every run (initial factors drawn on the host, Grams,
//     ||T||^2) runs on parallel host threads, one plan each.
//   * A batch whose loop graph is kept on plans[0] for these plans and
//     options runs every iteration, the first included, in one launch of
//     that graph (the eager first iteration's allocations and tuning were
//     done by the call that captured it).
//   * Otherwise every plan's first iteration is launched on its own stream
//     before any is waited for, then the remaining iterations run as
//     parallel device loops of one graph launch, and that graph is kept.
int cpals_batch_run(Plan* const* plans, int count, const dgpu_cp_options& o,
                    dgpu_cp_result* res, double* fit_history) {
    std::vector<std::unique_ptr<CpSession>> ss;
    for (int k = 0; k < count; ++k)
        ss.emplace_back(new CpSession(*plans[k], o, res[k],
                                      fit_history ? fit_history + (size_t)k * std::max(1, o.max_iters)
                                                  : nullptr));
    {
        std::vector<int> rc(count, DGPU_OK);
        std::vector<std::string> msg(count);
        std::atomic<int> next{0};
        const int nth = std::max(1, std::min<int>(count, (int)std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (int t = 0; t < nth; ++t)
            th.emplace_back([&]() {
                for (int k = next++; k < count; k = next++) {
                    if (cudaSetDevice(plans[k]->device) != cudaSuccess) {
                        rc[k] = DGPU_ERR_CUDA;
                        msg[k] = "cudaSetDevice failed";
                        continue;
                    }
                    rc[k] = ss[k]->setup();
                    if (rc[k] != DGPU_OK) msg[k] = last_error();
                }
            });
        for (auto& t : th) t.join();
        DGPU_CUDA(cudaSetDevice(plans[0]->device));
        for (int k = 0; k < count; ++k)
            if (rc[k] != DGPU_OK) {
                set_error("cpals batch, plan %d: %s", k, msg[k].c_str());
                return rc[k];
            }
    }
    std::vector<CpSession*> all;
    for (auto& s : ss) all.push_back(s.get());
    Plan& owner = *plans[0];
    bool cached = owner.cp_batch_exec != nullptr && !o.verbose;
    for (CpSession* s : all) cached = cached && s->graphs && !s->done;
    if (cached) {
        for (CpSession* s : all) DGPU_TRY(s->ensure_state());
        cached = owner.cp_batch_exec != nullptr && batch_key(all) == owner.cp_batch_key;
    }
    if (cached) {
        for (CpSession* s : all) {
            DGPU_TRY(s->refresh_mirrors());
            DGPU_TRY(s->write_state());
        }
        DGPU_TRY(launch_loops(all, owner.cp_batch_exec, owner.stream));
    } else {
        for (CpSession* s : all)
            if (!s->done) DGPU_TRY(s->launch_iteration());
        for (CpSession* s : all)
            if (!s->done) DGPU_TRY(s->collect_iteration());
        std::vector<CpSession*> loop;
        for (CpSession* s : all)
            if (s->loop_eligible()) loop.push_back(s);
        if (!loop.empty()) DGPU_TRY(run_loops(loop, owner));
    }
    for (CpSession* s : all) {
        while (!s->done) DGPU_TRY(s->step_host());
        s->finish();
    }
    return DGPU_OK;
}

// ---------------------------------------------------------------------------
//  CP-OPT adjoint.  For the dense CP model M = [[Y_0, ..., Y_{N-1}]] and
//  f = 0.5 * ||X - M||_F^2 (zeros outside the nonzeros), the gradient is
//      df/dY_n = Y_n * H_n - MTTKRP_n(X),   H_n = Hadamard_{m != n} Y_m^T Y_m.
//  MTTKRP_n comes from one all-modes pass (same factor snapshot for every
//  mode); nothing per nonzero is stored between the passes.
// ---------------------------------------------------------------------------
namespace {

__global__ void k_hadamard_others(const double* __restrict__ Gd, int N, int n, int R,
                                  double* __restrict__ H)
{
    const size_t RR = (size_t)R * R;
    for (size_t e = threadIdx.x + (size_t)blockIdx.x * blockDim.x; e < RR;
         e += (size_t)gridDim.x * blockDim.x) {
        double v = 1.0;
        for (int m = 0; m < N; ++m)
            if (m != n) v *= Gd[(size_t)m * RR + e];
        H[e] = v;
    }
}

// grad[i][c] = sum_k Y[i][k] H[k][c] - Yhat[i][c]
__global__ void __launch_bounds__(kLaThreads)
k_grad_rows(const float* __restrict__ Y, const float* __restrict__ Yhat, uint32_t rows, int R,
            int Rp, const double* __restrict__ H, float* __restrict__ grad)
{
    extern __shared__ unsigned char smem_raw[];
    double* Hs = reinterpret_cast<double*>(smem_raw);
    for (int e = threadIdx.x; e < R * R; e += blockDim.x) Hs[e] = H[e];
    __syncthreads();
    const size_t total = (size_t)rows * Rp;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t i = e / Rp;
        const int c = (int)(e - i * Rp);
        if (c >= R) { grad[e] = 0.f; continue; }
        const float* y = Y + i * Rp;
        double s = 0;
        for (int k = 0; k < R; ++k) s += (double)__ldg(y + k) * Hs[(size_t)k * R + c];
        grad[e] = (float)(s - (double)Yhat[e]);
    }
}

}  // namespace

int cpopt_gradient(Plan& p, float* const* grad_host) {
    LaLayout L{};
    DGPU_TRY(la_ensure(p, L));
    // MTTKRP_n for every n from one factor snapshot.  The mode passes keep
    // each output row in registers; the all-modes pass adds every nonzero to
    // N output rows with vector atomics, which piles up on short modes (a
    // 1,000-row mode of a 20M-nonzero tensor takes 20,000 atomics per row).
    // NCopy plans and PingPong plans between sweeps run the mode passes (a
    // PingPong sweep leaves the slab primed for mode 0 again, in the order
    // the reference's next sweep would have); otherwise, and on Morton
    // plans, the all-modes pass.  Gathers are FP32 whatever the plan's
    // precision: this is a gradient check path, not a BF16 one.
    p.gather_fp32_all = true;
    struct Reset { Plan& p; ~Reset() { p.gather_fp32_all = false; } } reset{p};
    if (p.layout == DGPU_LAYOUT_NCOPY) {
        for (int n = 0; n < p.N; ++n) DGPU_TRY(mode_ncopy(p, n));
    } else if (p.layout == DGPU_LAYOUT_PINGPONG && p.next_mode == 0) {
        for (int n = 0; n < p.N; ++n) DGPU_TRY(mode_pingpong(p, n));
        DGPU_TRY(pingpong_drain(p));
    } else {
        DGPU_TRY(launch_mttkrp_all_modes(p));
    }
    for (int n = 0; n < p.N; ++n) DGPU_TRY(gram_into(p, L, n, 0));
    // one device buffer for all modes' gradients, kept on the plan
    size_t total = 0;
    for (int n = 0; n < p.N; ++n) total += (size_t)p.dims[n] * p.Rp;
    if (p.grad_cap < total) {
        dev_free(p.grad_buf);
        p.device_bytes -= p.grad_cap * sizeof(float);
        p.grad_buf = nullptr;
        p.grad_cap = 0;
        DGPU_TRY(dev_alloc(p, (void**)&p.grad_buf, total * sizeof(float)));
        p.grad_cap = total;
    }
    const size_t sm = (size_t)p.R * p.R * sizeof(double);
    if (sm > 48 * 1024 &&
        cudaFuncSetAttribute(k_grad_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) !=
            cudaSuccess) {
        cudaGetLastError();
        set_error("cpopt_gradient: rank %d needs %zu B of shared memory", p.R, sm);
        return DGPU_ERR_ARG;
    }
    size_t off = 0;
    for (int n = 0; n < p.N; ++n) {
        float* g = p.grad_buf + off;
        k_hadamard_others<<<4, 256, 0, p.stream>>>(L.Gd, p.N, n, p.R, L.Wd);
        k_grad_rows<<<grid_for((size_t)p.dims[n] * p.Rp), kLaThreads, sm, p.stream>>>(
            p.Y[n], p.Yhat[n], p.dims[n], p.R, p.Rp, L.Wd, g);
        DGPU_CUDA(cudaGetLastError());
        off += (size_t)p.dims[n] * p.Rp;
    }
    // to the caller's (possibly pageable) buffers through pinned chunks
    off = 0;
    for (int n = 0; n < p.N; ++n) {
        const size_t cnt = (size_t)p.dims[n] * p.Rp;
        DGPU_TRY(copy_to_host_staged(p, grad_host[n], p.grad_buf + off, cnt * sizeof(float)));
        off += cnt;
    }
    return DGPU_OK;
}

}  // namespace dgpu

// The reference's initial factor of mode n (init_random_factors,
// src/dynasor_cpals.cpp:42-69) into host memory: no device involved.
extern "C" int dgpu_init_factor(uint64_t seed, int n, uint32_t rows, int R, int Rp, float* Y) {
    using namespace dgpu;
    if (!Y || n < 0 || n >= kMaxModes || R < 1 || Rp < R) {
        set_error("dgpu_init_factor: bad argument");
        return DGPU_ERR_ARG;
    }
    draw_factor(seed, n, rows, R, Rp, Y);
    return DGPU_OK;
}

// Standalone Gram G = Y^T Y (R x R, leading dimension R) of a device matrix
// (replaces la::gram, src/dynasor_linalg.cpp:47-99).  Temporary partials
// come from the stream-ordered allocator.
extern "C" int dgpu_la_gram(void* stream, const float* Y, uint64_t rows, int R, int Rp, float* G) {
    using namespace dgpu;
    if (!Y || !G || R < 1 || Rp < R || rows == 0 || rows > 0xffffffffull) {
        set_error("dgpu_la_gram: bad argument");
        return DGPU_ERR_ARG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int tiles = (R + kGramTile - 1) / kGramTile;
    const int chunks = (int)std::min<uint64_t>(kGramChunks, (rows + 63) / 64);
    const size_t RR = (size_t)R * R;
    double* part = nullptr;
    double* gd = nullptr;
    double* lam = nullptr;
    DGPU_CUDA(cudaMallocAsync((void**)&part, (size_t)chunks * RR * sizeof(double), st));
    DGPU_CUDA(cudaMallocAsync((void**)&gd, RR * sizeof(double), st));
    DGPU_CUDA(cudaMallocAsync((void**)&lam, (size_t)R * sizeof(double), st));
    DGPU_CUDA(cudaMemsetAsync(G, 0, RR / R * Rp * sizeof(float), st));
    const int rc = launch_gram_partial(dim3(chunks, tiles, tiles), st, Y, (uint32_t)rows, R, Rp, part);
    if (rc == DGPU_OK) k_finalize_mode<<<1, 1024, 0, st>>>(part, chunks, R, Rp, 0, gd, G, nullptr, lam);
    const cudaError_t e = rc == DGPU_OK ? cudaGetLastError() : cudaSuccess;
    cudaFreeAsync(part, st);
    cudaFreeAsync(gd, st);
    cudaFreeAsync(lam, st);
    if (rc != DGPU_OK) return rc;
    if (e != cudaSuccess) {
        set_error("dgpu_la_gram: %s", cudaGetErrorString(e));
        return DGPU_ERR_CUDA;
    }
    return DGPU_OK;
}
