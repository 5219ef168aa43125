// ============================================================================
//  multistart.cu -- K random-restart CP-ALS runs batched into one plan.
//
//  The reference runs restarts one after another (each a full cpals call,
//  src/dynasor_cpals.cpp:120-396, with its own seed).  Here the K restarts'
//  factors are concatenated column-wise into one plan of rank K * Re, so one
//  MTTKRP sweep over the FLYCOO layout serves all restarts (MTTKRP is
//  column-separable: column c of Yhat depends only on column c of the other
//  factors).  Everything that mixes columns is per restart: the Grams are
//  the K diagonal Re x Re blocks, each restart solves its own normal
//  equations, normalises its own columns and has its own fit and stop rule.
//  A restart that meets the stop rule is frozen (its columns are no longer
//  updated) while the others continue, so every restart follows the
//  trajectory of the corresponding single run.
//
//  Restart k starts from the reference's N(0,1) initialisation with seed
//  `seed + k`.  After the first (eager) iteration the remaining ones run
//  as one graph launch with a device-side WHILE loop (as in cpals.cu).
// ============================================================================
#include "dgpu_internal.h"
#include "la_warp.cuh"
#include "apply_map.cuh"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <atomic>
#include <random>
#include <thread>
#include <vector>

namespace dgpu {

int mode_pingpong(Plan& p, int n);
int mode_ncopy(Plan& p, int n);

namespace {

constexpr int kMsChunks = 148;
constexpr int kMsThreads = 256;

// Partial Gram blocks: grid (chunks, K).  Block k covers columns
// [k*Re, (k+1)*Re); entries e = tid + 256 q (Re <= 64, so q < 16).
__global__ void __launch_bounds__(kMsThreads)
k_ms_gram_partial(const float* __restrict__ Y, uint32_t rows, int Rp, int Re,
                  const int* __restrict__ active, float* __restrict__ partial)
{
    const int k = blockIdx.y, K = gridDim.y;
    if (active && !active[k]) return;
    __shared__ float sy[64][65];
    const int RR = Re * Re;
    const uint32_t chunk = (rows + gridDim.x - 1) / gridDim.x;
    const uint32_t r0 = min(rows, blockIdx.x * chunk), r1 = min(rows, r0 + chunk);
    float acc[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc[q] = 0.f;
    for (uint32_t base = r0; base < r1; base += 64) {
        const uint32_t nr = min(64u, r1 - base);
        for (int e = threadIdx.x; e < 64 * Re; e += blockDim.x) {
            const int rr = e / Re, cc = e % Re;
            sy[rr][cc] = rr < (int)nr ? Y[(size_t)(base + rr) * Rp + (size_t)k * Re + cc] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int e = threadIdx.x + kMsThreads * q;
            if (e < RR) {
                const int a = e / Re, b = e % Re;
                float s = acc[q];
                for (uint32_t rr = 0; rr < nr; ++rr) s = fmaf(sy[rr][a], sy[rr][b], s);
                acc[q] = s;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int e = threadIdx.x + kMsThreads * q;
        if (e < RR) partial[((size_t)blockIdx.x * K + k) * RR + e] = acc[q];
    }
}

__device__ __forceinline__ void ms_cp_async16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;"
                 :: "r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))), "l"(src),
                    "r"(src_bytes) : "memory");
}

// The same partial Gram blocks for RE in {16, 32} with register tiles: a
// thread owns a 4 x 4 tile of its restart's RE x RE block (RE*RE/16
// threads per row group, 256 / that many row groups taking interleaved
// rows), rows stream in 64-row steps through a 4-stage cp.async ring, and
// the row groups' tiles are added in group order at the end.
template <int RE>
__global__ void __launch_bounds__(kMsThreads)
k_ms_gram_tiles(const float* __restrict__ Y, uint32_t rows, int Rp,
                const int* __restrict__ active, float* __restrict__ partial)
{
    constexpr int TPG = RE * RE / 16;                 // threads per row group
    constexpr int NG = kMsThreads / TPG;              // row groups
    constexpr int ROWS = 64, STAGES = 4;
    constexpr int CPR = RE / 4;                       // 16-byte chunks per row
    static_assert(NG >= 1 && ROWS * CPR <= 2 * kMsThreads, "one or two copies per thread");
    __shared__ __align__(16) float ring[STAGES][ROWS][RE];
    const int k = blockIdx.y, K = gridDim.y;
    if (active && !active[k]) return;
    const int grp = threadIdx.x / TPG, u = threadIdx.x % TPG;
    const int ta = u % (RE / 4), tb = u / (RE / 4);
    const uint32_t chunk = (rows + gridDim.x - 1) / gridDim.x;
    const uint32_t r0 = min(rows, blockIdx.x * chunk), r1 = min(rows, r0 + chunk);
    const uint32_t nsteps = (r1 - r0 + ROWS - 1) / ROWS;
    auto issue = [&](uint32_t st) {
        const uint32_t base = r0 + st * ROWS;
        const uint32_t nr = min((uint32_t)ROWS, r1 - base);
        for (int q = threadIdx.x; q < ROWS * CPR; q += kMsThreads) {
            const int rr = q / CPR, c4 = q % CPR;
            const bool ok = (uint32_t)rr < nr;
            const float* src = ok ? Y + (size_t)(base + rr) * Rp + (size_t)k * RE + 4 * c4 : Y;
            ms_cp_async16(&ring[st % STAGES][rr][4 * c4], src, ok ? 16 : 0);
        }
    };
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
#pragma unroll
    for (int st = 0; st < STAGES - 1; ++st) {
        if ((uint32_t)st < nsteps) issue(st);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (uint32_t st = 0; st < nsteps; ++st) {
        asm volatile("cp.async.wait_group %0;" :: "n"(STAGES - 2) : "memory");
        __syncthreads();
        if (st + STAGES - 1 < nsteps) issue(st + STAGES - 1);
        asm volatile("cp.async.commit_group;" ::: "memory");
        const uint32_t nr = min((uint32_t)ROWS, r1 - (r0 + st * ROWS));
        const float (*A)[RE] = ring[st % STAGES];
#pragma unroll 4
        for (uint32_t rr = grp; rr < nr; rr += NG) {
            const float4 av = *reinterpret_cast<const float4*>(&A[rr][4 * ta]);
            const float4 bv = *reinterpret_cast<const float4*>(&A[rr][4 * tb]);
            const float x[4] = {av.x, av.y, av.z, av.w};
            const float y[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(x[i], y[j], acc[i][j]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    // row-group tiles -> shared memory (the ring is free now), summed in
    // group order by the first group
    float* red = &ring[0][0][0];
    static_assert(NG * RE * RE <= STAGES * ROWS * RE, "reduction fits in the ring");
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) red[(size_t)grp * RE * RE + (4 * ta + i) * RE + 4 * tb + j] = acc[i][j];
    __syncthreads();
    for (int e = threadIdx.x; e < RE * RE; e += kMsThreads) {
        double sum = 0.0;
        for (int g = 0; g < NG; ++g) sum += (double)red[(size_t)g * RE * RE + e];
        partial[((size_t)blockIdx.x * K + k) * RE * RE + e] = (float)sum;
    }
}

// Reduce the partial blocks (FP64); with `normalise`, lambda = sqrt(diag)
// and the block of the column-normalised factor is kept.  grid K.
__global__ void __launch_bounds__(kMsThreads)
k_ms_finalize(const float* __restrict__ partial, int chunks, int Re, int normalise,
              const int* __restrict__ active, double* __restrict__ Gd_n,
              double* __restrict__ lam, float* __restrict__ lambda)
{
    const int k = blockIdx.x, K = gridDim.x;
    if (active && !active[k]) return;
    const int RR = Re * Re;
    double* G = Gd_n + (size_t)k * RR;
    for (int e = threadIdx.x; e < RR; e += blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < chunks; ++c) s += (double)partial[((size_t)c * K + k) * RR + e];
        G[e] = s;
    }
    __syncthreads();
    if (!normalise) return;
    for (int r = threadIdx.x; r < Re; r += blockDim.x) {
        const double l = sqrt(max(G[r * Re + r], 0.0));
        lam[k * Re + r] = l;
        lambda[k * Re + r] = (float)l;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < RR; e += blockDim.x) {
        const double la = lam[k * Re + e / Re], lb = lam[k * Re + e % Re];
        const double ia = la > 1e-20 ? 1.0 / la : 0.0, ib = lb > 1e-20 ? 1.0 / lb : 0.0;
        G[e] *= ia * ib;
    }
}

// Solve map of restart k (one warp): V = Hadamard of the other modes'
// blocks, ridge, Cholesky, W.  grid K, 32 threads.
template <typename Real>
__global__ void __launch_bounds__(32)
k_ms_solve(const double* __restrict__ Gd, int N, int n, int Re, double ridge,
           const int* __restrict__ active, double* __restrict__ W)
{
    const int k = blockIdx.x, K = gridDim.x;
    if (!active[k]) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int RR = Re * Re, LDA = Re + 1;
    double* Wx = reinterpret_cast<double*>(smraw);           // Re x Re
    Real* A = reinterpret_cast<Real*>(Wx + RR);              // Re x LDA
    Real* invd = A + Re * LDA;                               // Re
    for (int e = threadIdx.x; e < RR; e += 32) {
        double v = 1.0;
        for (int m = 0; m < N; ++m)
            if (m != n) v *= Gd[((size_t)m * K + k) * RR + e];
        A[(e / Re) * LDA + e % Re] = (Real)v;
    }
    __syncwarp();
    warp_chol_solve_map<Real>(A, LDA, Re, invd, Wx, ridge);
    for (int e = threadIdx.x; e < RR; e += 32) W[(size_t)k * RR + e] = Wx[e];
}

// Y[i][k*Re + c] = sum_j Yhat[i][k*Re + j] W_k[j][c] for active restarts.
template <typename Real>
__global__ void __launch_bounds__(kMsThreads)
k_ms_apply(const float* __restrict__ Yhat, uint32_t rows, int Rp, int K, int Re,
           const double* __restrict__ W, const int* __restrict__ active, float* __restrict__ Y)
{
    const int KR = K * Re, RR = Re * Re;
    const size_t total = (size_t)rows * KR;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t i = e / KR;
        const int col = (int)(e - i * KR), k = col / Re, c = col - k * Re;
        if (!active[k]) continue;
        const float* yh = Yhat + i * Rp + (size_t)k * Re;
        const double* w = W + (size_t)k * RR + c;
        Real a0 = 0, a1 = 0;
        int j = 0;
        for (; j + 2 <= Re; j += 2) {
            a0 += (Real)__ldg(yh + j) * (Real)__ldg(w + (size_t)j * Re);
            a1 += (Real)__ldg(yh + j + 1) * (Real)__ldg(w + (size_t)(j + 1) * Re);
        }
        if (j < Re) a0 += (Real)__ldg(yh + j) * (Real)__ldg(w + (size_t)j * Re);
        Y[i * Rp + col] = (float)(a0 + a1);
    }
}

// Column scaling by 1/lambda and (last mode) per-column <Y, Yhat> partials,
// float4 per thread: every float4 a thread visits lies in one group of four
// columns (the grid-stride is a multiple of Rp / 4), so the reciprocals and
// the active flags are read once and the dot takes one shared-memory atomic
// per column and thread.  Inactive restarts and padding columns are left as
// they are (scale 1, no dot).
__global__ void __launch_bounds__(kMsThreads)
k_ms_scale4(float* __restrict__ Y, const float* __restrict__ Yhat, uint32_t rows, int Rp, int K,
            int Re, const double* __restrict__ lam, const int* __restrict__ active,
            double* __restrict__ dot_partial)
{
    extern __shared__ double sdot[];                         // [K*Re]
    const int KR = K * Re;
    if (Yhat) for (int c = threadIdx.x; c < KR; c += blockDim.x) sdot[c] = 0.0;
    __syncthreads();
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t first = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int c0 = (int)(first % (size_t)(Rp >> 2)) * 4;
    float inv[4];
    bool use[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int col = c0 + j;
        use[j] = col < KR && active[col / Re] != 0;
        const double l = use[j] ? lam[col] : 0.0;
        inv[j] = !use[j] ? 1.f : (l > 1e-20 ? (float)(1.0 / l) : 0.f);
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    float4* Y4 = reinterpret_cast<float4*>(Y);
    const float4* H4 = reinterpret_cast<const float4*>(Yhat);
    const size_t total4 = (size_t)rows * (Rp >> 2);
    constexpr int U = 4;
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
            if (use[j]) atomicAdd(&sdot[c0 + j], acc[j]);
    }
    __syncthreads();
    if (Yhat)
        for (int c = threadIdx.x; c < KR; c += blockDim.x)
            dot_partial[(size_t)blockIdx.x * KR + c] = sdot[c];
}

// Column scaling by 1/lambda and (last mode) per-column <Y, Yhat> partials.
__global__ void __launch_bounds__(kMsThreads)
k_ms_scale(float* __restrict__ Y, const float* __restrict__ Yhat, uint32_t rows, int Rp, int K,
           int Re, const double* __restrict__ lam, const int* __restrict__ active,
           double* __restrict__ dot_partial)
{
    extern __shared__ double sdot[];                         // [K*Re]
    const int KR = K * Re;
    if (Yhat) for (int c = threadIdx.x; c < KR; c += blockDim.x) sdot[c] = 0.0;
    __syncthreads();
    const size_t total = (size_t)rows * KR;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t i = e / KR;
        const int col = (int)(e - i * KR);
        if (!active[col / Re]) continue;
        const double l = lam[col];
        const float inv = l > 1e-20 ? (float)(1.0 / l) : 0.f;
        const float y = Y[i * Rp + col] * inv;
        Y[i * Rp + col] = y;
        if (Yhat) atomicAdd(&sdot[col], (double)y * (double)Yhat[i * Rp + col]);
    }
    __syncthreads();
    if (Yhat)
        for (int c = threadIdx.x; c < KR; c += blockDim.x)
            dot_partial[(size_t)blockIdx.x * KR + c] = sdot[c];
}

// Per-restart fit, the reference's stop rule (|fit_i - fit_{i-1}| < tol
// after the first iteration, src/dynasor_cpals.cpp:371-379), freezing of
// converged restarts and, under the device loop, the WHILE condition.
// One block; warp w handles restarts w, w + 32, ...
__global__ void __launch_bounds__(1024)
k_ms_fit(const double* __restrict__ Gd, int N, int K, int Re, const double* __restrict__ lam,
         const double* __restrict__ dot_partial, int chunks, double tnorm2, double tol,
         int max_iters, int* __restrict__ active, double* __restrict__ prevfit,
         int* __restrict__ iters, double* __restrict__ hist, double* __restrict__ st,
         cudaGraphConditionalHandle h, int use_handle)
{
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int it = (int)st[0];
    const int RR = Re * Re, KR = K * Re;
    for (int k = warp; k < K; k += nw) {
        if (!active[k]) continue;
        double s_in = 0.0, s_m = 0.0;
        for (int r = lane; r < Re; r += 32) {
            double d = 0.0;
            for (int c = 0; c < chunks; ++c) d += dot_partial[(size_t)c * KR + k * Re + r];
            s_in += lam[k * Re + r] * d;
        }
        for (int e = lane; e < RR; e += 32) {
            double g = 1.0;
            for (int m = 0; m < N; ++m) g *= Gd[((size_t)m * K + k) * RR + e];
            s_m += lam[k * Re + e / Re] * lam[k * Re + e % Re] * g;
        }
        for (int o = 16; o > 0; o >>= 1) {
            s_in += __shfl_xor_sync(0xffffffffu, s_in, o);
            s_m += __shfl_xor_sync(0xffffffffu, s_m, o);
        }
        if (lane == 0) {
            double r2 = tnorm2 - 2.0 * s_in + max(0.0, s_m);
            if (r2 < 0.0) r2 = 0.0;
            const double fit = 1.0 - sqrt(r2) / max(sqrt(tnorm2), 1e-30);
            hist[(size_t)k * max_iters + it] = fit;
            iters[k] = it + 1;
            const bool stop = (it > 0 && fabs(fit - prevfit[k]) < tol) || (it + 1 >= max_iters);
            prevfit[k] = fit;
            if (stop) active[k] = 0;
            else atomicOr(&any, 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        st[0] = (double)(it + 1);
        st[1] = (double)any;
        if (use_handle) cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

unsigned ms_grid(size_t work) {
    return (unsigned)std::max<size_t>(1, std::min<size_t>((work + kMsThreads - 1) / kMsThreads,
                                                          148 * 8));
}

}  // namespace

int cpals_multistart_run(Plan& p, int K, const dgpu_cp_options& o, dgpu_cp_result* res,
                         double* fit_history)
{
    using clk = std::chrono::steady_clock;
    const int N = p.N, R = p.R, Re = R / K, RR = Re * Re, KR = R;
    const int max_iters = o.max_iters;
    for (int k = 0; k < K; ++k) res[k] = dgpu_cp_result{};
    if (max_iters <= 0) return DGPU_OK;

    // ---- scratch ----------------------------------------------------------
    const size_t nd = (size_t)N * K * RR + (size_t)K * RR + KR + (size_t)kMsChunks * KR + K +
                      (size_t)K * max_iters + 4;
    const size_t nf = (size_t)kMsChunks * K * RR;
    double* dbuf = nullptr;
    float* fbuf = nullptr;
    int* ibuf = nullptr;
    DGPU_TRY(dev_alloc(p, (void**)&dbuf, nd * sizeof(double)));
    struct Free {
        Plan& p; void* a; void* b; void* c; size_t bytes;
        ~Free() { dev_free(a); dev_free(b); dev_free(c); p.device_bytes -= bytes; }
    } fr{p, dbuf, nullptr, nullptr, 0};
    DGPU_TRY(dev_alloc(p, (void**)&fbuf, nf * sizeof(float)));
    fr.b = fbuf;
    DGPU_TRY(dev_alloc(p, (void**)&ibuf, 2 * (size_t)K * sizeof(int)));
    fr.c = ibuf;
    fr.bytes = nd * sizeof(double) + nf * sizeof(float) + 2 * (size_t)K * sizeof(int);
    double* Gd = dbuf;
    double* W = Gd + (size_t)N * K * RR;
    double* lam = W + (size_t)K * RR;
    double* dot = lam + KR;
    double* prevfit = dot + (size_t)kMsChunks * KR;
    double* hist = prevfit + K;
    double* st = hist + (size_t)K * max_iters;
    float* partial = fbuf;
    int* active = ibuf;
    int* iters = ibuf + K;

    // ---- initial factors: restart k from seed + k, the reference's draw ---
    if (!o.use_init) {
        // one generator per (mode, restart), drawn on parallel host threads;
        // Gauss-Seidel never reads mode 0's initial factor (it is solved
        // first, from the other modes' Grams), so its draw is skipped and the
        // factor zeroed -- the other draws are unchanged (own generators)
        const int first = (o.kernel != DGPU_CP_JACOBI && max_iters > 0) ? 1 : 0;
        std::vector<std::vector<float>> Y(N);
        for (int n = first; n < N; ++n) Y[n].assign((size_t)p.dims[n] * p.Rp, 0.f);
        const int jobs = (N - first) * K;
        const int nth = std::max(1, std::min<int>(jobs, (int)std::thread::hardware_concurrency()));
        std::atomic<int> next{0};
        std::vector<std::thread> th;
        for (int t = 0; t < nth; ++t)
            th.emplace_back([&]() {
                for (int j = next++; j < jobs; j = next++) {
                    const int n = first + j / K, k = j % K;
                    uint64_t z = (o.seed + (uint64_t)k) + 0x9E3779B97F4A7C15ULL * (uint64_t)(n + 1);
                    z ^= z >> 30; z *= 0xBF58476D1CE4E5B9ULL;
                    z ^= z >> 27; z *= 0x94D049BB133111EBULL;
                    z ^= z >> 31;
                    std::mt19937_64 rng(z);
                    std::normal_distribution<float> g(0.0f, 1.0f);
                    float* y = Y[n].data();
                    for (uint32_t i = 0; i < p.dims[n]; ++i)
                        for (int r = 0; r < Re; ++r) y[(size_t)i * p.Rp + (size_t)k * Re + r] = g(rng);
                }
            });
        for (auto& t : th) t.join();
        for (int n = 0; n < N; ++n) {
            if (n < first)
                DGPU_CUDA(cudaMemsetAsync(p.Y[n], 0, (size_t)p.dims[n] * p.Rp * sizeof(float),
                                          p.stream));
            else
                DGPU_CUDA(cudaMemcpyAsync(p.Y[n], Y[n].data(), Y[n].size() * sizeof(float),
                                          cudaMemcpyHostToDevice, p.stream));
            p.yb_stale[n] = true;
        }
        DGPU_CUDA(cudaStreamSynchronize(p.stream));
    }
    {
        std::vector<int> ones(K, 1);
        DGPU_CUDA(cudaMemcpyAsync(active, ones.data(), K * sizeof(int), cudaMemcpyHostToDevice,
                                  p.stream));
        DGPU_CUDA(cudaMemsetAsync(iters, 0, K * sizeof(int), p.stream));
        DGPU_CUDA(cudaMemsetAsync(prevfit, 0, K * sizeof(double), p.stream));
        DGPU_CUDA(cudaMemsetAsync(st, 0, 4 * sizeof(double), p.stream));
        DGPU_CUDA(cudaStreamSynchronize(p.stream));
    }
    const int chunks_of = kMsChunks;
    auto gram = [&](int n, int normalise) -> int {
        const int chunks = (int)std::min<uint32_t>(chunks_of, std::max<uint32_t>(1u, (p.dims[n] + 63) / 64));
        if (Re == 16)
            k_ms_gram_tiles<16><<<dim3(chunks, K), kMsThreads, 0, p.stream>>>(
                p.Y[n], p.dims[n], p.Rp, normalise ? active : nullptr, partial);
        else if (Re == 32)
            k_ms_gram_tiles<32><<<dim3(chunks, K), kMsThreads, 0, p.stream>>>(
                p.Y[n], p.dims[n], p.Rp, normalise ? active : nullptr, partial);
        else
            k_ms_gram_partial<<<dim3(chunks, K), kMsThreads, 0, p.stream>>>(p.Y[n], p.dims[n], p.Rp, Re,
                                                                              normalise ? active : nullptr,
                                                                              partial);
        k_ms_finalize<<<K, kMsThreads, 0, p.stream>>>(partial, chunks, Re, normalise,
                                                      normalise ? active : nullptr,
                                                      Gd + (size_t)n * K * RR, lam, p.lambda);
        DGPU_CUDA(cudaGetLastError());
        return DGPU_OK;
    };
    for (int n = 0; n < N; ++n) DGPU_TRY(gram(n, 0));
    double tn2 = 0.0;
    const Slab& vs = (p.layout == DGPU_LAYOUT_NCOPY) ? p.slab[0] : p.slab[p.cur];
    DGPU_TRY(cp_tensor_norm(p, vs.vals, &tn2));

    const size_t solve_sm = (size_t)RR * sizeof(double) +
                            (size_t)Re * (Re + 2) * (o.solve_fp64 ? sizeof(double) : sizeof(float));
    const bool jacobi = (o.kernel == DGPU_CP_JACOBI);
    if (solve_sm > 48 * 1024) {
        DGPU_CUDA(cudaFuncSetAttribute(k_ms_solve<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)solve_sm));
        DGPU_CUDA(cudaFuncSetAttribute(k_ms_solve<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)solve_sm));
    }
    cudaEvent_t ev[3];
    for (auto& e : ev) DGPU_CUDA(cudaEventCreate(&e));
    struct Ev { cudaEvent_t* e; ~Ev() { for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]); } } evg{ev};

    auto update = [&](int n, bool last) -> int {
        if (o.solve_fp64)
            k_ms_solve<double><<<K, 32, solve_sm, p.stream>>>(Gd, N, n, Re, o.ridge, active, W);
        else
            k_ms_solve<float><<<K, 32, solve_sm, p.stream>>>(Gd, N, n, Re, o.ridge, active, W);
        const unsigned g = ms_grid((size_t)p.dims[n] * KR);
        if (o.solve_fp64 && (Re == 16 || Re == 32)) {
            // block-diagonal map, one column block per restart, on the FP64
            // tensor pipe
            const unsigned gx = std::max(1u, std::min(g, (unsigned)(148 * 2 * 8 / K + 1)));
            if (Re == 16)
                k_apply_map_dmma<16><<<dim3(gx, K), kApplyThreads, 0, p.stream>>>(
                    p.Yhat[n], p.dims[n], Re, p.Rp, W, (size_t)RR, active, p.Y[n]);
            else
                k_apply_map_dmma<32><<<dim3(gx, K), kApplyThreads, 0, p.stream>>>(
                    p.Yhat[n], p.dims[n], Re, p.Rp, W, (size_t)RR, active, p.Y[n]);
        } else if (o.solve_fp64)
            k_ms_apply<double><<<g, kMsThreads, 0, p.stream>>>(p.Yhat[n], p.dims[n], p.Rp, K, Re, W,
                                                               active, p.Y[n]);
        else
            k_ms_apply<float><<<g, kMsThreads, 0, p.stream>>>(p.Yhat[n], p.dims[n], p.Rp, K, Re, W,
                                                              active, p.Y[n]);
        DGPU_CUDA(cudaGetLastError());
        DGPU_TRY(gram(n, 1));
        const unsigned gs = std::min<unsigned>(ms_grid((size_t)p.dims[n] * KR), kMsChunks);
        if (((size_t)gs * kMsThreads) % (size_t)(p.Rp / 4) == 0)
            k_ms_scale4<<<gs, kMsThreads, (size_t)KR * sizeof(double), p.stream>>>(
                p.Y[n], last ? p.Yhat[n] : nullptr, p.dims[n], p.Rp, K, Re, lam, active, dot);
        else
            k_ms_scale<<<gs, kMsThreads, (size_t)KR * sizeof(double), p.stream>>>(
                p.Y[n], last ? p.Yhat[n] : nullptr, p.dims[n], p.Rp, K, Re, lam, active, dot);
        DGPU_CUDA(cudaGetLastError());
        p.yb_stale[n] = true;
        return DGPU_OK;
    };
    // one iteration; `record` brackets the MTTKRPs and updates with events
    auto enqueue = [&](bool record, cudaGraphConditionalHandle h, int use_h) -> int {
        if (record) DGPU_CUDA(cudaEventRecord(ev[0], p.stream));
        if (jacobi)
            for (int n = 0; n < N; ++n)
                DGPU_TRY(p.layout == DGPU_LAYOUT_NCOPY ? mode_ncopy(p, n) : mode_pingpong(p, n));
        for (int n = 0; n < N; ++n) {
            if (!jacobi)
                DGPU_TRY(p.layout == DGPU_LAYOUT_NCOPY ? mode_ncopy(p, n) : mode_pingpong(p, n));
            DGPU_TRY(update(n, n == N - 1));
        }
        const int chunks_last = (int)std::min<unsigned>(ms_grid((size_t)p.dims[N - 1] * KR), kMsChunks);
        k_ms_fit<<<1, 1024, 0, p.stream>>>(Gd, N, K, Re, lam, dot, chunks_last, tn2, o.tol, max_iters,
                                           active, prevfit, iters, hist, st, h, use_h);
        DGPU_CUDA(cudaGetLastError());
        if (record) DGPU_CUDA(cudaEventRecord(ev[1], p.stream));
        return DGPU_OK;
    };

    const auto t0 = clk::now();
    const int cur_start = p.cur;
    double any = 0.0;
    cudaGraphConditionalHandle none{};
    DGPU_TRY(enqueue(true, none, 0));
    DGPU_CUDA(cudaMemcpyAsync(&any, st + 1, sizeof(double), cudaMemcpyDeviceToHost, p.stream));
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    float first_ms = 0.f;
    cudaEventElapsedTime(&first_ms, ev[0], ev[1]);
    double gpu_ms = first_ms;

    bool looped = false;
    if (any != 0.0 && o.graphs && !p.timing &&
        (p.layout == DGPU_LAYOUT_NCOPY || p.cur == cur_start)) {
        // remaining iterations: one graph launch with a device-side loop
        const int cur0 = p.cur, nm0 = p.next_mode;
        const uint64_t pp0 = p.pp_transitions;
        bool stale0[kMaxModes];
        for (int n = 0; n < kMaxModes; ++n) stale0[n] = p.yb_stale[n];
        cudaGraph_t outer = nullptr;
        cudaGraphExec_t gx = nullptr;
        struct G { cudaGraph_t& g; cudaGraphExec_t& x;
                   ~G() { if (x) cudaGraphExecDestroy(x); if (g) cudaGraphDestroy(g); } } gg{outer, gx};
        bool ok = cudaGraphCreate(&outer, 0) == cudaSuccess;
        cudaGraphConditionalHandle h{};
        cudaGraphNodeParams np{};
        if (ok) ok = cudaGraphConditionalHandleCreate(&h, outer, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        cudaGraphNode_t node;
        if (ok) {
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = h;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            ok = cudaGraphAddNode(&node, outer, nullptr, 0, &np) == cudaSuccess;
        }
        if (ok)
            ok = cudaStreamBeginCaptureToGraph(p.stream, np.conditional.phGraph_out[0], nullptr,
                                               nullptr, 0, cudaStreamCaptureModeRelaxed) == cudaSuccess;
        if (ok) {
            const int rc = enqueue(false, h, 1);
            cudaGraph_t cap = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(p.stream, &cap);
            ok = rc == DGPU_OK && ec == cudaSuccess &&
                 cudaGraphInstantiate(&gx, outer, 0) == cudaSuccess;
            if (rc != DGPU_OK && rc != DGPU_ERR_CUDA) return rc;
        }
        if (ok) {
            DGPU_CUDA(cudaEventRecord(ev[0], p.stream));
            DGPU_CUDA(cudaGraphLaunch(gx, p.stream));
            DGPU_CUDA(cudaEventRecord(ev[1], p.stream));
            DGPU_CUDA(cudaStreamSynchronize(p.stream));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[0], ev[1]);
            gpu_ms += ms;
            looped = true;
        } else {
            cudaGetLastError();
            p.cur = cur0;
            p.next_mode = nm0;
            p.pp_transitions = pp0;
            for (int n = 0; n < kMaxModes; ++n) p.yb_stale[n] = stale0[n];
        }
    }
    if (!looped) {
        for (int it = 1; it < max_iters && any != 0.0; ++it) {
            DGPU_TRY(enqueue(true, none, 0));
            DGPU_CUDA(cudaMemcpyAsync(&any, st + 1, sizeof(double), cudaMemcpyDeviceToHost, p.stream));
            DGPU_CUDA(cudaStreamSynchronize(p.stream));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[0], ev[1]);
            gpu_ms += ms;
        }
    }
    const double total_s = std::chrono::duration<double>(clk::now() - t0).count();
    (void)gpu_ms;

    std::vector<double> hh((size_t)K * max_iters);
    std::vector<int> ih(K);
    DGPU_CUDA(cudaMemcpy(hh.data(), hist, hh.size() * sizeof(double), cudaMemcpyDeviceToHost));
    DGPU_CUDA(cudaMemcpy(ih.data(), iters, K * sizeof(int), cudaMemcpyDeviceToHost));
    for (int k = 0; k < K; ++k) {
        dgpu_cp_result& r = res[k];
        r.iters_done = ih[k];
        r.final_fit = ih[k] > 0 ? hh[(size_t)k * max_iters + ih[k] - 1] : 0.0;
        r.final_residual = (1.0 - r.final_fit) * std::sqrt(tn2);   // fit = 1 - resid/||T||
        r.tensor_norm = std::sqrt(tn2);
        // the batch's wall time; the device time is not split by phase
        r.total_time_s = total_s;
        r.mttkrp_time_s = 0.0;
        r.linalg_time_s = 0.0;
        if (fit_history)
            for (int i = 0; i < max_iters; ++i)
                fit_history[(size_t)k * max_iters + i] = i < ih[k] ? hh[(size_t)k * max_iters + i] : 0.0;
    }
    if (o.verbose)
        for (int k = 0; k < K; ++k)
            std::printf("[cpals] restart %d (seed %llu): iters=%d  final_fit=%.6f\n", k,
                        (unsigned long long)(o.seed + k), res[k].iters_done, res[k].final_fit);
    return DGPU_OK;
}

}  // namespace dgpu
