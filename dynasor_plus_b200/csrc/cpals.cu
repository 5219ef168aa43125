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
#include "dgpu_internal.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

namespace dgpu {

int mode_pingpong(Plan& p, int n);
int mode_ncopy(Plan& p, int n);
int launch_mttkrp_all_modes(Plan& p, const Slab& in);

namespace {

constexpr int kLaThreads = 256;
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
    const size_t total = (size_t)rows * Rp;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const size_t i = e / Rp;
        const int c = (int)(e - i * Rp);
        if (c >= R) { Y[e] = 0.f; continue; }
        const float* yh = Yhat + i * Rp;
        Real s = 0;
        for (int k = 0; k < R; ++k) s += (Real)__ldg(yh + k) * Ws[(size_t)k * R + c];
        Y[e] = (float)s;
    }
}

// Partial Grams: grid (chunks, tilesA, tilesB), 32 x 32 output tile per CTA,
// 4 outputs per thread.  partial[(chunk * R + a) * R + b] (FP64).
__global__ void __launch_bounds__(kLaThreads)
k_gram_partial(const float* __restrict__ Y, uint32_t rows, int R, int Rp,
               double* __restrict__ partial)
{
    __shared__ float sa[64][kGramTile];
    __shared__ float sb[64][kGramTile];
    const int a0 = blockIdx.y * kGramTile, b0 = blockIdx.z * kGramTile;
    const int ta = threadIdx.x >> 3;            // 0..31
    const int tb = (threadIdx.x & 7) * 4;       // 0..28
    const uint32_t chunk = (rows + gridDim.x - 1) / gridDim.x;
    const uint32_t r0 = min(rows, blockIdx.x * chunk), r1 = min(rows, r0 + chunk);
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (uint32_t base = r0; base < r1; base += 64) {
        const uint32_t nr = min(64u, r1 - base);
        for (int e = threadIdx.x; e < 64 * kGramTile; e += blockDim.x) {
            const int rr = e / kGramTile, cc = e % kGramTile;
            float va = 0.f, vb = 0.f;
            if (rr < (int)nr) {
                const float* y = Y + (size_t)(base + rr) * Rp;
                if (a0 + cc < R) va = y[a0 + cc];
                if (b0 + cc < R) vb = y[b0 + cc];
            }
            sa[rr][cc] = va;
            sb[rr][cc] = vb;
        }
        __syncthreads();
        for (uint32_t rr = 0; rr < nr; ++rr) {
            const float x = sa[rr][ta];
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] = fmaf(x, sb[rr][tb + q], acc[q]);
        }
        __syncthreads();
    }
    const int a = a0 + ta;
    if (a < R)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int b = b0 + tb + q;
            if (b < R) partial[((size_t)blockIdx.x * R + a) * R + b] = (double)acc[q];
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
    extern __shared__ double sdot[];   // [R]
    if (Yhat) for (int r = threadIdx.x; r < R; r += blockDim.x) sdot[r] = 0.0;
    __syncthreads();
    const size_t total = (size_t)rows * Rp;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % Rp);
        if (c >= R) continue;
        const double l = lam64[c];
        const float inv = l > 1e-20 ? (float)(1.0 / l) : 0.f;
        const float y = Y[e] * inv;
        Y[e] = y;
        if (Yhat) atomicAdd(&sdot[c], (double)y * (double)Yhat[e]);
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

__global__ void k_sumsq(const float* __restrict__ v, uint64_t n, double* __restrict__ out) {
    __shared__ double red[256];
    double s = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
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
    k_gram_partial<<<grid, kLaThreads, 0, p.stream>>>(p.Y[n], p.dims[n], p.R, p.Rp, L.partial);
    const size_t RR = (size_t)p.R * p.R;
    k_finalize_mode<<<1, 1024, 0, p.stream>>>(L.partial, chunks, p.R, p.R, normalise,
                                              L.Gd + (size_t)n * RR, L.G32 + (size_t)n * RR,
                                              p.lambda, L.lam64);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

unsigned grid_for(size_t work, unsigned cap = 148 * 8) {
    return (unsigned)std::max<size_t>(1, std::min<size_t>((work + kLaThreads - 1) / kLaThreads, cap));
}

// One ALS factor update of mode n from Yhat[n] (cpals.cpp:290-321).
int update_mode(Plan& p, const LaLayout& L, int n, int solve_fp64, double ridge, bool last) {
    const size_t RR = (size_t)p.R * p.R;
    if (solve_fp64) {
        k_build_solve_map<double><<<1, 1024, 0, p.stream>>>(L.Gd, p.N, n, p.R, ridge, L.A, L.Wd, L.W32);
        const size_t sm = RR * sizeof(double);
        if (sm > 48 * 1024)
            DGPU_CUDA(cudaFuncSetAttribute(k_apply_map<double>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_apply_map<double><<<grid_for((size_t)p.dims[n] * p.Rp), kLaThreads, sm, p.stream>>>(
            p.Yhat[n], p.dims[n], p.R, p.Rp, L.Wd, p.Y[n]);
    } else {
        k_build_solve_map<float><<<1, 1024, 0, p.stream>>>(L.Gd, p.N, n, p.R, ridge,
                                                           reinterpret_cast<float*>(L.A), L.Wd, L.W32);
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
    k_scale_cols<<<g, kLaThreads, (size_t)p.R * sizeof(double), p.stream>>>(
        p.Y[n], last ? p.Yhat[n] : nullptr, p.dims[n], p.R, p.Rp, L.lam64, L.dot);
    DGPU_CUDA(cudaGetLastError());
    p.yb_stale[n] = true;
    return DGPU_OK;
}

// N(0,1) initial factors exactly as the reference draws them
// (src/dynasor_cpals.cpp:42-69): a splitmix64 step of (seed, n) seeds a
// std::mt19937_64, entries from std::normal_distribution<float>(0, 1),
// row-major, padding zero.  Generated on the host, uploaded once.
int init_factors_host(Plan& p, uint64_t seed) {
    for (int n = 0; n < p.N; ++n) {
        uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (uint64_t)(n + 1);
        z ^= z >> 30; z *= 0xBF58476D1CE4E5B9ULL;
        z ^= z >> 27; z *= 0x94D049BB133111EBULL;
        z ^= z >> 31;
        std::mt19937_64 rng(z);
        std::normal_distribution<float> g(0.0f, 1.0f);
        std::vector<float> Y((size_t)p.dims[n] * p.Rp, 0.f);
        for (uint32_t i = 0; i < p.dims[n]; ++i)
            for (int r = 0; r < p.R; ++r) Y[(size_t)i * p.Rp + r] = g(rng);
        DGPU_CUDA(cudaMemcpyAsync(p.Y[n], Y.data(), Y.size() * sizeof(float),
                                  cudaMemcpyHostToDevice, p.stream));
        DGPU_CUDA(cudaStreamSynchronize(p.stream));
        p.yb_stale[n] = true;
    }
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

int cpals_run(Plan& p, const dgpu_cp_options& o, dgpu_cp_result& res, double* fit_history) {
    using clk = std::chrono::steady_clock;
    res = dgpu_cp_result{};
    LaLayout L{};
    DGPU_TRY(la_ensure(p, L));
    if (!o.use_init) DGPU_TRY(init_factors_host(p, o.seed));
    for (int n = 0; n < p.N; ++n) DGPU_TRY(gram_into(p, L, n, 0));
    double tn2 = 0;
    const Slab& vs = (p.layout == DGPU_LAYOUT_NCOPY) ? p.slab[0] : p.slab[p.cur];
    DGPU_TRY(cp_tensor_norm(p, vs.vals, &tn2));
    res.tensor_norm = std::sqrt(tn2);
    if (o.verbose)
        std::printf("[cpals] modes=%d  rank=%d  padded=%d  nnz=%llu  ||T|| = %.6e  max_iters=%d  "
                    "tol=%.1e  seed=%llu\n", p.N, p.R, p.Rp, (unsigned long long)p.nnz,
                    res.tensor_norm, o.max_iters, o.tol, (unsigned long long)o.seed);

    cudaEvent_t ev[4];
    for (auto& e : ev) DGPU_CUDA(cudaEventCreate(&e));
    const bool jacobi = (o.kernel == DGPU_CP_JACOBI);
    double fit_prev = 0.0;
    const auto t_start = clk::now();
    for (int it = 0; it < o.max_iters; ++it) {
        const auto t_it = clk::now();
        float mt_ms = 0.f, la_ms = 0.f;
        if (jacobi) {
            DGPU_CUDA(cudaEventRecord(ev[0], p.stream));
            DGPU_TRY(launch_mttkrp_all_modes(p, p.layout == DGPU_LAYOUT_NCOPY ? p.slab[0]
                                                                              : p.slab[p.cur]));
            DGPU_CUDA(cudaEventRecord(ev[1], p.stream));
            DGPU_CUDA(cudaEventSynchronize(ev[1]));
            cudaEventElapsedTime(&mt_ms, ev[0], ev[1]);
        }
        for (int n = 0; n < p.N; ++n) {
            DGPU_CUDA(cudaEventRecord(ev[0], p.stream));
            if (!jacobi)
                DGPU_TRY(p.layout == DGPU_LAYOUT_NCOPY ? mode_ncopy(p, n) : mode_pingpong(p, n));
            DGPU_CUDA(cudaEventRecord(ev[1], p.stream));
            DGPU_TRY(update_mode(p, L, n, o.solve_fp64, o.ridge, n == p.N - 1));
            DGPU_CUDA(cudaEventRecord(ev[2], p.stream));
            DGPU_CUDA(cudaEventSynchronize(ev[2]));
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, ev[0], ev[1]);
            cudaEventElapsedTime(&b, ev[1], ev[2]);
            mt_ms += a;
            la_ms += b;
        }
        const int nblk = (int)grid_for((size_t)p.dims[p.N - 1] * p.Rp, kGramChunks);
        k_fit<<<1, 1024, 0, p.stream>>>(L.Gd, p.N, p.R, L.lam64, L.dot, nblk, tn2, L.fitout);
        DGPU_CUDA(cudaGetLastError());
        double fo[4];
        DGPU_CUDA(cudaMemcpyAsync(fo, L.fitout, sizeof(fo), cudaMemcpyDeviceToHost, p.stream));
        DGPU_CUDA(cudaStreamSynchronize(p.stream));
        const double fit = fo[2];
        res.mttkrp_time_s += mt_ms * 1e-3;
        res.linalg_time_s += la_ms * 1e-3;
        if (fit_history) fit_history[it] = fit;
        res.final_fit = fit;
        res.final_residual = fo[3];
        res.iters_done = it + 1;
        const double iter_s = std::chrono::duration<double>(clk::now() - t_it).count();
        if (o.verbose)
            std::printf("[cpals] iter %3d  fit = %.6f  dfit = %.2e  resid = %.3e  iter = %.3f s\n",
                        it, fit, it == 0 ? 0.0 : std::fabs(fit - fit_prev), fo[3], iter_s);
        if (it > 0 && std::fabs(fit - fit_prev) < o.tol) {
            if (o.verbose)
                std::printf("[cpals] converged after %d iterations (|dfit|=%.2e < %.1e)\n", it + 1,
                            std::fabs(fit - fit_prev), o.tol);
            break;
        }
        fit_prev = fit;
    }
    res.total_time_s = std::chrono::duration<double>(clk::now() - t_start).count();
    for (auto& e : ev) cudaEventDestroy(e);
    if (o.verbose)
        std::printf("[cpals] done  iters=%d  final_fit=%.6f  resid=%.3e\n"
                    "[cpals] total = %.3f s   spMTTKRP = %.3f s (%.1f%%)   linalg  = %.3f s (%.1f%%)\n",
                    res.iters_done, res.final_fit, res.final_residual, res.total_time_s,
                    res.mttkrp_time_s, 100.0 * res.mttkrp_time_s / std::max(res.total_time_s, 1e-30),
                    res.linalg_time_s, 100.0 * res.linalg_time_s / std::max(res.total_time_s, 1e-30));
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
    const Slab& in = (p.layout == DGPU_LAYOUT_NCOPY) ? p.slab[0] : p.slab[p.cur];
    DGPU_TRY(launch_mttkrp_all_modes(p, in));
    for (int n = 0; n < p.N; ++n) DGPU_TRY(gram_into(p, L, n, 0));
    float* g = nullptr;
    size_t gmax = 0;
    for (int n = 0; n < p.N; ++n) gmax = std::max(gmax, (size_t)p.dims[n] * p.Rp);
    DGPU_TRY(dev_alloc(p, (void**)&g, gmax * sizeof(float)));
    int rc = DGPU_OK;
    const size_t sm = (size_t)p.R * p.R * sizeof(double);
    if (sm > 48 * 1024 &&
        cudaFuncSetAttribute(k_grad_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) !=
            cudaSuccess) {
        set_error("cpopt_gradient: rank %d needs %zu B of shared memory", p.R, sm);
        rc = DGPU_ERR_ARG;
    }
    for (int n = 0; n < p.N && rc == DGPU_OK; ++n) {
        k_hadamard_others<<<4, 256, 0, p.stream>>>(L.Gd, p.N, n, p.R, L.Wd);
        k_grad_rows<<<grid_for((size_t)p.dims[n] * p.Rp), kLaThreads, sm, p.stream>>>(
            p.Y[n], p.Yhat[n], p.dims[n], p.R, p.Rp, L.Wd, g);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(grad_host[n], g, (size_t)p.dims[n] * p.Rp * sizeof(float),
                            cudaMemcpyDeviceToHost, p.stream) != cudaSuccess ||
            cudaStreamSynchronize(p.stream) != cudaSuccess) {
            set_error("cpopt_gradient: mode %d failed", n);
            rc = DGPU_ERR_CUDA;
        }
    }
    dev_free(g);
    p.device_bytes -= gmax * sizeof(float);
    return rc;
}

}  // namespace dgpu

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
    k_gram_partial<<<dim3(chunks, tiles, tiles), kLaThreads, 0, st>>>(Y, (uint32_t)rows, R, Rp, part);
    k_finalize_mode<<<1, 1024, 0, st>>>(part, chunks, R, Rp, 0, gd, G, nullptr, lam);
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(part, st);
    cudaFreeAsync(gd, st);
    cudaFreeAsync(lam, st);
    if (e != cudaSuccess) {
        set_error("dgpu_la_gram: %s", cudaGetErrorString(e));
        return DGPU_ERR_CUDA;
    }
    return DGPU_OK;
}
