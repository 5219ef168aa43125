// ============================================================================
//  la_warp.cuh -- the R x R normal-equation solve of one CP-ALS factor
//  update, done by a single warp in shared memory (R <= 64).
//
//  Semantics of the reference's la::cholesky_lower + right_solve_chol
//  (src/dynasor_linalg.cpp:160-246): relative ridge eps = ridge * max diag,
//  negative pivots clamped to 0, a zero pivot gives solution component 0.
//  The map W with W[c][:] = solve(e_c) is built so that a factor row is
//  y = yhat * W.
// ============================================================================
#pragma once

namespace dgpu {

// A: R x LDA work matrix holding V (lower triangle used, overwritten by the
// Cholesky factor); invd: R reciprocal pivots (0 for a zero pivot); Wx:
// R x R, entry (r, c) of the solve map stored at Wx[r * R + c].  Called by
// all 32 lanes of one warp.
template <typename Real>
__device__ __forceinline__ void warp_chol_solve_map(Real* A, int LDA, int R, Real* invd,
                                                    double* Wx, double ridge)
{
    const int lane = threadIdx.x & 31;
    Real dmax = 0;
    for (int r = lane; r < R; r += 32) dmax = max(dmax, A[r * LDA + r]);
    for (int o = 16; o > 0; o >>= 1) dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    const Real eps = max((Real)ridge * dmax, (Real)0);
    for (int r = lane; r < R; r += 32) A[r * LDA + r] += eps;
    __syncwarp();
    // right-looking Cholesky.  Step j: one lane takes the pivot (one
    // reciprocal square root: d = s * rsqrt(s), 1/d = rsqrt(s); a serial
    // chain of 2R FP64 divides and square roots costs more otherwise), the
    // lanes scale column j, then the trailing update
    //     A[i][k] -= A[i][j] * A[k][j],   j < k <= i < R
    // is spread over the lanes pair by pair (each element sees the steps j
    // in order, so the arithmetic is that of a row-by-row update).
    for (int j = 0; j < R; ++j) {
        if (lane == 0) {
            Real sj = A[j * LDA + j];
            if (sj < (Real)0) sj = 0;
            const Real rs = sj > (Real)0 ? rsqrt(sj) : (Real)0;
            A[j * LDA + j] = sj * rs;
            invd[j] = rs;
        }
        __syncwarp();
        const Real inv = invd[j];
        for (int i = j + 1 + lane; i < R; i += 32) A[i * LDA + j] *= inv;
        __syncwarp();
        const int m = R - j - 1;                     // trailing block size
        const int pairs = m * (m + 1) / 2;
        for (int q = lane; q < pairs; q += 32) {
            // q -> (a, b), b <= a, row-major over the trailing lower triangle
            int a = (int)((sqrtf(8.0f * (float)q + 1.0f) - 1.0f) * 0.5f);
            while ((a + 1) * (a + 2) / 2 <= q) ++a;
            while (a * (a + 1) / 2 > q) --a;
            const int b = q - a * (a + 1) / 2;
            const int i = j + 1 + a, k = j + 1 + b;
            A[i * LDA + k] -= A[i * LDA + j] * A[k * LDA + j];
        }
        __syncwarp();
    }
    // lane owns columns c = lane, lane + 32; x_c[r] lives at Wx[r * R + c]
    // (the lanes of one access are consecutive doubles); the inner products
    // use four partial sums to shorten the FMA chains
    for (int c = lane; c < R; c += 32) {
        double* xc = Wx + c;
        for (int r = 0; r < R; ++r) xc[(size_t)r * R] = (r == c) ? 1.0 : 0.0;
        for (int r = 0; r < R; ++r) {
            Real s0 = (Real)xc[(size_t)r * R], s1 = 0, s2 = 0, s3 = 0;
            int k = 0;
            for (; k + 4 <= r; k += 4) {
                s0 -= A[r * LDA + k] * (Real)xc[(size_t)k * R];
                s1 -= A[r * LDA + k + 1] * (Real)xc[(size_t)(k + 1) * R];
                s2 -= A[r * LDA + k + 2] * (Real)xc[(size_t)(k + 2) * R];
                s3 -= A[r * LDA + k + 3] * (Real)xc[(size_t)(k + 3) * R];
            }
            for (; k < r; ++k) s0 -= A[r * LDA + k] * (Real)xc[(size_t)k * R];
            xc[(size_t)r * R] = (double)(((s0 + s1) + (s2 + s3)) * invd[r]);
        }
        for (int r = R - 1; r >= 0; --r) {
            Real s0 = (Real)xc[(size_t)r * R], s1 = 0, s2 = 0, s3 = 0;
            int k = r + 1;
            for (; k + 4 <= R; k += 4) {
                s0 -= A[k * LDA + r] * (Real)xc[(size_t)k * R];
                s1 -= A[(k + 1) * LDA + r] * (Real)xc[(size_t)(k + 1) * R];
                s2 -= A[(k + 2) * LDA + r] * (Real)xc[(size_t)(k + 2) * R];
                s3 -= A[(k + 3) * LDA + r] * (Real)xc[(size_t)(k + 3) * R];
            }
            for (; k < R; ++k) s0 -= A[k * LDA + r] * (Real)xc[(size_t)k * R];
            xc[(size_t)r * R] = (double)(((s0 + s1) + (s2 + s3)) * invd[r]);
        }
    }
    __syncwarp();
}

// The same solve with the Cholesky factor in registers (lane i holds row i,
// R <= RMAX; used with RMAX = 16) and each column of the map in its lane's registers:
// the trailing updates take their column-j entries by shuffle, the
// substitutions read the factor's rows from shared memory as broadcasts.
// Arithmetic order per element and per inner product is that of
// warp_chol_solve_map.  A holds V on entry (its ridge already added by the
// caller's helper below) and the factor on exit.
template <typename Real, int RMAX>
__device__ __forceinline__ void warp_chol_solve_map_reg(Real* A, int LDA, int R, Real* invd,
                                                        double* Wx)
{
    const int lane = threadIdx.x & 31;
    Real a[RMAX];
#pragma unroll
    for (int k = 0; k < RMAX; ++k) a[k] = (lane < R && k < R) ? A[lane * LDA + k] : (Real)0;
#pragma unroll
    for (int j = 0; j < RMAX; ++j) {
        if (j >= R) continue;
        Real rs = 0;
        if (lane == j) {
            Real sj = a[j];
            if (sj < (Real)0) sj = 0;
            rs = sj > (Real)0 ? rsqrt(sj) : (Real)0;
            a[j] = sj * rs;
            invd[j] = rs;
        }
        rs = __shfl_sync(0xffffffffu, rs, j);
        if (lane > j) a[j] *= rs;
        const Real aij = a[j];
#pragma unroll
        for (int k = j + 1; k < RMAX; ++k) {
            const Real akj = __shfl_sync(0xffffffffu, aij, k);
            if (k <= lane && k < R) a[k] -= aij * akj;
        }
    }
    if (lane < R) {
#pragma unroll
        for (int k = 0; k < RMAX; ++k)
            if (k < R) A[lane * LDA + k] = a[k];
    }
    __syncwarp();
    const int c = lane;
    double x[RMAX];
#pragma unroll
    for (int r = 0; r < RMAX; ++r) {
        if (r >= R) continue;
        Real s0 = (r == c) ? (Real)1 : (Real)0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
        for (int k = 0; k + 4 <= r; k += 4) {
            s0 -= A[r * LDA + k] * (Real)x[k];
            s1 -= A[r * LDA + k + 1] * (Real)x[k + 1];
            s2 -= A[r * LDA + k + 2] * (Real)x[k + 2];
            s3 -= A[r * LDA + k + 3] * (Real)x[k + 3];
        }
#pragma unroll
        for (int k = (r / 4) * 4; k < r; ++k) s0 -= A[r * LDA + k] * (Real)x[k];
        x[r] = (double)(((s0 + s1) + (s2 + s3)) * invd[r]);
    }
#pragma unroll
    for (int r = RMAX - 1; r >= 0; --r) {
        if (r >= R) continue;
        Real s0 = (Real)x[r], s1 = 0, s2 = 0, s3 = 0;
        const int k = r + 1 + ((R - r - 1) / 4) * 4;      // first index of the tail
#pragma unroll
        for (int kk = r + 1; kk + 4 <= RMAX; kk += 4) {
            if (kk + 4 <= R) {
                s0 -= A[kk * LDA + r] * (Real)x[kk];
                s1 -= A[(kk + 1) * LDA + r] * (Real)x[kk + 1];
                s2 -= A[(kk + 2) * LDA + r] * (Real)x[kk + 2];
                s3 -= A[(kk + 3) * LDA + r] * (Real)x[kk + 3];
            }
        }
#pragma unroll
        for (int kk = r + 1; kk < RMAX; ++kk)
            if (kk >= k && kk < R) s0 -= A[kk * LDA + r] * (Real)x[kk];
        x[r] = (double)(((s0 + s1) + (s2 + s3)) * invd[r]);
    }
    if (c < R) {
#pragma unroll
        for (int r = 0; r < RMAX; ++r)
            if (r < R) Wx[(size_t)r * R + c] = x[r];
    }
    __syncwarp();
}

// Relative ridge (eps = ridge * max diag, at least 0) on V's diagonal, as
// warp_chol_solve_map starts.
template <typename Real>
__device__ __forceinline__ void warp_ridge(Real* A, int LDA, int R, double ridge) {
    const int lane = threadIdx.x & 31;
    Real dmax = 0;
    for (int r = lane; r < R; r += 32) dmax = max(dmax, A[r * LDA + r]);
    for (int o = 16; o > 0; o >>= 1) dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    const Real eps = max((Real)ridge * dmax, (Real)0);
    for (int r = lane; r < R; r += 32) A[r * LDA + r] += eps;
    __syncwarp();
}

}  // namespace dgpu
