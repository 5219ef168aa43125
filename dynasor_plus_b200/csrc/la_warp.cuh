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
    // right-looking Cholesky; lane owns rows lane, lane + 32.  One reciprocal
    // square root per pivot: d = s * rsqrt(s), 1/d = rsqrt(s) (a serial
    // chain of 2R FP64 divides and square roots costs more otherwise).
    for (int j = 0; j < R; ++j) {
        Real inv = 0;
        if (lane == (j & 31)) {
            Real sj = A[j * LDA + j];
            if (sj < (Real)0) sj = 0;
            const Real rs = sj > (Real)0 ? rsqrt(sj) : (Real)0;
            A[j * LDA + j] = sj * rs;
            inv = rs;
            invd[j] = rs;
        }
        inv = __shfl_sync(0xffffffffu, inv, j & 31);
        for (int i = j + 1 + ((lane - j - 1) & 31); i < R; i += 32) A[i * LDA + j] *= inv;
        __syncwarp();
        for (int i = j + 1 + ((lane - j - 1) & 31); i < R; i += 32) {
            const Real aij = A[i * LDA + j];
            for (int k = j + 1; k <= i; ++k) A[i * LDA + k] -= aij * A[k * LDA + j];
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

}  // namespace dgpu
