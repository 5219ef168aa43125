// ============================================================================
//  apply_map.cuh -- Y = Yhat * W for one or several column blocks, FP64 on
//  the FP64 tensor pipe.  Used by the CP-ALS factor update (one block of Rp
//  columns) and by the batched restarts (one block per restart).
// ============================================================================
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dgpu {

constexpr int kApplyThreads = 256;
constexpr int kMapRows = 8;                    // rows a warp stages at a time

// mma.sync m8n8k4 .f64 for blocks of RP in {16, 32} columns: a warp
// multiplies blocks of 8 rows, Y(8 x RP) = Yhat(8 x RP) * W(RP x RP), as
// RP/4 k-steps x RP/8 column tiles.  W's fragments stay in registers
// (thread (g, t) = (lane / 4, lane % 4) holds W[4s + t][8j + g]); the 8 rows
// are staged in a padded shared-memory slice (row stride RP + 4 floats: the
// A-fragment reads A[g][4s + t] fall in 32 distinct banks) and converted to
// FP64 on the way into the fragments.  The next block is loaded while the
// current one is multiplied.  Column block k = blockIdx.y starts at column
// k * RP of Yhat / Y (row stride ld floats) and uses W + k * w_stride, an
// R x R map (R <= RP; columns R..RP-1 are written as 0); blocks whose
// active[k] is 0 are left untouched.
template <int RP>
__global__ void __launch_bounds__(kApplyThreads, 2)
k_apply_map_dmma(const float* __restrict__ Yhat, uint32_t rows, int R, int ld,
                 const double* __restrict__ W, size_t w_stride, const int* __restrict__ active,
                 float* __restrict__ Y)
{
    static_assert(RP == 16 || RP == 32, "two or four column tiles");
    constexpr int NT = RP / 8, KS = RP / 4, LD = RP + 4;
    constexpr int V4 = kMapRows * RP / 4 / 32;            // float4 loads per lane per block
    __shared__ __align__(16) float hs[kApplyThreads / 32][kMapRows][LD];
    const int kb = blockIdx.y;
    if (active && !active[kb]) return;
    Yhat += (size_t)kb * RP;
    Y += (size_t)kb * RP;
    W += (size_t)kb * w_stride;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    double b[KS][NT];
#pragma unroll
    for (int ks = 0; ks < KS; ++ks)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const int k = 4 * ks + t, c = 8 * j + g;
            b[ks][j] = (k < R && c < R) ? W[(size_t)k * R + c] : 0.0;
        }
    const uint32_t nblocks = (rows + kMapRows - 1) / kMapRows;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    float4 pf[V4];
    auto load = [&](uint32_t blk) {
#pragma unroll
        for (int v = 0; v < V4; ++v) {
            const int e = (v * 32 + lane) * 4;
            const uint32_t i = blk * kMapRows + e / RP;
            pf[v] = i < rows ? __ldg(reinterpret_cast<const float4*>(Yhat + (size_t)i * ld + e % RP))
                             : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };
    uint32_t blk = gw;
    if (blk < nblocks) load(blk);
    for (; blk < nblocks; blk += nw) {
#pragma unroll
        for (int v = 0; v < V4; ++v) {
            const int e = (v * 32 + lane) * 4;
            *reinterpret_cast<float4*>(&hs[warp][e / RP][e % RP]) = pf[v];
        }
        __syncwarp();
        if (blk + nw < nblocks) load(blk + nw);
        double a[KS];
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) a[ks] = (double)hs[warp][g][4 * ks + t];
        double acc[NT][2];
#pragma unroll
        for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < KS; ++ks)
#pragma unroll
            for (int j = 0; j < NT; ++j)
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                             : "+d"(acc[j][0]), "+d"(acc[j][1]) : "d"(a[ks]), "d"(b[ks][j]));
        const uint32_t i = blk * kMapRows + g;
        if (i < rows) {
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const int c = 8 * j + 2 * t;
                float2 o;
                o.x = c < R ? (float)acc[j][0] : 0.f;
                o.y = c + 1 < R ? (float)acc[j][1] : 0.f;
                *reinterpret_cast<float2*>(Y + (size_t)i * ld + c) = o;
            }
        }
        __syncwarp();
    }
}

}  // namespace dgpu
