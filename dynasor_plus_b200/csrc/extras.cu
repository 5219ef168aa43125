// ============================================================================
//  extras.cu -- all-modes (Jacobi) MTTKRP, CP model values at the nonzeros,
//  and the remaining C-ABI wrappers.
//
//  All-modes MTTKRP (replaces spmttkrp_all_modes_dynasor, src/dynasor.cpp:
//  592-817, kernel src/dynasor_kernel.cpp:830-1039): one pass over the slab
//  computes every Yhat[n] from the same factor snapshot.  Per nonzero the
//  N outputs use prefix/suffix products of the gathered rows, as the
//  reference does; instead of per-thread private output copies plus a
//  reduction (the reference's "ofibs"), partial rows are added to Yhat with
//  vector atomics in L2.
// ============================================================================
#include "dgpu_internal.h"

#include <cstring>

#include <algorithm>
#include <vector>

namespace dgpu {

int cpopt_gradient(Plan& p, float* const* grad_host);
int cp_tensor_norm(Plan& p, const float* vals, double* out);

namespace {

constexpr int kThreads = 256;

struct FacPtrs32 {
    const float* Y[kMaxModes];
};

// Where a nonzero's value and indices come from: the SoA slab, or a Morton
// key decoded in registers (pext of the key by each mode's mask,
// src/dynasor_morton.cpp:466-470).
struct SoaSrc {
    SlabPtrs s;
    template <int N>
    __device__ __forceinline__ float load(uint64_t i, uint32_t (&id)[N]) const {
#pragma unroll
        for (int w = 0; w < N; ++w) id[w] = __ldg(s.idx[w] + i);
        return __ldg(s.vals + i);
    }
};
struct MortonSrc {
    const uint64_t* keys;
    const float*    vals;
    MortonDec       d;
    template <int N>
    __device__ __forceinline__ float load(uint64_t i, uint32_t (&id)[N]) const {
        const uint64_t k = __ldg(keys + i);
#pragma unroll
        for (int w = 0; w < N; ++w) {
            uint32_t x = 0;
            for (int j = 0; j < d.bits[w]; ++j) x |= (uint32_t)((k >> d.pos[w][j]) & 1u) << j;
            id[w] = x;
        }
        return __ldg(vals + i);
    }
};

template <int N, int G, int V, class Src>
__global__ void __launch_bounds__(kThreads)
k_mttkrp_all(const __grid_constant__ Src in, uint64_t nnz, const __grid_constant__ FacPtrs32 F, float* Yh0, float* Yh1, float* Yh2, float* Yh3, float* Yh4, float* Yh5, float* Yh6,
             float* Yh7, int Rp)
{
    float* Yh[8] = {Yh0, Yh1, Yh2, Yh3, Yh4, Yh5, Yh6, Yh7};
    const int gl = threadIdx.x % G;
    const int C4 = Rp >> 2;
    const uint64_t groups = (uint64_t)gridDim.x * (kThreads / G);
    for (uint64_t i = (uint64_t)blockIdx.x * (kThreads / G) + threadIdx.x / G; i < nnz; i += groups) {
        uint32_t id[N];
        const float v = in.template load<N>(i, id);
#pragma unroll
        for (int q = 0; q < V; ++q) {
            const int c4 = gl + q * G;
            if (V > 1 && c4 >= C4) continue;
            float4 y[N];
#pragma unroll
            for (int w = 0; w < N; ++w)
                y[w] = __ldg(reinterpret_cast<const float4*>(F.Y[w] + (size_t)id[w] * Rp) + c4);
            // prefix[w] = prod_{u<w} y[u], suffix[w] = prod_{u>w} y[u]
            float4 pre[N], suf[N];
            pre[0] = make_float4(v, v, v, v);
#pragma unroll
            for (int w = 1; w < N; ++w)
                pre[w] = make_float4(pre[w - 1].x * y[w - 1].x, pre[w - 1].y * y[w - 1].y,
                                     pre[w - 1].z * y[w - 1].z, pre[w - 1].w * y[w - 1].w);
            suf[N - 1] = make_float4(1.f, 1.f, 1.f, 1.f);
#pragma unroll
            for (int w = N - 2; w >= 0; --w)
                suf[w] = make_float4(suf[w + 1].x * y[w + 1].x, suf[w + 1].y * y[w + 1].y,
                                     suf[w + 1].z * y[w + 1].z, suf[w + 1].w * y[w + 1].w);
#pragma unroll
            for (int w = 0; w < N; ++w) {
                const float4 o = make_float4(pre[w].x * suf[w].x, pre[w].y * suf[w].y,
                                             pre[w].z * suf[w].z, pre[w].w * suf[w].w);
                atomicAdd(reinterpret_cast<float4*>(Yh[w] + (size_t)id[w] * Rp) + c4, o);
            }
        }
    }
}

// model[i] = sum_r prod_w Y[w][i_w, r]  (one lane group per nonzero)
template <int N, int G, int V, class Src>
__global__ void __launch_bounds__(kThreads)
k_model_values(const __grid_constant__ Src in, uint64_t nnz, const __grid_constant__ FacPtrs32 F, int Rp, float* __restrict__ out)
{
    const int gl = threadIdx.x % G;
    const int C4 = Rp >> 2;
    const uint64_t groups = (uint64_t)gridDim.x * (kThreads / G);
    // all groups in a warp run the same trip count so the shuffles below
    // see full warps
    const uint64_t warp_first =
        (uint64_t)blockIdx.x * (kThreads / G) + (threadIdx.x / 32) * (32 / G);
    for (uint64_t base = warp_first; base < nnz; base += groups) {
        const uint64_t i = base + (threadIdx.x % 32) / G;
        const bool ok = i < nnz;
        float s = 0.f;
        if (ok) {
            uint32_t id[N];
            in.template load<N>(i, id);
#pragma unroll
            for (int q = 0; q < V; ++q) {
                const int c4 = gl + q * G;
                if (V > 1 && c4 >= C4) continue;
                float4 pr = make_float4(1.f, 1.f, 1.f, 1.f);
#pragma unroll
                for (int w = 0; w < N; ++w) {
                    const float4 y = __ldg(reinterpret_cast<const float4*>(F.Y[w] + (size_t)id[w] * Rp) + c4);
                    pr = make_float4(pr.x * y.x, pr.y * y.y, pr.z * y.z, pr.w * y.w);
                }
                s += (pr.x + pr.y) + (pr.z + pr.w);
            }
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (ok && gl == 0) out[i] = s;
    }
}

unsigned grid_groups(uint64_t nnz, int G) {
    const uint64_t per_block = kThreads / G;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((nnz + per_block - 1) / per_block,
                                                             148ull * 16));
}

template <int N, class Src>
int all_modes_n(Plan& p, const Src& sp) {
    FacPtrs32 F{};
    for (int w = 0; w < N; ++w) F.Y[w] = p.Y[w];
    float* Yh[8] = {nullptr};
    for (int w = 0; w < N; ++w) Yh[w] = p.Yhat[w];
    const int C4 = p.Rp / 4;
#define LAUNCH(G, V)                                                                        \
    k_mttkrp_all<N, G, V, Src><<<grid_groups(p.nnz, G), kThreads, 0, p.stream>>>(          \
        sp, p.nnz, F, Yh[0], Yh[1], Yh[2], Yh[3], Yh[4], Yh[5], Yh[6], Yh[7], p.Rp)
    if (C4 == 4) LAUNCH(4, 1);
    else if (C4 == 8) LAUNCH(8, 1);
    else if (C4 == 16) LAUNCH(16, 1);
    else if (C4 == 32) LAUNCH(32, 1);
    else if (C4 <= 64) LAUNCH(32, 2);
    else if (C4 <= 128) LAUNCH(32, 4);
    else if (C4 <= 256) LAUNCH(32, 8);
    else { set_error("all-modes: rank_padded %d too large", p.Rp); return DGPU_ERR_ARG; }
#undef LAUNCH
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

template <int N, class Src>
int model_values_n(Plan& p, const Src& sp, float* out) {
    FacPtrs32 F{};
    for (int w = 0; w < N; ++w) F.Y[w] = p.Y[w];
    const int C4 = p.Rp / 4;
#define LAUNCH(G, V) \
    k_model_values<N, G, V, Src><<<grid_groups(p.nnz, G), kThreads, 0, p.stream>>>(sp, p.nnz, F, p.Rp, out)
    if (C4 == 4) LAUNCH(4, 1);
    else if (C4 == 8) LAUNCH(8, 1);
    else if (C4 == 16) LAUNCH(16, 1);
    else if (C4 == 32) LAUNCH(32, 1);
    else if (C4 <= 64) LAUNCH(32, 2);
    else if (C4 <= 128) LAUNCH(32, 4);
    else if (C4 <= 256) LAUNCH(32, 8);
    else { set_error("model_values: rank_padded %d too large", p.Rp); return DGPU_ERR_ARG; }
#undef LAUNCH
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

template <typename Fn>
int by_modes(int N, Fn&& f) {
    switch (N) {
        case 2: return f(std::integral_constant<int, 2>{});
        case 3: return f(std::integral_constant<int, 3>{});
        case 4: return f(std::integral_constant<int, 4>{});
        case 5: return f(std::integral_constant<int, 5>{});
        case 6: return f(std::integral_constant<int, 6>{});
        case 7: return f(std::integral_constant<int, 7>{});
        case 8: return f(std::integral_constant<int, 8>{});
        default: set_error("unsupported mode count %d", N); return DGPU_ERR_ARG;
    }
}

const Slab& live_slab(const Plan& p) {
    return (p.layout == DGPU_LAYOUT_NCOPY) ? p.slab[0] : p.slab[p.cur];
}

}  // namespace

const float* live_vals(const Plan& p) {
    return p.layout == DGPU_LAYOUT_MORTON ? p.mvals : live_slab(p).vals;
}

int launch_mttkrp_all_modes(Plan& p) {
    for (int n = 0; n < p.N; ++n)
        DGPU_CUDA(cudaMemsetAsync(p.Yhat[n], 0, (size_t)p.dims[n] * p.Rp * sizeof(float), p.stream));
    if (p.layout == DGPU_LAYOUT_MORTON) {
        const MortonSrc src{p.mkeys, p.mvals, morton_decoder(p)};
        return by_modes(p.N, [&](auto NC) { return all_modes_n<decltype(NC)::value>(p, src); });
    }
    const SoaSrc src{slab_in(live_slab(p), p.N)};
    return by_modes(p.N, [&](auto NC) { return all_modes_n<decltype(NC)::value>(p, src); });
}

int launch_model_values(Plan& p, float* out) {
    if (p.layout == DGPU_LAYOUT_MORTON) {
        const MortonSrc src{p.mkeys, p.mvals, morton_decoder(p)};
        return by_modes(p.N, [&](auto NC) { return model_values_n<decltype(NC)::value>(p, src, out); });
    }
    const SoaSrc src{slab_in(live_slab(p), p.N)};
    return by_modes(p.N, [&](auto NC) { return model_values_n<decltype(NC)::value>(p, src, out); });
}

// Bytes from device memory to host memory the caller may not have pinned,
// through the plan's two pinned chunks: the GPU copies chunk k+1 while the
// host moves chunk k out (pageable copies otherwise run at a few GB/s).
int copy_to_host_staged(Plan& p, void* host, const void* dev, size_t bytes) {
    constexpr size_t kChunk = (size_t)8 << 20;
    if (bytes == 0) return DGPU_OK;
    if (p.stage_cap < kChunk) {
        for (int k = 0; k < 2; ++k) {
            if (p.stage_host[k]) cudaFreeHost(p.stage_host[k]);
            p.stage_host[k] = nullptr;
        }
        p.stage_cap = 0;
        for (int k = 0; k < 2; ++k) {
            if (cudaMallocHost(&p.stage_host[k], kChunk) != cudaSuccess) {
                cudaGetLastError();
                set_error("copy to host: pinned staging of %zu bytes failed", kChunk);
                return DGPU_ERR_NOMEM;
            }
            if (!p.stage_ev[k])
                DGPU_CUDA(cudaEventCreateWithFlags(&p.stage_ev[k], cudaEventDisableTiming));
        }
        p.stage_cap = kChunk;
    }
    const char* src = static_cast<const char*>(dev);
    char* dst = static_cast<char*>(host);
    const size_t nchunks = (bytes + kChunk - 1) / kChunk;
    auto issue = [&](size_t k) -> int {
        const size_t off = k * kChunk, len = std::min(kChunk, bytes - off);
        DGPU_CUDA(cudaMemcpyAsync(p.stage_host[k & 1], src + off, len, cudaMemcpyDeviceToHost,
                                  p.stream));
        DGPU_CUDA(cudaEventRecord(p.stage_ev[k & 1], p.stream));
        return DGPU_OK;
    };
    DGPU_TRY(issue(0));
    for (size_t k = 0; k < nchunks; ++k) {
        if (k + 1 < nchunks) DGPU_TRY(issue(k + 1));      // the other chunk, while this one drains
        DGPU_CUDA(cudaEventSynchronize(p.stage_ev[k & 1]));
        const size_t off = k * kChunk, len = std::min(kChunk, bytes - off);
        std::memcpy(dst + off, p.stage_host[k & 1], len);
    }
    return sync_checked(p);
}

}  // namespace dgpu

using namespace dgpu;

extern "C" {

int dgpu_mttkrp_all_modes(dgpu_plan* plan) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    if (!p) { set_error("dgpu_mttkrp_all_modes: null plan"); return DGPU_ERR_ARG; }
    DGPU_CUDA(cudaSetDevice(p->device));
    return launch_mttkrp_all_modes(*p);
}

int dgpu_model_values(dgpu_plan* plan, float* model_host) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    if (!p || !model_host) { set_error("dgpu_model_values: null argument"); return DGPU_ERR_ARG; }
    DGPU_CUDA(cudaSetDevice(p->device));
    // the device buffer is kept on the plan for later calls
    if (p->model_cap < p->nnz) {
        dev_free(p->model_buf);
        p->model_buf = nullptr;
        p->model_cap = 0;
        DGPU_TRY(dev_alloc(*p, (void**)&p->model_buf, p->nnz * sizeof(float)));
        p->model_cap = p->nnz;
    }
    DGPU_TRY(launch_model_values(*p, p->model_buf));
    return copy_to_host_staged(*p, model_host, p->model_buf, p->nnz * sizeof(float));
}

int dgpu_cpopt_gradient(dgpu_plan* plan, float* const* grad_host) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    if (!p || !grad_host) { set_error("dgpu_cpopt_gradient: null argument"); return DGPU_ERR_ARG; }
    for (int n = 0; n < p->N; ++n)
        if (!grad_host[n]) { set_error("dgpu_cpopt_gradient: grad[%d] null", n); return DGPU_ERR_ARG; }
    DGPU_CUDA(cudaSetDevice(p->device));
    return cpopt_gradient(*p, grad_host);
}

int dgpu_tensor_norm_sq(dgpu_plan* plan, double* norm_sq) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    if (!p || !norm_sq) { set_error("dgpu_tensor_norm_sq: null argument"); return DGPU_ERR_ARG; }
    DGPU_CUDA(cudaSetDevice(p->device));
    return cp_tensor_norm(*p, live_vals(*p), norm_sq);
}

}  // extern "C"
