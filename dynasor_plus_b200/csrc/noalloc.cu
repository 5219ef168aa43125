// ============================================================================
//  noalloc.cu -- dgpu_sort_slab_noalloc: the stable shard partition (the
//  counting sort behind the device remap and the initial mode-0 order) for
//  callers that cannot allocate device memory.
//
//  Who needs it: code that runs where every byte of device memory is owned
//  by a host framework's pool allocator that must not be bypassed, and
//  latency-critical paths where cudaMalloc/cudaFree (which can synchronise
//  the whole device) are not allowed.  Such callers pass their own input
//  and output buffers; the per-(bucket, tile) counters, offsets and scan
//  block sums live in one fixed file-scope device array instead of plan
//  memory.
//
//  Limits and sharing:
//    * the scratch array is kScratchWords 32-bit words (16 MiB); it exists
//      on every GPU that loads this library until the process exits;
//    * a call needs num_buckets * ceil(nnz / 4096) <= kMaxEntries
//      (2,095,104) counter slots; larger requests are rejected with
//      DGPU_ERR_ARG before any work is queued;
//    * every call reuses the same array and leaves its contents behind; the
//      counters and offsets are fully rewritten by each call and the fault
//      flag is cleared at the start of each call;
//    * calls whose device work overlaps (different streams, or different
//      host threads on one device) race on the array: serialise them;
//    * the first call on a device looks up the array's device address
//      (cudaGetSymbolAddress with that device current) and caches it; make
//      that first call before any stream capture.  The cached address is
//      not looked up again, so cudaDeviceReset on that device after the
//      first call is not supported (the array would move with the new
//      context);
//    * the call waits for its own stream once at the end to read the fault
//      flag (keys >= num_buckets are reported, never written out of range),
//      so a call on a stream that is being captured is rejected with
//      DGPU_ERR_ARG before any work is queued.
//
//  The kernels below are separate copies specialised for an input taken in
//  slab order (tile t = [t*4096, ...)), so no tile table is needed.
// ============================================================================
#include "dgpu_internal.h"

#include <mutex>

namespace dgpu {
namespace {

constexpr uint32_t kNaTile = 4096;
constexpr int kNaThreads = 256;
constexpr int kNaWarps = kNaThreads / 32;
constexpr size_t kScratchWords = (size_t)4 << 20;         // 16 MiB
constexpr size_t kAuxWords = 4096;                         // scan block sums + flag
constexpr size_t kMaxEntries = (kScratchWords - kAuxWords) / 2;
constexpr int kScanT = 1024;
constexpr int kScanI = 16;
constexpr uint32_t kScanC = kScanT * kScanI;

// [0, kMaxEntries)              per-(bucket, tile) counts
// [kMaxEntries, 2*kMaxEntries)  their exclusive scan (global slots)
// [2*kMaxEntries, +kAuxWords)   scan block sums; the last word is the fault flag
static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

__global__ void __launch_bounds__(kNaThreads)
k_na_hist(const uint32_t* __restrict__ keycol, uint64_t nnz, uint32_t ntiles, int shift,
          uint32_t nb, uint32_t* __restrict__ cnt, uint32_t* __restrict__ flag)
{
    extern __shared__ uint32_t h[];
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const uint64_t begin = (uint64_t)blockIdx.x * kNaTile;
    const uint64_t rem = nnz - begin;
    const uint32_t count = rem < kNaTile ? (uint32_t)rem : kNaTile;
    for (uint32_t j = threadIdx.x; j < count; j += blockDim.x) {
        const uint32_t k = __ldg(keycol + begin + j) >> shift;
        if (k < nb) atomicAdd(&h[k], 1u);
        else atomicExch(flag, 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x)
        cnt[(size_t)b * ntiles + blockIdx.x] = h[b];
}

__device__ __forceinline__ uint32_t na_block_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t s = lane < nw ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    const uint32_t r = (warp ? sh[warp - 1] : 0u) + x - v;
    if (total) *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanT)
k_na_scan_reduce(const uint32_t* __restrict__ in, size_t n, uint32_t* __restrict__ aux) {
    __shared__ uint32_t sh[32];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanI; ++i) {
        const size_t j = (size_t)blockIdx.x * kScanC + (size_t)i * kScanT + threadIdx.x;
        if (j < n) s += in[j];
    }
    uint32_t tot;
    na_block_scan(s, sh, &tot);
    if (threadIdx.x == 0) aux[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanT)
k_na_scan_aux(uint32_t* aux, uint32_t nblk) {
    __shared__ uint32_t sh[32];
    uint32_t v[kScanI];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanI; ++i) {
        const uint32_t j = threadIdx.x * kScanI + i;
        v[i] = j < nblk ? aux[j] : 0u;
        s += v[i];
    }
    uint32_t pre = na_block_scan(s, sh, nullptr);
#pragma unroll
    for (int i = 0; i < kScanI; ++i) {
        const uint32_t j = threadIdx.x * kScanI + i;
        if (j < nblk) aux[j] = pre;
        pre += v[i];
    }
}

__global__ void __launch_bounds__(kScanT)
k_na_scan_down(const uint32_t* __restrict__ in, size_t n, const uint32_t* __restrict__ aux,
               uint32_t* __restrict__ out) {
    __shared__ uint32_t sh[32];
    const size_t base = (size_t)blockIdx.x * kScanC + (size_t)threadIdx.x * kScanI;
    uint32_t v[kScanI];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanI; ++i) {
        v[i] = (base + i) < n ? in[base + i] : 0u;
        s += v[i];
    }
    uint32_t pre = na_block_scan(s, sh, nullptr) + aux[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanI; ++i) {
        if (base + i < n) out[base + i] = pre;
        pre += v[i];
    }
}

template <int N>
__global__ void __launch_bounds__(kNaThreads)
k_na_scatter(const __grid_constant__ SlabPtrs in, const __grid_constant__ SlabOut out,
             uint64_t nnz, uint32_t ntiles, const uint32_t* __restrict__ off, int key_mode,
             int shift, uint32_t nb)
{
    extern __shared__ uint32_t wcnt[];   // [kNaWarps][nb]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t i = threadIdx.x; i < kNaWarps * nb; i += blockDim.x) wcnt[i] = 0;
    __syncthreads();
    const uint64_t begin = (uint64_t)blockIdx.x * kNaTile;
    const uint64_t rem = nnz - begin;
    const uint32_t count = rem < kNaTile ? (uint32_t)rem : kNaTile;
    const uint32_t per = (count + kNaWarps - 1) / kNaWarps;
    const uint32_t wb = min(count, (uint32_t)warp * per);
    const uint32_t we = min(count, wb + per);
    const uint32_t* kc = in.idx[key_mode] + begin;
    uint32_t* my = wcnt + (size_t)warp * nb;
    for (uint32_t j = wb + lane; j < we; j += 32) {
        const uint32_t k = __ldg(kc + j) >> shift;
        if (k < nb) atomicAdd(&my[k], 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
        uint32_t run = off[(size_t)b * ntiles + blockIdx.x];
        for (int w = 0; w < kNaWarps; ++w) {
            const uint32_t c = wcnt[(size_t)w * nb + b];
            wcnt[(size_t)w * nb + b] = run;
            run += c;
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    for (uint32_t s = wb; s < we; s += 32) {
        const uint32_t j = s + lane;
        const uint32_t key = j < we ? (__ldg(kc + j) >> shift) : nb;
        const bool act = key < nb;                 // out-of-range keys are skipped
        const unsigned am = __ballot_sync(0xffffffffu, act);
        if (act) {
            const unsigned peers = __match_any_sync(am, key);
            const uint32_t rank = __popc(peers & lt);
            const uint32_t start = my[key];
            __syncwarp(am);
            if (rank == 0) my[key] = start + __popc(peers);
            const uint32_t dst = start + rank;
            const uint64_t src = begin + j;
            out.vals[dst] = __ldg(in.vals + src);
#pragma unroll
            for (int w = 0; w < N; ++w) out.idx[w][dst] = __ldg(in.idx[w] + src);
        }
        __syncwarp();
    }
}

std::mutex g_na_mutex;
uint32_t* g_na_ptr[64] = {nullptr};

int na_scratch(uint32_t** out) {
    int dev = 0;
    DGPU_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("dgpu_sort_slab_noalloc: device ordinal %d unsupported", dev);
        return DGPU_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void* ptr = nullptr;
        DGPU_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_na_ptr[dev] = static_cast<uint32_t*>(ptr);
    }
    *out = g_na_ptr[dev];
    return DGPU_OK;
}

template <int N>
int na_scatter(cudaStream_t st, const SlabPtrs& in, const SlabOut& out, uint64_t nnz,
               uint32_t ntiles, const uint32_t* off, int key_mode, int shift, uint32_t nb)
{
    const size_t sm = (size_t)kNaWarps * nb * sizeof(uint32_t);
    DGPU_CUDA(cudaFuncSetAttribute(k_na_scatter<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(kNaWarps * kMaxBuckets * sizeof(uint32_t))));
    k_na_scatter<N><<<ntiles, kNaThreads, sm, st>>>(in, out, nnz, ntiles, off, key_mode, shift, nb);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

extern "C" int dgpu_sort_slab_noalloc(void* stream, int num_modes, uint64_t nnz,
                                      const float* vals_in, const uint32_t* const* idx_in,
                                      float* vals_out, uint32_t* const* idx_out, int key_mode,
                                      int key_shift, uint32_t num_buckets)
{
    if (num_modes < 2 || num_modes > DGPU_MAX_MODES || !vals_in || !idx_in || !vals_out ||
        !idx_out || key_mode < 0 || key_mode >= num_modes || key_shift < 0 || key_shift > 31) {
        set_error("dgpu_sort_slab_noalloc: bad argument");
        return DGPU_ERR_ARG;
    }
    if (nnz == 0 || nnz >= 0xffffffffull) {
        set_error("dgpu_sort_slab_noalloc: nnz %llu outside [1, 2^32-1)", (unsigned long long)nnz);
        return DGPU_ERR_ARG;
    }
    if (num_buckets == 0 || num_buckets > kMaxBuckets) {
        set_error("dgpu_sort_slab_noalloc: %u buckets outside [1, %u]", num_buckets, kMaxBuckets);
        return DGPU_ERR_ARG;
    }
    const uint32_t ntiles = (uint32_t)((nnz + kNaTile - 1) / kNaTile);
    const size_t entries = (size_t)num_buckets * ntiles;
    if (entries > kMaxEntries) {
        set_error("dgpu_sort_slab_noalloc: buckets x tiles = %u x %u exceeds the fixed scratch "
                  "of %zu counters (16 MiB); use the plan API for this size",
                  num_buckets, ntiles, kMaxEntries);
        return DGPU_ERR_ARG;
    }
    SlabPtrs in{};
    SlabOut out{};
    in.vals = vals_in;
    out.vals = vals_out;
    for (int n = 0; n < num_modes; ++n) {
        if (!idx_in[n] || !idx_out[n]) {
            set_error("dgpu_sort_slab_noalloc: idx[%d] is null", n);
            return DGPU_ERR_ARG;
        }
        in.idx[n] = idx_in[n];
        out.idx[n] = idx_out[n];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the call ends with a blocking read of the fault flag, which a stream
    // capture cannot hold
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    DGPU_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
        set_error("dgpu_sort_slab_noalloc: the stream is being captured; this call waits for "
                  "its stream and reads a status back, so call it outside a capture");
        return DGPU_ERR_ARG;
    }
    uint32_t* base = nullptr;
    DGPU_TRY(na_scratch(&base));
    uint32_t* cnt = base;
    uint32_t* off = base + kMaxEntries;
    uint32_t* aux = base + 2 * kMaxEntries;
    uint32_t* flag = aux + kAuxWords - 1;

    DGPU_CUDA(cudaMemsetAsync(flag, 0, sizeof(uint32_t), st));
    k_na_hist<<<ntiles, kNaThreads, num_buckets * sizeof(uint32_t), st>>>(
        in.idx[key_mode], nnz, ntiles, key_shift, num_buckets, cnt, flag);
    const uint32_t nblk = (uint32_t)((entries + kScanC - 1) / kScanC);
    k_na_scan_reduce<<<nblk, kScanT, 0, st>>>(cnt, entries, aux);
    k_na_scan_aux<<<1, kScanT, 0, st>>>(aux, nblk);
    k_na_scan_down<<<nblk, kScanT, 0, st>>>(cnt, entries, aux, off);
    DGPU_CUDA(cudaGetLastError());
    int rc = DGPU_OK;
    switch (num_modes) {
#define NA_CASE(NN) case NN: rc = na_scatter<NN>(st, in, out, nnz, ntiles, off, key_mode, key_shift, num_buckets); break
        NA_CASE(2); NA_CASE(3); NA_CASE(4); NA_CASE(5); NA_CASE(6); NA_CASE(7); NA_CASE(8);
#undef NA_CASE
    }
    if (rc != DGPU_OK) return rc;
    uint32_t bad = 0;
    DGPU_CUDA(cudaMemcpyAsync(&bad, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DGPU_CUDA(cudaStreamSynchronize(st));
    if (bad) {
        set_error("dgpu_sort_slab_noalloc: a key (idx >> key_shift) is >= num_buckets; "
                  "those nonzeros were not written");
        return DGPU_ERR_INDEX;
    }
    return DGPU_OK;
}
