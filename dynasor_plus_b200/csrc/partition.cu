// ============================================================================
//  partition.cu -- the device remap: a stable counting sort over work tiles.
//
//  The reference remaps mode n's slab for mode n+1 with per-(thread, next
//  shard) cursors that each thread bumps while it walks its LPT shard list
//  (src/dynasor_kernel.cpp:220-227, cursor table src/dynasor_preprocess.cpp:
//  439-462).  The resulting permutation is a STABLE counting sort, keyed by
//  the next-mode shard id, of the processing sequence
//      concat_{tid} concat_{shard in ss_list[n][tid]} [shard_begin, shard_end).
//  This file computes the same permutation with three bandwidth-bound
//  kernels over tiles of that sequence (tiles listed in processing order):
//
//    1. k_part_hist    per-tile bucket histogram -> cnt
//    2. k_scan_*       exclusive scan of cnt -> off (global slot of the first
//                      element of bucket b in tile t)
//    3. k_part_scatter stable in-tile ranking (warp match + per-warp
//                      counters) and the scatter of (val, idx[0..N-1]).
//
//  cnt layout: entry (t, b) lives at seg_first(t) * nb + b * nt_seg(t) +
//  (t - seg_first(t)).  A global partition has one segment (seg_first = 0,
//  nt_seg = ntiles): bucket-major, tile-minor.  A segmented partition
//  (every super-shard sorted independently inside its own slab range, the
//  fiber sort) has one block per shard, bucket-major inside it; since the
//  shards' tiles are listed in slab order one flat scan yields the offsets
//  of every segment at once.
//
//  Keys wider than kMaxBuckets are sorted by least-significant-digit
//  passes; a stable LSD sort gives the same permutation as one stable
//  counting sort on the full key.  The same machinery builds the initial
//  mode-0 shard order (src/dynasor_preprocess.cpp:113-241) and the fiber
//  sort: a stable per-shard counting sort by row (src/dynasor_preprocess.cpp:
//  471-521, 2225-2256), keyed by the row's low bits (row - shard base).
// ============================================================================
#include "dgpu_internal.h"

#include <algorithm>

namespace dgpu {

namespace {

constexpr int kPartThreads = 256;
constexpr int kPartWarps = kPartThreads / 32;
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 16;
constexpr uint32_t kScanChunk = kScanThreads * kScanItems;   // entries per block

__device__ __forceinline__ uint32_t part_key(uint32_t v, int shift, uint32_t mask) {
    return (v >> shift) & mask;
}

// (segment base, tiles in segment) of tile t
__device__ __forceinline__ void seg_of(const Tile& tl, uint32_t t, uint32_t ntiles,
                                       const uint32_t* seg_n, uint32_t* first, uint32_t* nt) {
    if (seg_n) {
        *first = tl.seg_first;
        *nt = seg_n[tl.shard];
    } else {
        *first = 0;
        *nt = ntiles;
    }
    (void)t;
}

__global__ void __launch_bounds__(kPartThreads)
k_part_hist(const uint32_t* __restrict__ keycol, const Tile* __restrict__ tiles,
            uint32_t ntiles, const uint32_t* __restrict__ seg_n, int shift, uint32_t mask,
            uint32_t nb, uint32_t* __restrict__ cnt)
{
    extern __shared__ uint32_t h[];
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const uint32_t t = blockIdx.x;
    const Tile tl = tiles[t];
    const uint32_t* k = keycol + tl.begin;
    for (uint32_t j = threadIdx.x; j < tl.count; j += blockDim.x)
        atomicAdd(&h[part_key(__ldg(k + j), shift, mask)], 1u);
    __syncthreads();
    uint32_t first, nt;
    seg_of(tl, t, ntiles, seg_n, &first, &nt);
    uint32_t* c = cnt + (size_t)first * nb + (t - first);
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) c[(size_t)b * nt] = h[b];
}

// --- exclusive scan (three phases, u32) ----------------------------------
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sh,
                                                         uint32_t* total)
{
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
    const uint32_t warp_prefix = warp ? sh[warp - 1] : 0u;
    if (total) *total = sh[(blockDim.x >> 5) - 1];
    const uint32_t r = warp_prefix + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_reduce(const uint32_t* __restrict__ in, size_t n, uint32_t* __restrict__ aux)
{
    __shared__ uint32_t sh[32];
    const size_t base = (size_t)blockIdx.x * kScanChunk;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const size_t j = base + (size_t)i * kScanThreads + threadIdx.x;
        if (j < n) s += in[j];
    }
    uint32_t tot;
    block_exclusive_scan(s, sh, &tot);
    if (threadIdx.x == 0) aux[blockIdx.x] = tot;
}

// Single-block exclusive scan of the block sums (nblk <= kScanChunk).
__global__ void __launch_bounds__(kScanThreads)
k_scan_aux(uint32_t* aux, uint32_t nblk, uint32_t base)
{
    __shared__ uint32_t sh[32];
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint32_t j = threadIdx.x * kScanItems + i;
        v[i] = j < nblk ? aux[j] : 0u;
        s += v[i];
    }
    uint32_t pre = block_exclusive_scan(s, sh, nullptr) + base;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint32_t j = threadIdx.x * kScanItems + i;
        if (j < nblk) aux[j] = pre;
        pre += v[i];
    }
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_down(const uint32_t* __restrict__ in, size_t n, const uint32_t* __restrict__ aux,
            uint32_t* __restrict__ out)
{
    __shared__ uint32_t sh[32];
    // Each thread scans kScanItems consecutive entries of the block chunk.
    const size_t base = (size_t)blockIdx.x * kScanChunk + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const size_t j = base + i;
        v[i] = j < n ? in[j] : 0u;
        s += v[i];
    }
    uint32_t pre = block_exclusive_scan(s, sh, nullptr) + aux[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const size_t j = base + i;
        if (j < n) out[j] = pre;
        pre += v[i];
    }
}

// --- stable scatter ----------------------------------------------------------
// One CTA per tile.  Warp w owns the w-th contiguous eighth of the tile, so
// tile order = warp order = lane order within a 32-element step.  Per-warp
// counters are 16-bit (a warp handles at most kTile / 8 elements).
template <int N>
__global__ void __launch_bounds__(kPartThreads)
k_part_scatter(const __grid_constant__ SlabPtrs in, const __grid_constant__ SlabOut out,
               const Tile* __restrict__ tiles, uint32_t ntiles, const uint32_t* __restrict__ seg_n,
               const uint32_t* __restrict__ off, int key_mode, int shift, uint32_t mask,
               uint32_t nb)
{
    extern __shared__ uint32_t wcnt[];   // [kPartWarps][nb] running slots
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t i = threadIdx.x; i < kPartWarps * nb; i += blockDim.x) wcnt[i] = 0;
    __syncthreads();

    const uint32_t t = blockIdx.x;
    const Tile tl = tiles[t];
    const uint32_t per = (tl.count + kPartWarps - 1) / kPartWarps;
    const uint32_t wb = min(tl.count, (uint32_t)warp * per);
    const uint32_t we = min(tl.count, wb + per);
    const uint32_t* kc = in.idx[key_mode] + tl.begin;
    uint32_t* my = wcnt + (size_t)warp * nb;

    for (uint32_t j = wb + lane; j < we; j += 32)
        atomicAdd(&my[part_key(__ldg(kc + j), shift, mask)], 1u);
    __syncthreads();

    uint32_t first, nt;
    seg_of(tl, t, ntiles, seg_n, &first, &nt);
    const uint32_t* o = off + (size_t)first * nb + (t - first);
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
        uint32_t run = o[(size_t)b * nt];
#pragma unroll
        for (int w = 0; w < kPartWarps; ++w) {
            const uint32_t c = wcnt[(size_t)w * nb + b];
            wcnt[(size_t)w * nb + b] = run;
            run += c;
        }
    }
    __syncthreads();

    const unsigned lt = (1u << lane) - 1u;
    for (uint32_t s = wb; s < we; s += 32) {
        const uint32_t j = s + lane;
        const bool act = j < we;
        const unsigned am = __ballot_sync(0xffffffffu, act);
        if (act) {
            const uint32_t src = tl.begin + j;
            const uint32_t key = part_key(__ldg(kc + j), shift, mask);
            const unsigned peers = __match_any_sync(am, key);
            const uint32_t rank = __popc(peers & lt);
            const uint32_t start = my[key];
            __syncwarp(am);
            if (rank == 0) my[key] = start + __popc(peers);
            const uint32_t dst = start + rank;
            out.vals[dst] = __ldg(in.vals + src);
#pragma unroll
            for (int w = 0; w < N; ++w) out.idx[w][dst] = __ldg(in.idx[w] + src);
        }
        __syncwarp();
    }
}

int ensure_part_scratch(Plan& p, size_t entries) {
    if (entries <= p.part_cap) return DGPU_OK;
    dev_free(p.part_cnt);
    dev_free(p.part_off);
    dev_free(p.scan_aux);
    p.part_cnt = p.part_off = p.scan_aux = nullptr;
    p.part_cap = 0;
    DGPU_TRY(dev_alloc(p, (void**)&p.part_cnt, entries * sizeof(uint32_t)));
    DGPU_TRY(dev_alloc(p, (void**)&p.part_off, entries * sizeof(uint32_t)));
    const size_t nblk = (entries + kScanChunk - 1) / kScanChunk;
    DGPU_TRY(dev_alloc(p, (void**)&p.scan_aux, (nblk + 1) * sizeof(uint32_t)));
    p.part_cap = entries;
    return DGPU_OK;
}

int exclusive_scan(Plan& p, const uint32_t* in, size_t n, uint32_t* out, uint32_t base) {
    const size_t nblk = (n + kScanChunk - 1) / kScanChunk;
    if (nblk > kScanChunk) {
        set_error("exclusive_scan: %zu entries exceed the scan capacity", n);
        return DGPU_ERR_ARG;
    }
    k_scan_reduce<<<(unsigned)nblk, kScanThreads, 0, p.stream>>>(in, n, p.scan_aux);
    k_scan_aux<<<1, kScanThreads, 0, p.stream>>>(p.scan_aux, (uint32_t)nblk, base);
    k_scan_down<<<(unsigned)nblk, kScanThreads, 0, p.stream>>>(in, n, p.scan_aux, out);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

template <int N>
int launch_scatter(Plan& p, const Slab& in, const Slab& out, const Tile* tiles, uint32_t ntiles,
                   const uint32_t* seg_n, int key_mode, int key_shift, uint32_t key_mask,
                   uint32_t nb)
{
    static bool attr_set = false;
    if (!attr_set) {
        DGPU_CUDA(cudaFuncSetAttribute(k_part_scatter<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(kPartWarps * kMaxBuckets * sizeof(uint32_t))));
        attr_set = true;
    }
    const size_t ssm = (size_t)kPartWarps * nb * sizeof(uint32_t);
    k_part_scatter<N><<<ntiles, kPartThreads, ssm, p.stream>>>(
        slab_in(in, p.N), slab_out(out, p.N), tiles, ntiles, seg_n, p.part_off, key_mode,
        key_shift, key_mask, nb);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

}  // namespace

int stable_partition(Plan& p, const Slab& in, const Tile* tiles, uint32_t ntiles,
                     int key_mode, int key_shift, uint32_t key_mask, uint32_t nb,
                     const Slab& out, const uint32_t* seg_n)
{
    if (ntiles == 0) return DGPU_OK;
    if (nb == 0 || nb > kMaxBuckets) {
        set_error("stable_partition: %u buckets (max %u)", nb, kMaxBuckets);
        return DGPU_ERR_ARG;
    }
    const size_t entries = (size_t)nb * ntiles;
    DGPU_TRY(ensure_part_scratch(p, entries));
    const double elem = (double)p.nnz;
    const double row_bytes = 4.0 + 4.0 * p.N;
    {
        LaunchTimer t(p, KK_PART_HIST, elem * 4.0 + (double)entries * 4.0);
        const size_t hsm = nb * sizeof(uint32_t);
        k_part_hist<<<ntiles, kPartThreads, hsm, p.stream>>>(in.idx[key_mode], tiles, ntiles, seg_n,
                                                             key_shift, key_mask, nb, p.part_cnt);
        DGPU_CUDA(cudaGetLastError());
    }
    {
        LaunchTimer t(p, KK_PART_SCAN, (double)entries * 8.0);
        DGPU_TRY(exclusive_scan(p, p.part_cnt, entries, p.part_off, 0u));
    }
    {
        LaunchTimer t(p, KK_PART_SCATTER, elem * 2.0 * row_bytes + (double)entries * 4.0);
        switch (p.N) {
#define DGPU_SC(NN) case NN: return launch_scatter<NN>(p, in, out, tiles, ntiles, seg_n, key_mode, \
                                                    key_shift, key_mask, nb)
            DGPU_SC(2); DGPU_SC(3); DGPU_SC(4); DGPU_SC(5); DGPU_SC(6); DGPU_SC(7); DGPU_SC(8);
#undef DGPU_SC
            default:
                set_error("stable_partition: %d modes unsupported", p.N);
                return DGPU_ERR_ARG;
        }
    }
}

int stable_sort_pingpong(Plan& p, int a, int b, const Tile* tiles, uint32_t ntiles,
                         int key_mode, int key_shift, uint64_t key_limit, int* result)
{
    int bits = 0;
    while (bits < 32 && ((uint64_t)1 << bits) < key_limit) ++bits;
    if (key_limit <= 1) bits = 1;
    int passes = (bits + kDigitBits - 1) / kDigitBits;
    if (passes < 1) passes = 1;
    const int dbits = (bits + passes - 1) / passes;
    int src = a, dst = b;
    for (int k = 0; k < passes; ++k) {
        const int sh = key_shift + k * dbits;
        uint32_t nb, mask;
        if (passes == 1) {
            nb = (uint32_t)key_limit;
            mask = 0xffffffffu;
        } else {
            mask = (1u << dbits) - 1u;
            const uint64_t top = (key_limit - 1) >> (k * dbits);
            nb = (uint32_t)std::min<uint64_t>((uint64_t)mask + 1, top + 1);
        }
        const Tile* tl = (k == 0) ? tiles : p.ident_tiles_d;
        const uint32_t nt = (k == 0) ? ntiles : p.n_ident_tiles;
        DGPU_TRY(stable_partition(p, p.slab[src], tl, nt, key_mode, sh, mask, nb, p.slab[dst]));
        std::swap(src, dst);
    }
    *result = src;
    return DGPU_OK;
}

// Per-shard stable sort of mode n's slab by row: segmented LSD passes over
// the row's low shift_n bits (the row's offset inside its shard).
int fiber_sort(Plan& p, int n, int src, int other, int* result) {
    const int bits = p.shift[n];
    *result = src;
    if (bits == 0) return DGPU_OK;               // one row per shard: already sorted
    if (!p.ftiles_d[n]) {
        set_error("fiber_sort: mode %d has no fiber tiles", n);
        return DGPU_ERR_NOT_BUILT;
    }
    const int passes = (bits + kDigitBits - 1) / kDigitBits;
    const int dbits = (bits + passes - 1) / passes;
    int a = src, b = other;
    for (int k = 0; k < passes; ++k) {
        const int sh = k * dbits;
        const int hi = std::min(bits, sh + dbits);
        const uint32_t mask = (1u << (hi - sh)) - 1u;
        DGPU_TRY(stable_partition(p, p.slab[a], p.ftiles_d[n], p.nftiles[n], n, sh, mask, mask + 1,
                                  p.slab[b], p.fseg_d[n]));
        std::swap(a, b);
    }
    *result = a;
    return DGPU_OK;
}

}  // namespace dgpu
