// ============================================================================
//  partition.cu -- the device remap: a chunked stable counting sort.
//
//  The reference remaps mode n's slab for mode n+1 with per-(thread, next
//  shard) cursors that each thread bumps while it walks its LPT shard list
//  (src/dynasor_kernel.cpp:220-227, cursor table src/dynasor_preprocess.cpp:
//  439-462).  The resulting permutation is a STABLE counting sort, keyed by
//  the next-mode shard id, of the processing sequence
//      concat_{tid} concat_{shard in ss_list[n][tid]} [shard_begin, shard_end).
//  The same machinery builds the initial mode-0 shard order (a stable sort of
//  the input order, src/dynasor_preprocess.cpp:113-241) and the fiber sort (a
//  stable per-shard sort by row, src/dynasor_preprocess.cpp:471-521,
//  2225-2256) -- the latter as a "segmented" sort with one segment per shard.
//
//  The sequence is a tile list (tiles of <= 4096 consecutive slab
//  positions, in sequence order) cut into chunks (runs of tiles inside one
//  segment; ~2 per SM for a global sort, <= 64K elements for a segmented
//  one).  Per pass:
//
//    k_chunk_hist   one CTA per chunk: bucket histogram  -> cnt[c][b]
//    k_col_scan     per (segment, bucket): exclusive prefix over the
//                   segment's chunks -> off[c][b]; segment totals -> base
//    k_bucket_scan  per segment: exclusive prefix over buckets + segment
//                   start -> base[s][b]
//    k_chunk_scatter one CTA per chunk, 512 threads: walks its tiles in
//                   windows of W elements; each warp ranks its 32-element
//                   steps with __match_any_sync and 16-bit per-warp bucket
//                   counters; the window is staged in shared memory in
//                   bucket order and written out so consecutive threads
//                   store consecutive slots of one bucket; running bucket
//                   cursors carry across windows.
//
//  Per-bucket metadata is per chunk (hundreds), not per tile, so it stays
//  small next to the 4+4N bytes per element that each pass reads and writes
//  once.  Keys wider than kMaxBuckets are sorted by least-significant-digit
//  passes; a stable LSD sort gives the permutation of one stable counting
//  sort on the full key.
// ============================================================================
#include "dgpu_internal.h"

#include <algorithm>

namespace dgpu {

namespace {

constexpr int kHistThreads = 256;
constexpr int kScatThreads = 512;
constexpr int kScatWarps = kScatThreads / 32;
constexpr uint32_t kSegChunkTiles = 16;       // <= 64K elements per segmented chunk

__device__ __forceinline__ uint32_t part_key(uint32_t v, int shift, uint32_t mask) {
    return (v >> shift) & mask;
}

__global__ void __launch_bounds__(kHistThreads)
k_chunk_hist(const uint32_t* __restrict__ keycol, const Tile* __restrict__ tiles,
             const Chunk* __restrict__ chunks, int shift, uint32_t mask, uint32_t nb,
             uint32_t* __restrict__ cnt)
{
    extern __shared__ uint32_t h[];
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const Chunk c = chunks[blockIdx.x];
    for (uint32_t t = c.tile_begin; t < c.tile_end; ++t) {
        const Tile tl = tiles[t];
        const uint32_t* k = keycol + tl.begin;
        for (uint32_t j = threadIdx.x; j < tl.count; j += blockDim.x)
            atomicAdd(&h[part_key(__ldg(k + j), shift, mask)], 1u);
    }
    __syncthreads();
    uint32_t* out = cnt + (size_t)blockIdx.x * nb;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) out[b] = h[b];
}

// grid (segments, ceil(nb/256)); thread = bucket.
__global__ void __launch_bounds__(256)
k_col_scan(const uint32_t* __restrict__ cnt, const Seg* __restrict__ segs, uint32_t nb,
           uint32_t* __restrict__ off, uint32_t* __restrict__ segtot)
{
    const uint32_t b = blockIdx.y * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const Seg s = segs[blockIdx.x];
    uint32_t run = 0;
    uint32_t c = s.chunk_begin;
    for (; c + 8 <= s.chunk_end; c += 8) {
        uint32_t v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = cnt[(size_t)(c + k) * nb + b];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            off[(size_t)(c + k) * nb + b] = run;
            run += v[k];
        }
    }
    for (; c < s.chunk_end; ++c) {
        const uint32_t v = cnt[(size_t)c * nb + b];
        off[(size_t)c * nb + b] = run;
        run += v;
    }
    segtot[(size_t)blockIdx.x * nb + b] = run;
}

// grid = segments, 1024 threads: base[s][b] = seg.base + sum_{b' < b} tot[s][b']
__global__ void __launch_bounds__(1024)
k_bucket_scan(uint32_t* __restrict__ tot_base, const Seg* __restrict__ segs, uint32_t nb)
{
    __shared__ uint32_t wsum[32];
    const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;     // <= 2 for nb <= 2048
    uint32_t* row = tot_base + (size_t)blockIdx.x * nb;
    const uint32_t b0 = threadIdx.x * per;
    uint32_t v[2] = {0u, 0u};
    uint32_t s = 0;
    for (uint32_t k = 0; k < per && k < 2; ++k) {
        v[k] = (b0 + k < nb) ? row[b0 + k] : 0u;
        s += v[k];
    }
    // block exclusive scan of s
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        wsum[lane] = w;
    }
    __syncthreads();
    uint32_t pre = segs[blockIdx.x].base + (warp ? wsum[warp - 1] : 0u) + x - s;
    for (uint32_t k = 0; k < per && k < 2; ++k) {
        if (b0 + k < nb) row[b0 + k] = pre;
        pre += v[k];
    }
}

// One CTA per chunk.  Window W elements; warp w owns [w*W/16, (w+1)*W/16)
// of each window; S = W/512 steps of 32 per warp.
template <int N, int W>
__global__ void __launch_bounds__(kScatThreads, 1)
k_chunk_scatter(const __grid_constant__ SlabPtrs in, const __grid_constant__ SlabOut out,
                const Tile* __restrict__ tiles, const Chunk* __restrict__ chunks,
                const uint32_t* __restrict__ off, const uint32_t* __restrict__ base,
                int key_mode, int shift, uint32_t mask, uint32_t nb)
{
    constexpr int S = W / kScatThreads;           // steps per warp per window
    constexpr int PW = W / kScatWarps;            // elements per warp per window
    extern __shared__ __align__(16) uint32_t sm[];
    uint32_t* cursor = sm;                                   // [nb]
    uint32_t* lbase = cursor + nb;                           // [nb]
    uint16_t* wc = reinterpret_cast<uint16_t*>(lbase + nb);  // [16][nb]
    uint32_t* stage = lbase + nb + ((size_t)kScatWarps * nb + 1) / 2;
    float* sv = reinterpret_cast<float*>(stage);             // [W]
    uint32_t* si = stage + W;                                // [N][W]
    uint32_t* sd = si + (size_t)N * W;                       // [W]

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const Chunk c = chunks[blockIdx.x];
    const uint32_t* o = off + (size_t)blockIdx.x * nb;
    const uint32_t* bs = base + (size_t)c.seg * nb;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) cursor[b] = o[b] + bs[b];
    for (uint32_t i = threadIdx.x; i < kScatWarps * nb; i += blockDim.x) wc[i] = 0;
    __syncthreads();

    uint16_t* mywc = wc + (size_t)warp * nb;
    for (uint32_t t = c.tile_begin; t < c.tile_end; ++t) {
        const Tile tl = tiles[t];
        for (uint32_t w0 = 0; w0 < tl.count; w0 += W) {
            const uint32_t cnt = min((uint32_t)W, tl.count - w0);
            const uint32_t src0 = tl.begin + w0;
            // a. load + rank
            uint32_t key[S], rk[S];
            float val[S];
            uint32_t id[S][N];
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const uint32_t j = warp * PW + s * 32 + lane;
                const bool act = j < cnt;
                const uint32_t src = src0 + (act ? j : 0);
                key[s] = act ? part_key(__ldg(in.idx[key_mode] + src), shift, mask) : 0xffffffffu;
                val[s] = __ldg(in.vals + src);
#pragma unroll
                for (int k = 0; k < N; ++k) id[s][k] = __ldg(in.idx[k] + src);
            }
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const bool act = key[s] != 0xffffffffu;
                const unsigned am = __ballot_sync(0xffffffffu, act);
                rk[s] = 0;
                if (act) {
                    const unsigned peers = __match_any_sync(am, key[s]);
                    const uint32_t prior = mywc[key[s]];
                    __syncwarp(am);
                    if ((peers & lt) == 0) mywc[key[s]] = (uint16_t)(prior + __popc(peers));
                    rk[s] = prior + __popc(peers & lt);
                }
                __syncwarp();
            }
            __syncthreads();
            // b. per-bucket warp prefixes and window bucket totals -> lbase
            for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
                uint32_t run = 0;
#pragma unroll
                for (int w = 0; w < kScatWarps; ++w) {
                    const uint32_t v = wc[(size_t)w * nb + b];
                    wc[(size_t)w * nb + b] = (uint16_t)run;
                    run += v;
                }
                lbase[b] = run;
            }
            __syncthreads();
            // exclusive scan of lbase over buckets (each thread a run of buckets)
            {
                __shared__ uint32_t wsum[kScatWarps];
                const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
                const uint32_t b0 = threadIdx.x * per;
                uint32_t s = 0;
                for (uint32_t k = 0; k < per; ++k)
                    if (b0 + k < nb) s += lbase[b0 + k];
                uint32_t x = s;
#pragma unroll
                for (int q = 1; q < 32; q <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, x, q);
                    if (lane >= q) x += y;
                }
                if (lane == 31) wsum[warp] = x;
                __syncthreads();
                if (warp == 0) {
                    uint32_t v = lane < kScatWarps ? wsum[lane] : 0u;
#pragma unroll
                    for (int q = 1; q < 32; q <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xffffffffu, v, q);
                        if (lane >= q) v += y;
                    }
                    if (lane < kScatWarps) wsum[lane] = v;
                }
                __syncthreads();
                uint32_t pre = (warp ? wsum[warp - 1] : 0u) + x - s;
                for (uint32_t k = 0; k < per; ++k)
                    if (b0 + k < nb) {
                        const uint32_t v = lbase[b0 + k];
                        lbase[b0 + k] = pre;
                        pre += v;
                    }
            }
            __syncthreads();
            // c. stage in bucket order with the global slot of each element
#pragma unroll
            for (int s = 0; s < S; ++s) {
                if (key[s] == 0xffffffffu) continue;
                const uint32_t within = (uint32_t)mywc[key[s]] + rk[s];
                const uint32_t lp = lbase[key[s]] + within;
                sv[lp] = val[s];
#pragma unroll
                for (int k = 0; k < N; ++k) si[(size_t)k * W + lp] = id[s][k];
                sd[lp] = cursor[key[s]] + within;
            }
            __syncthreads();
            // d. coalesced write-out, runs of one bucket are contiguous
            for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
                const uint32_t d = sd[i];
                out.vals[d] = sv[i];
#pragma unroll
                for (int k = 0; k < N; ++k) out.idx[k][d] = si[(size_t)k * W + i];
            }
            // e. advance the cursors, clear the warp counters
            for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
                const uint32_t next = (b + 1 < nb) ? lbase[b + 1] : cnt;
                cursor[b] += next - lbase[b];
            }
            for (uint32_t i = threadIdx.x; i < kScatWarps * nb; i += blockDim.x) wc[i] = 0;
            __syncthreads();
        }
    }
}

template <int N>
constexpr int scatter_window() { return N <= 4 ? 4096 : 2048; }

size_t scatter_smem(int N, uint32_t nb) {
    const int W = N <= 4 ? 4096 : 2048;
    return ((size_t)2 * nb + ((size_t)kScatWarps * nb + 1) / 2 + (size_t)(2 + N) * W) * 4;
}

int ensure_part_scratch(Plan& p, size_t entries, size_t base_entries) {
    if (entries > p.part_cap) {
        dev_free(p.part_cnt);
        dev_free(p.part_off);
        p.part_cnt = p.part_off = nullptr;
        p.part_cap = 0;
        DGPU_TRY(dev_alloc(p, (void**)&p.part_cnt, entries * sizeof(uint32_t)));
        DGPU_TRY(dev_alloc(p, (void**)&p.part_off, entries * sizeof(uint32_t)));
        p.part_cap = entries;
    }
    if (base_entries > p.part_base_cap) {
        dev_free(p.part_base);
        p.part_base = nullptr;
        p.part_base_cap = 0;
        DGPU_TRY(dev_alloc(p, (void**)&p.part_base, base_entries * sizeof(uint32_t)));
        p.part_base_cap = base_entries;
    }
    return DGPU_OK;
}

template <int N>
int launch_scatter(Plan& p, const Slab& in, const Slab& out, const PartList& L, int key_mode,
                   int key_shift, uint32_t key_mask, uint32_t nb)
{
    constexpr int W = scatter_window<N>();
    const size_t smem = scatter_smem(N, nb);
    static bool attr_set = false;
    if (!attr_set) {
        DGPU_CUDA(cudaFuncSetAttribute(k_chunk_scatter<N, W>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)scatter_smem(N, kMaxBuckets)));
        attr_set = true;
    }
    k_chunk_scatter<N, W><<<L.nchunks, kScatThreads, smem, p.stream>>>(
        slab_in(in, p.N), slab_out(out, p.N), L.tiles, L.chunks, p.part_off, p.part_base,
        key_mode, key_shift, key_mask, nb);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

}  // namespace

void free_partlist(PartList& l) {
    if (l.own_tiles) dev_free(l.tiles);
    dev_free(l.chunks);
    dev_free(l.segs);
    l = PartList{};
}

int build_partlist(Plan& p, const std::vector<Tile>& tiles, const std::vector<uint32_t>& seg_of_tile,
                   const std::vector<uint32_t>& seg_base, PartList& out, Tile* shared_tiles)
{
    free_partlist(out);
    const bool global = seg_of_tile.empty();
    std::vector<Chunk> ch;
    std::vector<Seg> sg;
    if (global) {
        // ~2 chunks per SM of roughly equal element counts
        uint64_t total = 0;
        for (const Tile& t : tiles) total += t.count;
        const uint64_t target = std::max<uint64_t>(kTile, (total + 2 * p.sms - 1) / (2 * p.sms));
        Seg s{0, 0, 0, 0};
        uint32_t t0 = 0;
        uint64_t acc = 0;
        for (uint32_t t = 0; t < tiles.size(); ++t) {
            acc += tiles[t].count;
            if (acc >= target || t + 1 == tiles.size()) {
                ch.push_back(Chunk{t0, t + 1, 0, 0});
                t0 = t + 1;
                acc = 0;
            }
        }
        s.chunk_end = (uint32_t)ch.size();
        sg.push_back(s);
    } else {
        const uint32_t nseg = (uint32_t)seg_base.size();
        sg.assign(nseg, Seg{0, 0, 0, 0});
        for (uint32_t s = 0; s < nseg; ++s) sg[s].base = seg_base[s];
        uint32_t t = 0;
        for (uint32_t s = 0; s < nseg; ++s) {
            sg[s].chunk_begin = (uint32_t)ch.size();
            while (t < tiles.size() && seg_of_tile[t] == s) {
                const uint32_t t0 = t;
                while (t < tiles.size() && seg_of_tile[t] == s && t - t0 < kSegChunkTiles) ++t;
                ch.push_back(Chunk{t0, t, s, 0});
            }
            sg[s].chunk_end = (uint32_t)ch.size();
        }
    }
    out.ntiles = (uint32_t)tiles.size();
    out.nchunks = (uint32_t)ch.size();
    out.nsegs = (uint32_t)sg.size();
    if (shared_tiles) {
        out.tiles = shared_tiles;
        out.own_tiles = false;
    } else {
        DGPU_TRY(dev_alloc(p, (void**)&out.tiles, std::max<size_t>(1, tiles.size()) * sizeof(Tile)));
        out.own_tiles = true;
        if (!tiles.empty())
            DGPU_CUDA(cudaMemcpyAsync(out.tiles, tiles.data(), tiles.size() * sizeof(Tile),
                                      cudaMemcpyHostToDevice, p.stream));
    }
    DGPU_TRY(dev_alloc(p, (void**)&out.chunks, std::max<size_t>(1, ch.size()) * sizeof(Chunk)));
    DGPU_TRY(dev_alloc(p, (void**)&out.segs, std::max<size_t>(1, sg.size()) * sizeof(Seg)));
    if (!ch.empty())
        DGPU_CUDA(cudaMemcpyAsync(out.chunks, ch.data(), ch.size() * sizeof(Chunk),
                                  cudaMemcpyHostToDevice, p.stream));
    DGPU_CUDA(cudaMemcpyAsync(out.segs, sg.data(), sg.size() * sizeof(Seg), cudaMemcpyHostToDevice,
                              p.stream));
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    return DGPU_OK;
}

int stable_partition(Plan& p, const Slab& in, const PartList& L, int key_mode, int key_shift,
                     uint32_t key_mask, uint32_t nb, const Slab& out)
{
    if (L.nchunks == 0) return DGPU_OK;
    if (nb == 0 || nb > kMaxBuckets) {
        set_error("stable_partition: %u buckets (max %u)", nb, kMaxBuckets);
        return DGPU_ERR_ARG;
    }
    DGPU_TRY(ensure_part_scratch(p, (size_t)L.nchunks * nb, (size_t)L.nsegs * nb));
    const double elem = (double)p.nnz;
    const double row_bytes = 4.0 + 4.0 * p.N;
    {
        LaunchTimer t(p, KK_PART_HIST, elem * 4.0 + (double)L.nchunks * nb * 4.0);
        k_chunk_hist<<<L.nchunks, kHistThreads, nb * sizeof(uint32_t), p.stream>>>(
            in.idx[key_mode], L.tiles, L.chunks, key_shift, key_mask, nb, p.part_cnt);
        DGPU_CUDA(cudaGetLastError());
    }
    {
        LaunchTimer t(p, KK_PART_SCAN, (double)L.nchunks * nb * 8.0);
        dim3 g(L.nsegs, (nb + 255) / 256);
        k_col_scan<<<g, 256, 0, p.stream>>>(p.part_cnt, L.segs, nb, p.part_off, p.part_base);
        k_bucket_scan<<<L.nsegs, 1024, 0, p.stream>>>(p.part_base, L.segs, nb);
        DGPU_CUDA(cudaGetLastError());
    }
    LaunchTimer t(p, KK_PART_SCATTER, elem * 2.0 * row_bytes + (double)L.nchunks * nb * 4.0);
    switch (p.N) {
#define DGPU_SC(NN) case NN: return launch_scatter<NN>(p, in, out, L, key_mode, key_shift, key_mask, nb)
        DGPU_SC(2); DGPU_SC(3); DGPU_SC(4); DGPU_SC(5); DGPU_SC(6); DGPU_SC(7); DGPU_SC(8);
#undef DGPU_SC
        default:
            set_error("stable_partition: %d modes unsupported", p.N);
            return DGPU_ERR_ARG;
    }
}

int stable_sort_pingpong(Plan& p, int a, int b, const PartList& first, int key_mode,
                         int key_shift, uint64_t key_limit, int* result)
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
        const PartList& L = (k == 0) ? first : p.ident;
        DGPU_TRY(stable_partition(p, p.slab[src], L, key_mode, sh, mask, nb, p.slab[dst]));
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
    if (!p.fib[n].chunks) {
        set_error("fiber_sort: mode %d has no fiber tile list", n);
        return DGPU_ERR_NOT_BUILT;
    }
    const int passes = (bits + kDigitBits - 1) / kDigitBits;
    const int dbits = (bits + passes - 1) / passes;
    int a = src, b = other;
    for (int k = 0; k < passes; ++k) {
        const int sh = k * dbits;
        const int hi = std::min(bits, sh + dbits);
        const uint32_t mask = (1u << (hi - sh)) - 1u;
        DGPU_TRY(stable_partition(p, p.slab[a], p.fib[n], n, sh, mask, mask + 1, p.slab[b]));
        std::swap(a, b);
    }
    *result = a;
    return DGPU_OK;
}

}  // namespace dgpu
