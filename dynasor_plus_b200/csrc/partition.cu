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
#include <map>
#include <mutex>
#include <numeric>

namespace dgpu {

namespace {

constexpr int kHistThreads = 1024;
#ifndef DGPU_SCAT_THREADS
#define DGPU_SCAT_THREADS 512
#endif
#ifndef DGPU_SCAT_WINDOW
#define DGPU_SCAT_WINDOW 2048
#endif
#ifndef DGPU_SCAT_MINB
#define DGPU_SCAT_MINB 2
#endif
constexpr int kScatThreads = DGPU_SCAT_THREADS;   // threads of a scatter CTA
constexpr int kScatWarps = kScatThreads / 32;
// Most window buffers a scatter CTA uses (see scatter_bufs).
constexpr int kScatBufsMax = 3;
// Thread that issues a scatter CTA's bulk copies: the last one, whose warp
// has no bucket-prefix work for up to kScatThreads / 2 buckets.
constexpr int kIssuer = kScatThreads - 1;
constexpr uint32_t kSegChunkTilesMax = 16;    // <= 64K elements per segmented chunk

__device__ __forceinline__ uint32_t part_key(uint32_t v, int shift, uint32_t mask) {
    return (v >> shift) & mask;
}

// Counts the keys of positions [begin, begin + count) into hc: scalar head
// up to a 16-byte boundary (the column starts 256-byte aligned), 16-byte
// loads four at a time (16 keys per thread in flight), scalar tail.
// Threads `tid` of `nt` share the range.
__device__ __forceinline__ void hist_range(const uint32_t* __restrict__ keycol, uint32_t begin,
                                           uint32_t count, int shift, uint32_t mask,
                                           uint32_t* hc, uint32_t tid, uint32_t nt)
{
    const uint32_t* k = keycol + begin;
    const uint32_t head = min(count, (4u - (begin & 3u)) & 3u);
    for (uint32_t j = tid; j < head; j += nt)
        atomicAdd(&hc[part_key(__ldg(k + j), shift, mask)], 1u);
    const uint32_t n4 = (count - head) >> 2;
    const uint4* k4 = reinterpret_cast<const uint4*>(k + head);
    for (uint32_t i = tid; i < n4; i += 4 * nt) {
        uint4 a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t ii = i + u * nt;
            a[u] = ii < n4 ? __ldg(k4 + ii) : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i + u * nt >= n4) break;
            atomicAdd(&hc[part_key(a[u].x, shift, mask)], 1u);
            atomicAdd(&hc[part_key(a[u].y, shift, mask)], 1u);
            atomicAdd(&hc[part_key(a[u].z, shift, mask)], 1u);
            atomicAdd(&hc[part_key(a[u].w, shift, mask)], 1u);
        }
    }
    for (uint32_t j = head + 4 * n4 + tid; j < count; j += nt)
        atomicAdd(&hc[part_key(__ldg(k + j), shift, mask)], 1u);
}

// One CTA per chunk.  With `copies` > 1 every warp group counts into its
// own copy of the histogram (fewer shared-atomic collisions on skewed keys:
// hot rows of a Zipf mode land in few buckets); the copies are summed at the
// end.  A chunk whose tiles are consecutive slab ranges (Chunk::contiguous = 1:
// identity order and the shard-segmented fiber sorts) is counted as one
// range, so no tile descriptor load sits between its key loads; otherwise
// (processing order) each warp takes its own tiles, so the warps' loads
// overlap.
__global__ void __launch_bounds__(kHistThreads)
k_chunk_hist(const uint32_t* __restrict__ keycol, const Tile* __restrict__ tiles,
             const Chunk* __restrict__ chunks, int shift, uint32_t mask, uint32_t nb,
             int copies, uint32_t* __restrict__ cnt)
{
    extern __shared__ uint32_t h[];                 // [copies][nb]
    for (uint32_t b = threadIdx.x; b < nb * copies; b += blockDim.x) h[b] = 0;
    __syncthreads();
    uint32_t* hc = h + (size_t)((threadIdx.x >> 5) % copies) * nb;
    const Chunk c = chunks[blockIdx.x];
    if (c.contiguous && c.tile_end > c.tile_begin) {
        const Tile a = tiles[c.tile_begin], z = tiles[c.tile_end - 1];
        hist_range(keycol, a.begin, z.begin + z.count - a.begin, shift, mask, hc, threadIdx.x,
                   blockDim.x);
    } else {
        const uint32_t lane = threadIdx.x & 31u, nw = blockDim.x >> 5;
        for (uint32_t t = c.tile_begin + (threadIdx.x >> 5); t < c.tile_end; t += nw) {
            const Tile tl = tiles[t];
            hist_range(keycol, tl.begin, tl.count, shift, mask, hc, lane, 32u);
        }
    }
    __syncthreads();
    uint32_t* out = cnt + (size_t)blockIdx.x * nb;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
        uint32_t v = 0;
        for (int q = 0; q < copies; ++q) v += h[(size_t)q * nb + b];
        out[b] = v;
    }
}

// grid (segments, ceil(nb/32)), 1024 threads: lane = bucket of the CTA's
// 32, warp = one of 32 slices of the segment's chunks.  Each slice sums its
// chunks, the slices' sums are prefixed in shared memory, then each slice
// writes its chunks' exclusive offsets; the last slice's running total is
// the segment total of the bucket.
__global__ void __launch_bounds__(1024)
k_col_scan(const uint32_t* __restrict__ cnt, const Seg* __restrict__ segs, uint32_t nb,
           uint32_t* __restrict__ off, uint32_t* __restrict__ segtot)
{
    __shared__ uint32_t part[32][33];
    const uint32_t lane = threadIdx.x & 31u, sl = threadIdx.x >> 5;
    const uint32_t b = blockIdx.y * 32u + lane;
    const Seg s = segs[blockIdx.x];
    const uint32_t nc = s.chunk_end - s.chunk_begin;
    const uint32_t per = (nc + 31u) / 32u;
    const uint32_t c0 = s.chunk_begin + min(nc, sl * per);
    const uint32_t c1 = s.chunk_begin + min(nc, (sl + 1u) * per);
    uint32_t sum = 0;
    if (b < nb) {
        uint32_t c = c0;
        for (; c + 4 <= c1; c += 4) {
            uint32_t v[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) v[k] = cnt[(size_t)(c + k) * nb + b];
            sum += (v[0] + v[1]) + (v[2] + v[3]);
        }
        for (; c < c1; ++c) sum += cnt[(size_t)c * nb + b];
    }
    part[sl][lane] = sum;
    __syncthreads();
    uint32_t run = 0;
    for (uint32_t k = 0; k < sl; ++k) run += part[k][lane];
    if (b >= nb) return;
    for (uint32_t c = c0; c < c1; ++c) {
        const uint32_t v = cnt[(size_t)c * nb + b];
        off[(size_t)c * nb + b] = run;
        run += v;
    }
    if (sl == 31u) segtot[(size_t)blockIdx.x * nb + b] = run;
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

// ---- bulk-copy (TMA) helpers: one elected thread streams each window's
// columns into shared memory; an mbarrier with a transaction count tells the
// CTA when they have landed.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait: false after ~2^22 polls (each poll may suspend the thread).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < (1u << 22); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Device fault-flag codes written by the partition kernels.
constexpr int kErrPartWait = 0x100;      // a bulk copy did not complete in time
constexpr int kErrPartRange = 0x200;     // a slot outside its window or slab (skipped)
constexpr int kErrPartCache = 0x1000;    // a kept offset table differs from a recomputed one

// Flags kErrPartCache where a[i] != b[i] (check mode of the kept tables).
__global__ void k_cmp_tables(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                             size_t n, int* __restrict__ err)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        if (a[i] != b[i]) {
            atomicOr(err, kErrPartCache);
            return;
        }
}

// Tile descriptors of a chunk that a scatter CTA copies to shared memory
// when it takes the chunk (a chunk with more tiles reads the rest from
// global memory).
constexpr uint32_t kTileStage = 64;

// Next non-empty window of a chunk after (t, w0): windows are W-element
// pieces of the chunk's tiles in order.  Returns false at the chunk's end.
// Tiles tb .. tb + kTileStage - 1 come from the shared copy `st`.
template <int W>
__device__ __forceinline__ bool next_window(const Tile* __restrict__ tiles, const Tile* st,
                                            uint32_t tb, uint32_t tend, uint32_t& t, uint32_t& w0,
                                            Tile& tl)
{
    w0 += W;
    while (w0 >= tl.count) {
        if (++t >= tend) return false;
        tl = (t - tb < kTileStage) ? st[t - tb] : tiles[t];
        w0 = 0;
    }
    return true;
}

// Column stride of a window buffer: W elements plus the up-to-3-element head
// and tail that 16-byte alignment of the bulk copies adds.
template <int W> constexpr int win_stride() { return W + 8; }

// Streams window (tl.begin + w0, cnt) of every column into `buf` (column c
// at buf + c * BW); the head (begin & 3) is where element 0 lands.
template <int N, int W>
__device__ __forceinline__ void issue_window(uint32_t* buf, const SlabPtrs& in, uint32_t src,
                                             uint32_t cnt, uint64_t* bar)
{
    constexpr int BW = win_stride<W>();
    const uint32_t a = src & ~3u;
    const uint32_t e = (src + cnt + 3u) & ~3u;
    const uint32_t bytes = (e - a) * 4u;
    mbar_expect_tx(bar, bytes * (N + 1));
    bulk_g2s(buf, in.vals + a, bytes, bar);
#pragma unroll
    for (int k = 0; k < N; ++k) bulk_g2s(buf + (size_t)(k + 1) * BW, in.idx[k] + a, bytes, bar);
}

// Per-warp 16-bit bucket counters, bucket-major: bucket b's 16 counters
// (one per warp) fill the 32 bytes at b * 16, so one thread reads and
// rewrites a bucket's counters with two 16-byte accesses.  The pair of warps
// (2j, 2j+1) sits in word j ^ (b & 7) of the row, which spreads the lanes of
// one warp that touch different buckets over all 32 banks.
__device__ __forceinline__ uint32_t wc_slot(uint32_t b, int warp) {
    return b * 16u + (((((uint32_t)warp >> 1) ^ (b & 7u))) << 1) + ((uint32_t)warp & 1u);
}

// Row of bucket b <-> the 8 words in warp-pair order: word j and j ^ (b & 7)
// swap places (an involution, so the same call maps both ways).
__device__ __forceinline__ void wc_unswizzle(uint32_t (&u)[8], uint32_t b) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const bool sw = (b >> k) & 1u;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (j & (1 << k)) continue;
            const uint32_t a = u[j], c = u[j | (1 << k)];
            u[j] = sw ? c : a;
            u[j | (1 << k)] = sw ? a : c;
        }
    }
}

// Window size of the scatter and its buffer column count: N+1 input
// columns; staging needs a 16-byte record (4 words) when N <= 3, else the
// N+1 columns again.  A staged element's destination is recomputed at
// write-out from its key, so it is not stored.
template <int N>
constexpr int scatter_window() { return N <= 4 ? DGPU_SCAT_WINDOW : DGPU_SCAT_WINDOW / 2; }
template <int N>
constexpr int scatter_cols() { return N + 1 <= 4 ? 4 : N + 1; }
// Window buffers: three (window k+2 streams in while window k is ranked and
// written) while two CTAs per SM still fit in shared memory (4-column
// buffers, N <= 3), else two.
template <int N>
constexpr int scatter_bufs() { return scatter_cols<N>() <= 4 ? 3 : 2; }

// Persistent CTAs of 512 threads take chunks from a work queue (largest
// first).  A chunk is walked in windows of W elements; while window k is
// ranked and written, window k+1 streams into the other of two shared
// buffers.  Per window (four block barriers):
//   a. each warp ranks its W/16 elements (32 per step) with __match_any_sync
//      and 16-bit per-warp bucket counters;
//   b. per bucket: exclusive prefix over the 16 warps and the window total;
//      exclusive scan over buckets; bucket cursors advance by the totals;
//   c. each element is staged at its bucket-ordered window slot, with its
//      destination, in the buffer it came from; warps reset their counters;
//   d. the staged window is written out: consecutive threads store
//      consecutive slots of one bucket.
template <int N, int W, bool REC>
__global__ void __launch_bounds__(kScatThreads, DGPU_SCAT_MINB)
k_chunk_scatter(const __grid_constant__ SlabPtrs in, const __grid_constant__ SlabOut out,
                const Tile* __restrict__ tiles, const Chunk* __restrict__ chunks,
                const uint32_t* __restrict__ order, uint32_t nchunks,
                const uint32_t* __restrict__ off, const uint32_t* __restrict__ base,
                int key_mode, int shift, uint32_t mask, uint32_t nb, uint32_t total,
                uint32_t* __restrict__ queue, int* __restrict__ err,
                const uint32_t* __restrict__ tile_pre, const uint32_t* __restrict__ tile_wb,
                uint16_t* __restrict__ rec_inv, uint32_t* __restrict__ rec_tab)
{
    constexpr int S = W / kScatThreads;           // steps per warp per window
    constexpr int PW = W / kScatWarps;            // elements per warp per window
    constexpr int BW = win_stride<W>();
    // staged element: one 16-byte record (val, idx...) when N <= 3, else columns
    constexpr bool kRec = (N + 1 <= 4);
    constexpr int C = scatter_cols<N>();          // buffer columns (input, then stage)
    constexpr int BPT = (kMaxBuckets + kScatThreads - 1) / kScatThreads;  // buckets per thread, at most
    extern __shared__ __align__(128) uint32_t sm[];
    constexpr int NBUF = scatter_bufs<N>();
    __shared__ __align__(8) uint64_t bar[kScatBufsMax];
    __shared__ uint32_t wsum[kScatWarps];
    __shared__ uint32_t s_chunk[2];     // alternating: a slot is rewritten two barriers later
    __shared__ Tile s_tiles[kTileStage];
    __shared__ int fail;
    const uint32_t nbp = (nb + 7u) & ~7u;
    uint32_t* buf = sm;                                      // [NBUF][C][BW]
    uint32_t* cursor = buf + NBUF * C * BW;                  // [nbp]
    uint32_t* wbase = cursor + nbp;                          // [nbp] bucket's first window slot
    uint32_t* wdst = wbase + nbp;                            // [nbp] destination - slot
    uint16_t* wc = reinterpret_cast<uint16_t*>(wdst + nbp);  // [nbp][16], see wc_slot
    static_assert(kScatWarps == 16, "bucket counter rows hold 16 warps");

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (uint32_t i = threadIdx.x; i < kScatWarps * nbp / 2; i += blockDim.x)
        reinterpret_cast<uint32_t*>(wc)[i] = 0;
    if (threadIdx.x == 0) {
        fail = 0;
        for (int k = 0; k < NBUF; ++k) mbar_init(&bar[k], 1);
        fence_mbar_init();
    }
    // window k (counted over the CTA's life) streams into buffer k % NBUF
    // and completes phase (k / NBUF) & 1 of that buffer's mbarrier
    uint32_t kw = 0;               // window being processed
    uint32_t issued = 0;           // windows whose bulk copies were issued
    auto bufk = [&](uint32_t k) { return buf + (size_t)(k % NBUF) * C * BW; };
    auto bark = [&](uint32_t k) { return &bar[k % NBUF]; };
    auto park = [](uint32_t k) { return (k / NBUF) & 1u; };

    for (uint32_t it = 0;; ++it) {
        if (threadIdx.x == 0) s_chunk[it & 1] = atomicAdd(queue, 1u);
        __syncthreads();           // previous chunk fully written; s_chunk visible
        const uint32_t qi = s_chunk[it & 1];
        if (qi >= nchunks || fail) break;
        const uint32_t ci = order[qi];
        const Chunk c = chunks[ci];
        const uint32_t* o = off + (size_t)ci * nb;
        const uint32_t* bs = base + (size_t)c.seg * nb;
        for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) cursor[b] = o[b] + bs[b];
        if (c.tile_begin >= c.tile_end) continue;
        const uint32_t nst = min(kTileStage, c.tile_end - c.tile_begin);
        for (uint32_t i = threadIdx.x; i < nst; i += blockDim.x) s_tiles[i] = tiles[c.tile_begin + i];
        __syncthreads();           // tile descriptors staged
        // the chunk's first window (t, w0, tl), and with three buffers its
        // second (t1, w1, tl1); with two buffers the second is found after
        // barrier (1) of the first
        uint32_t t = c.tile_begin, w0 = 0u - (uint32_t)W;
        Tile tl = s_tiles[0];
        if (!next_window<W>(tiles, s_tiles, c.tile_begin, c.tile_end, t, w0, tl)) continue;
        if (threadIdx.x == kIssuer)
            issue_window<N, W>(bufk(kw), in, tl.begin + w0, min((uint32_t)W, tl.count - w0), bark(kw));
        issued = kw + 1;
        uint32_t t1 = t, w1 = w0;
        Tile tl1 = tl;
        bool has1 = false;
        if constexpr (NBUF == 3) {
            has1 = next_window<W>(tiles, s_tiles, c.tile_begin, c.tile_end, t1, w1, tl1);
            if (has1) {
                if (threadIdx.x == kIssuer)
                    issue_window<N, W>(bufk(kw + 1), in, tl1.begin + w1,
                                       min((uint32_t)W, tl1.count - w1), bark(kw + 1));
                issued = kw + 2;
            }
        }

        for (;;) {
            const uint32_t cnt = min((uint32_t)W, tl.count - w0);
            const uint32_t head = (tl.begin + w0) & 3u;
            uint32_t* bk = bufk(kw);
            if (!mbar_wait(bark(kw), park(kw))) {
                fail = 1;
                atomicOr(err, kErrPartWait);
            }
            // REC: the window's list offset and index
            uint32_t ro = 0, wid = 0;
            if constexpr (REC) {
                ro = tile_pre[t] + w0;
                wid = tile_wb[t] + w0 / (uint32_t)W;
            }
            // a. load the window's elements and rank them per warp
            uint32_t key[S], rk[S];
            float val[S];
            uint32_t id[S][N];
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const uint32_t j = warp * PW + s * 32 + lane;
                const bool act = j < cnt;
                const uint32_t q = head + (act ? j : 0);
#pragma unroll
                for (int m = 0; m < N; ++m) id[s][m] = bk[(size_t)(m + 1) * BW + q];
                val[s] = __uint_as_float(bk[q]);
                const uint32_t kv = bk[(size_t)(key_mode + 1) * BW + q];
                key[s] = act ? part_key(kv, shift, mask) : 0xffffffffu;
            }
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const bool act = key[s] != 0xffffffffu;
                const unsigned am = __ballot_sync(0xffffffffu, act);
                rk[s] = 0;
                if (act) {
                    const unsigned peers = __match_any_sync(am, key[s]);
                    const uint32_t slot = wc_slot(key[s], warp);
                    const uint32_t prior = wc[slot];
                    __syncwarp(am);
                    if ((peers & lt) == 0) wc[slot] = (uint16_t)(prior + __popc(peers));
                    rk[s] = prior + __popc(peers & lt);
                }
                __syncwarp();
            }
            __syncthreads();       // (1) buffer read, counters complete, `fail` visible
            if (fail) break;
            // prefetch window kw + NBUF - 1 into the buffer window kw-1
            // used: its write-out finished before barrier (1)
            uint32_t t2 = t1, w2 = w1;
            Tile tl2 = tl1;
            bool has2 = false;
            if constexpr (NBUF == 3) {
                has2 = has1 && next_window<W>(tiles, s_tiles, c.tile_begin, c.tile_end, t2, w2, tl2);
                if (has2) {
                    if (threadIdx.x == kIssuer)
                        issue_window<N, W>(bufk(kw + 2), in, tl2.begin + w2,
                                           min((uint32_t)W, tl2.count - w2), bark(kw + 2));
                    issued = kw + 3;
                }
            } else {
                has1 = next_window<W>(tiles, s_tiles, c.tile_begin, c.tile_end, t1, w1, tl1);
                if (has1) {
                    if (threadIdx.x == kIssuer)
                        issue_window<N, W>(bufk(kw + 1), in, tl1.begin + w1,
                                           min((uint32_t)W, tl1.count - w1), bark(kw + 1));
                    issued = kw + 2;
                }
            }
            // b. warp prefixes per bucket (only counters a warp used become
            //    prefixes, so the warps' resets in c leave all counters zero)
            const uint32_t per = (nb + kScatThreads - 1) / kScatThreads;
            const uint32_t b0 = threadIdx.x * per;
            uint32_t tot[BPT];
            uint32_t sum = 0;
#pragma unroll
            for (int u = 0; u < BPT; ++u) {
                tot[u] = 0;
                const uint32_t b = b0 + u;
                if ((uint32_t)u < per && b < nb) {
                    uint4* row = reinterpret_cast<uint4*>(wc + (size_t)b * 16);
                    const uint4 q0 = row[0], q1 = row[1];
                    uint32_t r8[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
                    wc_unswizzle(r8, b);
                    uint32_t run = 0;
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const uint32_t lo = r8[j] & 0xffffu, hi = r8[j] >> 16;
                        const uint32_t plo = lo ? run : 0u;
                        run += lo;
                        const uint32_t phi = hi ? run : 0u;
                        run += hi;
                        r8[j] = plo | (phi << 16);
                    }
                    wc_unswizzle(r8, b);
                    row[0] = make_uint4(r8[0], r8[1], r8[2], r8[3]);
                    row[1] = make_uint4(r8[4], r8[5], r8[6], r8[7]);
                    tot[u] = run;
                    sum += run;
                }
            }
            uint32_t x = sum;
#pragma unroll
            for (int q = 1; q < 32; q <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, q);
                if (lane >= q) x += y;
            }
            if (lane == 31) wsum[warp] = x;
            __syncthreads();       // (2)
            {
                uint32_t v = (lane < warp) ? wsum[lane] : 0u;
#pragma unroll
                for (int q = 16; q >= 1; q >>= 1) v += __shfl_xor_sync(0xffffffffu, v, q);
                uint32_t pre = v + x - sum;
#pragma unroll
                for (int u = 0; u < BPT; ++u) {
                    const uint32_t b = b0 + u;
                    if ((uint32_t)u < per && b < nb) {
                        const uint32_t cur = cursor[b];
                        wbase[b] = pre;
                        wdst[b] = cur - pre;
                        if constexpr (REC) rec_tab[(size_t)wid * nb + b] = cur - pre;
                        cursor[b] = cur + tot[u];
                        pre += tot[u];
                    }
                }
            }
            __syncthreads();       // (3)
            // c. stage in bucket order (REC: for each slot, the window index
            //    of the element staged there)
#pragma unroll
            for (int s = 0; s < S; ++s) {
                if (key[s] == 0xffffffffu) continue;
                const uint32_t lp = wbase[key[s]] + wc[wc_slot(key[s], warp)] + rk[s];
                if (lp >= cnt) { atomicOr(err, kErrPartRange); continue; }
                if constexpr (REC) rec_inv[ro + lp] = (uint16_t)(warp * PW + s * 32 + lane);
                if constexpr (kRec) {
                    uint32_t r[4] = {__float_as_uint(val[s]), 0u, 0u, 0u};
#pragma unroll
                    for (int m = 0; m < N; ++m) r[m + 1] = id[s][m];
                    reinterpret_cast<uint4*>(bk)[lp] = make_uint4(r[0], r[1], r[2], r[3]);
                } else {
                    bk[lp] = __float_as_uint(val[s]);
#pragma unroll
                    for (int m = 0; m < N; ++m) bk[(size_t)(m + 1) * BW + lp] = id[s][m];
                }
            }
            __syncwarp();
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (key[s] != 0xffffffffu) wc[wc_slot(key[s], warp)] = 0;
            __syncthreads();       // (4)
            // d. write-out: runs of one bucket are contiguous; slot i of
            //    bucket b goes to (cursor of b before this window) + i - (the
            //    bucket's first slot), i.e. wdst[b] + i, b from the element's key
            for (uint32_t i = threadIdx.x; i < cnt; i += kScatThreads) {
                if constexpr (kRec) {
                    const uint4 r = reinterpret_cast<const uint4*>(bk)[i];
                    const uint32_t rv[4] = {r.x, r.y, r.z, r.w};
                    const uint32_t kv = key_mode == 0 ? r.y : (key_mode == 1 ? r.z : r.w);
                    const uint32_t kb = part_key(kv, shift, mask);
                    const uint32_t d = kb < nb ? wdst[kb] + i : total;
                    if (d >= total) { atomicOr(err, kErrPartRange); continue; }
                    out.vals[d] = __uint_as_float(rv[0]);
#pragma unroll
                    for (int m = 0; m < N; ++m) out.idx[m][d] = rv[m + 1];
                } else {
                    const uint32_t kb = part_key(bk[(size_t)(key_mode + 1) * BW + i], shift, mask);
                    const uint32_t d = kb < nb ? wdst[kb] + i : total;
                    if (d >= total) { atomicOr(err, kErrPartRange); continue; }
                    out.vals[d] = __uint_as_float(bk[i]);
#pragma unroll
                    for (int m = 0; m < N; ++m) out.idx[m][d] = bk[(size_t)(m + 1) * BW + i];
                }
            }
            fence_proxy_async_smem();   // generic accesses before a later bulk write
            ++kw;
            if (!has1) break;
            t = t1; w0 = w1; tl = tl1;
            if constexpr (NBUF == 3) {
                t1 = t2; w1 = w2; tl1 = tl2; has1 = has2;
            } else {
                has1 = false;
            }
        }
        if (fail) break;
    }
    // leave no bulk copy in flight into this CTA's shared memory: on a
    // failure, windows kw .. issued-1 may still be streaming
    if (fail && threadIdx.x == kIssuer)
        for (uint32_t k = kw; k < issued; ++k) mbar_wait(bark(k), park(k));
}



// Replay of a recorded pass: the window list in order, grid-strided when
// the grid is capped, else one CTA per window (the destinations are
// recorded, so windows are independent).  Per window each
// thread loads its elements (input order) and the recorded source element
// of each slot it will write, and the CTA the window's bucket table -- all
// before the barrier, so one memory latency per window; the elements are
// stored in shared memory in input order (a 16-byte record when N <= 3, else
// one word per column); then slot i takes element inv[i] and goes to
// tab[b] + i (b from its key): the bucket-ordered runs of the ranked
// scatter, without its ranking, counters and prefixes.  512 threads of
// <= 40 registers, 3 CTAs per SM: the kernel waits on its loads, so it is
// built for warps in flight (4 CTAs at 32 registers spill and measured
// slower: 2.90 -> 3.20 ms of fiber passes per 3-mode sweep).
constexpr int kReplayThreads = 512;
constexpr int kReplayMinBlocks = 3;
template <int N, int W>
__global__ void __launch_bounds__(kReplayThreads, kReplayMinBlocks)
k_part_replay(const __grid_constant__ SlabPtrs in, const __grid_constant__ SlabOut out,
              const uint4* __restrict__ wins, uint32_t nwin, const uint16_t* __restrict__ inv,
              const uint32_t* __restrict__ tab, int key_mode, int shift, uint32_t mask,
              uint32_t nb, uint32_t total, int* __restrict__ err)
{
    constexpr int U = W / kReplayThreads;         // elements per thread per window
    constexpr bool kRec = (N + 1 <= 4);
    constexpr int C = kRec ? 4 : N + 1;
    extern __shared__ __align__(128) uint32_t sm[];  // [W] records or [N+1][W] columns, then [nb]
    uint32_t* stab = sm + (size_t)C * W;
    for (uint32_t w = blockIdx.x; w < nwin; w += gridDim.x) {
        const uint4 d = wins[w];                  // {src, list offset, count, -}
        const uint32_t cnt = min(d.z, (uint32_t)W);
        uint32_t src[U];
        float val[U];
        uint32_t id[U][N];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t j = u * kReplayThreads + threadIdx.x;
            src[u] = 0xffffffffu;
            if (j < cnt) {
                src[u] = inv[d.y + j];
                val[u] = in.vals[d.x + j];
#pragma unroll
                for (int m = 0; m < N; ++m) id[u][m] = in.idx[m][d.x + j];
            }
        }
        for (uint32_t b = threadIdx.x; b < nb; b += kReplayThreads) stab[b] = tab[(size_t)w * nb + b];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t j = u * kReplayThreads + threadIdx.x;
            if (j >= cnt) break;
            if constexpr (kRec) {
                uint32_t r[4] = {__float_as_uint(val[u]), 0u, 0u, 0u};
#pragma unroll
                for (int m = 0; m < N; ++m) r[m + 1] = id[u][m];
                reinterpret_cast<uint4*>(sm)[j] = make_uint4(r[0], r[1], r[2], r[3]);
            } else {
                sm[j] = __float_as_uint(val[u]);
#pragma unroll
                for (int m = 0; m < N; ++m) sm[(size_t)(m + 1) * W + j] = id[u][m];
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t i = u * kReplayThreads + threadIdx.x;
            if (i >= cnt) break;
            const uint32_t e = src[u];
            if (e >= cnt) { atomicOr(err, kErrPartRange); continue; }
            if constexpr (kRec) {
                const uint4 r = reinterpret_cast<const uint4*>(sm)[e];
                const uint32_t rv[4] = {r.x, r.y, r.z, r.w};
                const uint32_t kv = key_mode == 0 ? r.y : (key_mode == 1 ? r.z : r.w);
                const uint32_t kb = part_key(kv, shift, mask);
                const uint32_t g = kb < nb ? stab[kb] + i : total;
                if (g >= total) { atomicOr(err, kErrPartRange); continue; }
                out.vals[g] = __uint_as_float(rv[0]);
#pragma unroll
                for (int m = 0; m < N; ++m) out.idx[m][g] = rv[m + 1];
            } else {
                const uint32_t kb = part_key(sm[(size_t)(key_mode + 1) * W + e], shift, mask);
                const uint32_t g = kb < nb ? stab[kb] + i : total;
                if (g >= total) { atomicOr(err, kErrPartRange); continue; }
                out.vals[g] = __uint_as_float(sm[e]);
#pragma unroll
                for (int m = 0; m < N; ++m) out.idx[m][g] = sm[(size_t)(m + 1) * W + e];
            }
        }
        __syncthreads();                          // staging reused by the next window
    }
}

template <int N>
size_t replay_smem(uint32_t nb) {
    return ((N + 1 <= 4 ? 4 : N + 1) * (size_t)scatter_window<N>() + nb) * sizeof(uint32_t);
}

template <int N>
size_t scatter_smem(uint32_t nb) {
    const size_t nbp = (nb + 7u) & ~7u;
    return (scatter_bufs<N>() * (size_t)scatter_cols<N>() * win_stride<scatter_window<N>()>() + 3 * nbp) * 4 +
           (size_t)kScatWarps * nbp * 2;
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

// Raises kernel `k`'s dynamic shared memory limit on this device (function
// attributes are per context) to `smem` if it is below (the limit only
// grows; guarded because plans may be driven from several host threads).
// Kept per (kernel, device): instantiations share a function type.
template <typename K>
int ensure_smem_limit(K* k, size_t smem, int device) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> have;
    std::lock_guard<std::mutex> lk(mu);
    size_t& h = have[std::make_pair(reinterpret_cast<const void*>(k), device)];
    if (smem <= h) return DGPU_OK;
    if (smem > 227u * 1024u) {
        set_error("stable_partition: a pass needs %zu bytes of shared memory", smem);
        return DGPU_ERR_ARG;
    }
    DGPU_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    h = smem;
    return DGPU_OK;
}

// The ranked scatter of one pass; with `rec` it also records the pass into
// rec's slot and destination arrays.
template <int N>
int launch_scatter(Plan& p, const Slab& in, const Slab& out, const PartList& L, int key_mode,
                   int key_shift, uint32_t key_mask, uint32_t nb, const uint32_t* off,
                   const uint32_t* base, const PartCacheSlot* rec)
{
    constexpr int W = scatter_window<N>();
    const size_t smem = scatter_smem<N>(nb);
    auto* kern = rec ? k_chunk_scatter<N, W, true> : k_chunk_scatter<N, W, false>;
    DGPU_TRY(ensure_smem_limit(kern, smem, p.device));
    int per_sm = 0;
    DGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kScatThreads, smem));
    const uint32_t grid = std::max(1u, std::min(L.nchunks, (uint32_t)(std::max(1, per_sm) * p.sms)));
    DGPU_CUDA(cudaMemsetAsync(p.part_ctr, 0, sizeof(uint32_t), p.stream));
    kern<<<grid, kScatThreads, smem, p.stream>>>(
        slab_in(in, p.N), slab_out(out, p.N), L.tiles, L.chunks, L.order, L.nchunks, off,
        base, key_mode, key_shift, key_mask, nb, (uint32_t)p.nnz, p.part_ctr, p.err_flag,
        L.tile_pre, L.tile_wb, rec ? rec->inv : nullptr, rec ? rec->tab : nullptr);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

template <int N>
int launch_replay(Plan& p, const Slab& in, const Slab& out, const PartList& L,
                  const PartCacheSlot& cs)
{
    constexpr int W = scatter_window<N>();
    const size_t smem = replay_smem<N>(cs.nb);
    auto* kern = k_part_replay<N, W>;
    DGPU_TRY(ensure_smem_limit(kern, smem, p.device));
    int per_sm = 0;
    DGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kReplayThreads, smem));
    if (p.replay_cap > 0) per_sm = std::min(per_sm, p.replay_cap);   // beside the MTTKRP
    // one CTA per window: CTAs retire window by window, so work queued on
    // other streams (a CP-ALS factor update beside a fiber-sort pass) gets
    // SM slots as they free, and a pass's tail is one window deep (measured
    // against a grid-strided 3 CTAs per SM: fiber passes 2.90 -> 2.50 ms,
    // remap 1.54 -> 1.33 ms per 3-mode sweep).  A pass capped beside the
    // MTTKRP keeps its grid-strided CTAs (replay_cap per SM).
    const uint32_t grid = p.replay_cap > 0
        ? std::max(1u, std::min(L.nwin, (uint32_t)(std::max(1, per_sm) * p.sms)))
        : std::max(1u, L.nwin);
    kern<<<grid, kReplayThreads, smem, p.stream>>>(slab_in(in, p.N), slab_out(out, p.N), L.wins,
                                                   L.nwin, cs.inv, cs.tab, cs.key_mode, cs.shift,
                                                   cs.mask, cs.nb, (uint32_t)p.nnz, p.err_flag);
    DGPU_CUDA(cudaGetLastError());
    return DGPU_OK;
}

// Window size of the scatter for N modes (host side).
uint32_t scatter_window_host(int N) {
    return N <= 4 ? (uint32_t)DGPU_SCAT_WINDOW : (uint32_t)DGPU_SCAT_WINDOW / 2u;
}

}  // namespace

void free_partlist(PartList& l) {
    if (l.own_tiles) dev_free(l.tiles);
    dev_free(l.chunks);
    dev_free(l.segs);
    dev_free(l.order);
    dev_free(l.wins);
    dev_free(l.tile_pre);
    dev_free(l.tile_wb);
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
        // chunks_per_sm (default 4) chunks per SM of near-equal element
        // counts (cut where the running total crosses the next multiple of
        // total / want), so the chunk count divides evenly over 1 or 2
        // resident scatter CTAs per SM
        uint64_t total = 0;
        for (const Tile& t : tiles) total += t.count;
        const uint64_t per_sm = (uint64_t)std::max(1, std::min(32, p.chunks_per_sm));
        const uint64_t want = std::max<uint64_t>(
            1, std::min<uint64_t>(per_sm * (uint64_t)p.sms, (total + kTile - 1) / kTile));
        Seg s{0, 0, 0, 0};
        uint32_t t0 = 0;
        uint64_t acc = 0;
        for (uint32_t t = 0; t < tiles.size(); ++t) {
            acc += tiles[t].count;
            const uint64_t cut = (ch.size() + 1) * total / want;
            if (acc >= cut || t + 1 == tiles.size()) {
                ch.push_back(Chunk{t0, t + 1, 0, 0});
                t0 = t + 1;
            }
        }
        s.chunk_end = (uint32_t)ch.size();
        sg.push_back(s);
    } else {
        const uint32_t per_chunk = (uint32_t)std::max(
            1, std::min((int)kSegChunkTilesMax, p.seg_chunk_tiles));
        const uint32_t nseg = (uint32_t)seg_base.size();
        sg.assign(nseg, Seg{0, 0, 0, 0});
        for (uint32_t s = 0; s < nseg; ++s) sg[s].base = seg_base[s];
        uint32_t t = 0;
        for (uint32_t s = 0; s < nseg; ++s) {
            sg[s].chunk_begin = (uint32_t)ch.size();
            while (t < tiles.size() && seg_of_tile[t] == s) {
                const uint32_t t0 = t;
                while (t < tiles.size() && seg_of_tile[t] == s && t - t0 < per_chunk) ++t;
                ch.push_back(Chunk{t0, t, s, 0});
            }
            sg[s].chunk_end = (uint32_t)ch.size();
        }
    }
    // chunks whose tiles are consecutive slab ranges
    for (Chunk& c : ch) {
        bool contiguous = true;
        for (uint32_t t = c.tile_begin; t + 1 < c.tile_end && contiguous; ++t)
            contiguous = tiles[t + 1].begin == tiles[t].begin + tiles[t].count;
        c.contiguous = contiguous ? 1u : 0u;
    }
    // work order of the persistent scatter: largest chunks first
    std::vector<uint64_t> csize(ch.size(), 0);
    for (size_t c = 0; c < ch.size(); ++c)
        for (uint32_t t = ch[c].tile_begin; t < ch[c].tile_end; ++t) csize[c] += tiles[t].count;
    std::vector<uint32_t> order(ch.size());
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return csize[a] > csize[b]; });
    // the scatter's windows (W-element pieces of each tile) and tile offsets
    // in list order: the layout of a recorded pass
    const uint32_t W = scatter_window_host(p.N);
    std::vector<uint32_t> pre(tiles.size()), wb(tiles.size());
    std::vector<uint4> wins;
    uint64_t acc = 0;
    for (size_t t = 0; t < tiles.size(); ++t) {
        pre[t] = (uint32_t)acc;
        wb[t] = (uint32_t)wins.size();
        for (uint32_t w0 = 0; w0 < tiles[t].count; w0 += W)
            wins.push_back(make_uint4(tiles[t].begin + w0, (uint32_t)acc + w0,
                                      std::min(W, tiles[t].count - w0), 0u));
        acc += tiles[t].count;
    }
    out.total = acc;
    out.nwin = (uint32_t)wins.size();
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
    DGPU_TRY(dev_alloc(p, (void**)&out.order, std::max<size_t>(1, ch.size()) * sizeof(uint32_t)));
    DGPU_TRY(dev_alloc(p, (void**)&out.wins, std::max<size_t>(1, wins.size()) * sizeof(uint4)));
    DGPU_TRY(dev_alloc(p, (void**)&out.tile_pre, std::max<size_t>(1, pre.size()) * sizeof(uint32_t)));
    DGPU_TRY(dev_alloc(p, (void**)&out.tile_wb, std::max<size_t>(1, wb.size()) * sizeof(uint32_t)));
    if (!wb.empty())
        DGPU_CUDA(cudaMemcpyAsync(out.tile_wb, wb.data(), wb.size() * sizeof(uint32_t),
                                  cudaMemcpyHostToDevice, p.stream));
    if (!wins.empty())
        DGPU_CUDA(cudaMemcpyAsync(out.wins, wins.data(), wins.size() * sizeof(uint4),
                                  cudaMemcpyHostToDevice, p.stream));
    if (!pre.empty())
        DGPU_CUDA(cudaMemcpyAsync(out.tile_pre, pre.data(), pre.size() * sizeof(uint32_t),
                                  cudaMemcpyHostToDevice, p.stream));
    if (!ch.empty()) {
        DGPU_CUDA(cudaMemcpyAsync(out.chunks, ch.data(), ch.size() * sizeof(Chunk),
                                  cudaMemcpyHostToDevice, p.stream));
        DGPU_CUDA(cudaMemcpyAsync(out.order, order.data(), order.size() * sizeof(uint32_t),
                                  cudaMemcpyHostToDevice, p.stream));
    }
    DGPU_CUDA(cudaMemcpyAsync(out.segs, sg.data(), sg.size() * sizeof(Seg), cudaMemcpyHostToDevice,
                              p.stream));
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    return DGPU_OK;
}

// Recording buffers of a slot (a 2-byte source element per listed slot and
// a destination per window and bucket), grown only while the device keeps
// at least a quarter of its memory free; a slot without them runs its
// ranked scatter on the kept tables.
static int reserve_recording(Plan& p, const PartList& L, uint32_t nb, PartCacheSlot& cs) {
    const size_t tab_n = (size_t)L.nwin * nb;
    if (cs.inv_cap >= L.total && cs.tab_cap >= tab_n) return DGPU_OK;
    dev_free(cs.inv);
    dev_free(cs.tab);
    cs.inv = nullptr;
    cs.tab = nullptr;
    cs.inv_cap = cs.tab_cap = 0;
    size_t free_b = 0, total_b = 0;
    DGPU_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t need = (size_t)L.total * sizeof(uint16_t) + tab_n * sizeof(uint32_t) + 512;
    if (free_b < need || free_b - need < total_b / 4) return DGPU_OK;
    if (dev_alloc(p, (void**)&cs.inv, (size_t)L.total * sizeof(uint16_t)) != DGPU_OK ||
        dev_alloc(p, (void**)&cs.tab, tab_n * sizeof(uint32_t)) != DGPU_OK) {
        dev_free(cs.inv);
        dev_free(cs.tab);
        cs.inv = nullptr;
        cs.tab = nullptr;
        return DGPU_OK;                          // no recording: not an error
    }
    cs.inv_cap = L.total;
    cs.tab_cap = tab_n;
    return DGPU_OK;
}

// Histogram + scans of one partition pass.  The offsets go to the plan's
// shared scratch, or, given a cache slot that is not valid while the stream
// is not being captured, to the slot, which becomes valid.  In check mode a
// valid slot's tables are compared with freshly computed ones (fault flag
// kErrPartCache on a difference).  *off / *base receive the tables to use.
static int compute_offsets(Plan& p, const Slab& in, const PartList& L, int key_mode,
                           int key_shift, uint32_t key_mask, uint32_t nb, PartCacheSlot* cs,
                           bool hit, const uint32_t** off_out, const uint32_t** base_out,
                           bool* filled)
{
    *filled = false;
    const size_t off_n = (size_t)L.nchunks * nb, base_n = (size_t)L.nsegs * nb;
    DGPU_TRY(ensure_part_scratch(p, off_n, base_n));
    uint32_t* off = p.part_off;
    uint32_t* base = p.part_base;
    bool fill = false;
    if (cs && !hit) {
        cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
        DGPU_CUDA(cudaStreamIsCapturing(p.stream, &cst));
        if (cst == cudaStreamCaptureStatusNone) {
            cs->valid = false;
            if (cs->off_cap < off_n) {
                dev_free(cs->off);
                cs->off = nullptr;
                cs->off_cap = 0;
                DGPU_TRY(dev_alloc(p, (void**)&cs->off, off_n * sizeof(uint32_t)));
                cs->off_cap = off_n;
            }
            if (cs->base_cap < base_n) {
                dev_free(cs->base);
                cs->base = nullptr;
                cs->base_cap = 0;
                DGPU_TRY(dev_alloc(p, (void**)&cs->base, base_n * sizeof(uint32_t)));
                cs->base_cap = base_n;
            }
            off = cs->off;
            base = cs->base;
            fill = true;
        }
    }
    const double elem = (double)p.nnz;
    {
        LaunchTimer t(p, p.part_fiber ? KK_FIB_HIST : KK_PART_HIST,
                      elem * 4.0 + (double)L.nchunks * nb * 4.0);
        // one histogram copy per warp while 32 copies fit in 48 KB
        const int copies = (int)std::max<uint32_t>(1u, std::min<uint32_t>(kHistThreads / 32,
                                                                          12288u / nb));
        k_chunk_hist<<<L.nchunks, kHistThreads, (size_t)copies * nb * sizeof(uint32_t), p.stream>>>(
            in.idx[key_mode], L.tiles, L.chunks, key_shift, key_mask, nb, copies, p.part_cnt);
        DGPU_CUDA(cudaGetLastError());
    }
    {
        LaunchTimer t(p, p.part_fiber ? KK_FIB_SCAN : KK_PART_SCAN, (double)L.nchunks * nb * 8.0);
        dim3 g(L.nsegs, (nb + 31) / 32);
        k_col_scan<<<g, 1024, 0, p.stream>>>(p.part_cnt, L.segs, nb, off, base);
        k_bucket_scan<<<L.nsegs, 1024, 0, p.stream>>>(base, L.segs, nb);
        DGPU_CUDA(cudaGetLastError());
    }
    if (hit) {
        // check mode: the kept tables must equal this sweep's
        const uint32_t grid = (uint32_t)std::min<size_t>(4u * (uint32_t)p.sms, (off_n + 255) / 256);
        k_cmp_tables<<<std::max(1u, grid), 256, 0, p.stream>>>(cs->off, off, off_n, p.err_flag);
        k_cmp_tables<<<1, 256, 0, p.stream>>>(cs->base, base, base_n, p.err_flag);
        DGPU_CUDA(cudaGetLastError());
    }
    if (fill) {
        cs->valid = true;
        cs->list = &L;
        cs->lists_gen = p.lists_gen;
        cs->key_mode = key_mode;
        cs->shift = key_shift;
        cs->mask = key_mask;
        cs->nb = nb;
        cs->replay = false;
        ++p.tables_gen;              // graphs kept over older tables recapture
        *filled = true;
    }
    *off_out = off;
    *base_out = base;
    return DGPU_OK;
}

int stable_partition(Plan& p, const Slab& in, const PartList& L, int key_mode, int key_shift,
                     uint32_t key_mask, uint32_t nb, const Slab& out)
{
    PartCacheSlot* cs = p.pc_slot;
    p.pc_slot = nullptr;
    if (L.nchunks == 0) return DGPU_OK;
    if (nb == 0 || nb > kMaxBuckets) {
        set_error("stable_partition: %u buckets (max %u)", nb, kMaxBuckets);
        return DGPU_ERR_ARG;
    }
    // a PingPong pass past the slab's first cycle reuses its kept tables
    const bool hit = cs && cs->valid && cs->list == &L && cs->lists_gen == p.lists_gen &&
                     cs->key_mode == key_mode && cs->shift == key_shift &&
                     cs->mask == key_mask && cs->nb == nb;
    const uint32_t* off = nullptr;
    const uint32_t* base = nullptr;
    const PartCacheSlot* rec = nullptr;       // record this pass into the slot
    if (hit && !p.part_cache_check) {
        off = cs->off;
        base = cs->base;
    } else {
        bool filled = false;
        DGPU_TRY(compute_offsets(p, in, L, key_mode, key_shift, key_mask, nb, cs, hit, &off, &base,
                                 &filled));
        // a PingPong pass whose tables are not kept for the next sweep
        if (p.pc_mode >= 0 && !(cs && cs->valid)) ++p.pc_uncached;
        if (filled && p.part_replay) {
            DGPU_TRY(reserve_recording(p, L, nb, *cs));
            if (cs->inv_cap >= L.total && cs->tab_cap >= (size_t)L.nwin * nb) rec = cs;
        }
    }
    const double row_bytes = 4.0 + 4.0 * p.N;
    const double elem = (double)L.total;
    if (hit && cs->replay) {
        // algorithmic bytes: the records read and written (the recorded
        // slots and destinations, 6 bytes per element, are overhead)
        LaunchTimer t(p, p.part_fiber ? KK_FIB_SCATTER : KK_PART_SCATTER,
                      elem * 2.0 * row_bytes);
        switch (p.N) {
#define DGPU_RP(NN) case NN: return launch_replay<NN>(p, in, out, L, *cs)
            DGPU_RP(2); DGPU_RP(3); DGPU_RP(4); DGPU_RP(5); DGPU_RP(6); DGPU_RP(7); DGPU_RP(8);
#undef DGPU_RP
            default: break;
        }
        set_error("stable_partition: %d modes unsupported", p.N);
        return DGPU_ERR_ARG;
    }
    LaunchTimer t(p, p.part_fiber ? KK_FIB_SCATTER : KK_PART_SCATTER,
                  elem * 2.0 * row_bytes + (double)L.nchunks * nb * 4.0);
    int rc = DGPU_ERR_ARG;
    switch (p.N) {
#define DGPU_SC(NN) case NN: rc = launch_scatter<NN>(p, in, out, L, key_mode, key_shift, key_mask, nb, off, base, rec); break
        DGPU_SC(2); DGPU_SC(3); DGPU_SC(4); DGPU_SC(5); DGPU_SC(6); DGPU_SC(7); DGPU_SC(8);
#undef DGPU_SC
        default:
            set_error("stable_partition: %d modes unsupported", p.N);
            return DGPU_ERR_ARG;
    }
    if (rc == DGPU_OK && rec) cs->replay = true;
    return rc;
}

// The kept-table slot of LSD pass k of the running PingPong step's fiber
// sort (kind 0) or remap (kind 1); none outside a PingPong step, before the
// slab has been through one cycle of modes, or with the cache off.
static PartCacheSlot* cache_slot(Plan& p, int kind, int k) {
    if (p.pc_mode < 0 || k >= kPartCachePasses || p.pp_transitions < (uint64_t)p.N) return nullptr;
    return &p.pcache[p.pc_mode][kind][k];
}

int stable_sort_pingpong(Plan& p, int a, int b, const PartList& first, int key_mode,
                         int key_shift, uint64_t key_limit, int* result, int k0, int k1)
{
    int bits = 0;
    while (bits < 32 && ((uint64_t)1 << bits) < key_limit) ++bits;
    if (key_limit <= 1) bits = 1;
    const int digit = std::max(1, std::min(kDigitBits, p.sort_digit_bits));
    int passes = (bits + digit - 1) / digit;
    if (passes < 1) passes = 1;
    const int dbits = (bits + passes - 1) / passes;
    int src = a, dst = b;
    const int kend = k1 < 0 ? passes : std::min(passes, k1);
    for (int k = k0; k < kend; ++k) {
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
        p.pc_slot = cache_slot(p, 1, k);
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
    const int digit = std::max(1, std::min(kDigitBits, p.fiber_digit_bits));
    const int passes = (bits + digit - 1) / digit;
    const int dbits = (bits + passes - 1) / passes;
    int a = src, b = other;
    p.part_fiber = 1;
    for (int k = 0; k < passes; ++k) {
        const int sh = k * dbits;
        const int hi = std::min(bits, sh + dbits);
        const uint32_t mask = (1u << (hi - sh)) - 1u;
        p.pc_slot = cache_slot(p, 0, k);
        const int rc = stable_partition(p, p.slab[a], p.fib[n], n, sh, mask, mask + 1, p.slab[b]);
        if (rc != DGPU_OK) { p.part_fiber = 0; return rc; }
        std::swap(a, b);
    }
    p.part_fiber = 0;
    *result = a;
    return DGPU_OK;
}

}  // namespace dgpu
