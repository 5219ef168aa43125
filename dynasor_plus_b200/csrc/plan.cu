// ============================================================================
//  plan.cu -- FLYCOO plan construction on the device (replaces the FLYCOO
//  part of build_flycoo, src/dynasor_preprocess.cpp:2013-2163).
//
//    host    geometry: m_n = pick_mn(I_n, T), shift, K_n, kernel class
//            [src/dynasor_preprocess.cpp:87-99, 2031-2048, 2087-2095]
//    device  shard histogram of every mode + index range check
//            [sort_and_count_all pass A, :153-174]
//    host    greedy LPT schedule from the counts, shard_begin/end
//            [:291-323, :363-384]; work tiles in processing order
//    device  stable scatter into mode-0 shard order [pass B, :212-241]
//    device  NCopy copies (remap chain + fiber sorts) when requested
//            [:1740-1790]
//
//  The LPT step uses std::sort with the reference's comparator so ties
//  resolve identically (libstdc++ introsort), and the same (load, tid)
//  min-heap, which makes the processing order -- and therefore the remap
//  permutation -- identical to the reference's for the same worker count.
// ============================================================================
#include "dgpu_internal.h"

#include <atomic>

#include <algorithm>
#include <functional>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <queue>

namespace dgpu {


// ----------------------------------------------------------------------------
//  errors
// ----------------------------------------------------------------------------
static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
const char* last_error() { return g_err; }

// ----------------------------------------------------------------------------
//  memory
// ----------------------------------------------------------------------------
int dev_alloc(Plan& p, void** ptr, size_t bytes) {
    *ptr = nullptr;
    if (bytes == 0) bytes = 256;
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
        return DGPU_ERR_NOMEM;
    }
    p.device_bytes += bytes;
    return DGPU_OK;
}

void dev_free(void* ptr) {
    if (ptr) cudaFree(ptr);
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int slab_alloc(Plan& p, Slab& s) {
    const size_t vb = align256(p.nnz * sizeof(float));
    const size_t ib = align256(p.nnz * sizeof(uint32_t));
    s.bytes = vb + (size_t)p.N * ib;
    DGPU_TRY(dev_alloc(p, &s.raw, s.bytes));
    char* c = static_cast<char*>(s.raw);
    s.vals = reinterpret_cast<float*>(c);
    c += vb;
    for (int n = 0; n < p.N; ++n) {
        s.idx[n] = reinterpret_cast<uint32_t*>(c);
        c += ib;
    }
    return DGPU_OK;
}

int sync_checked(Plan& p) {
    int flag = 0;
    if (p.err_flag)
        DGPU_CUDA(cudaMemcpyAsync(&flag, p.err_flag, sizeof(int), cudaMemcpyDeviceToHost, p.stream));
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    if (flag) {
        DGPU_CUDA(cudaMemsetAsync(p.err_flag, 0, sizeof(int), p.stream));
        DGPU_CUDA(cudaStreamSynchronize(p.stream));
        set_error("device fault flag 0x%x: %s", flag,
                  (flag & 0x100) ? "a partition kernel's bulk copy did not complete in time"
                  : (flag & 0x200) ? "a partition kernel computed an out-of-range slot"
                  : (flag & 0x1000) ? "a kept partition offset table differs from a recomputed one"
                                    : "a device-side check failed");
        return DGPU_ERR_DEVICE;
    }
    return DGPU_OK;
}

SlabPtrs slab_in(const Slab& s, int N) {
    SlabPtrs r{};
    r.vals = s.vals;
    for (int n = 0; n < N; ++n) r.idx[n] = s.idx[n];
    return r;
}
SlabOut slab_out(const Slab& s, int N) {
    SlabOut r{};
    r.vals = s.vals;
    for (int n = 0; n < N; ++n) r.idx[n] = s.idx[n];
    return r;
}

// ----------------------------------------------------------------------------
//  optional per-launch timing
// ----------------------------------------------------------------------------
static cudaEvent_t pool_get(Plan& p) {
    if (!p.event_pool.empty()) {
        cudaEvent_t e = p.event_pool.back();
        p.event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}

LaunchTimer::LaunchTimer(Plan& pl, int k, double b) : p(pl), kind(k), bytes(b) {
    if (!p.timing) return;
    a = pool_get(p);
    if (a) cudaEventRecord(a, p.stream);
}

LaunchTimer::~LaunchTimer() {
    if (!p.timing || !a) return;
    cudaEvent_t b = pool_get(p);
    if (!b) { p.event_pool.push_back(a); return; }
    cudaEventRecord(b, p.stream);
    p.pending.push_back({kind, a, b, bytes});
    if (p.pending.size() > 4096) timing_collect(p);
}

int timing_collect(Plan& p) {
    if (p.pending.empty()) return DGPU_OK;
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    for (auto& t : p.pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t.a, t.b);
        p.t_ms[t.kind] += ms;
        p.t_bytes[t.kind] += t.bytes;
        p.t_launches[t.kind] += 1;
        p.event_pool.push_back(t.a);
        p.event_pool.push_back(t.b);
    }
    p.pending.clear();
    return DGPU_OK;
}

uint64_t next_plan_serial() {
    static std::atomic<uint64_t> counter{1};
    return counter.fetch_add(1);
}

Plan::~Plan() {
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    // internal streams are joined into `stream` before every call returns;
    // after a failed call some of their work may not be, so wait for them
    // before freeing anything they may still read
    for (cudaStream_t s2 : {copy_stream, side_stream, ovl_stream})
        if (s2) cudaStreamSynchronize(s2);
    for (auto& t : pending) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
    for (auto e : event_pool) cudaEventDestroy(e);
    for (auto& s : slab) dev_free(s.raw);
    for (int n = 0; n < kMaxModes; ++n) {
        free_partlist(proc[n]);
        free_partlist(fib[n]);
        dev_free(tiles_d[n]);
        dev_free(run_tiles_d[n]);
        dev_free(Y[n]);
        dev_free(Yhat[n]);
        dev_free(Yb[n]);
    }
    free_partlist(ident);
    dev_free(part_cnt);
    dev_free(part_off);
    dev_free(part_base);
    for (auto& per_mode : pcache)
        for (auto& per_kind : per_mode)
            for (PartCacheSlot& c : per_kind) {
                dev_free(c.off);
                dev_free(c.base);
                dev_free(c.inv);
                dev_free(c.tab);
            }
    dev_free(err_flag);
    dev_free(part_ctr);
    dev_free(lambda);
    dev_free(la_work);
    dev_free(la_f32);
    dev_free(mkeys);
    dev_free(mvals);
    if (cp_loop_exec) cudaGraphExecDestroy(cp_loop_exec);
    if (cp_batch_exec) cudaGraphExecDestroy(cp_batch_exec);
    dev_free(grad_buf);
    dev_free(model_buf);
    for (int k = 0; k < 2; ++k) {
        if (stage_host[k]) cudaFreeHost(stage_host[k]);
        if (stage_ev[k]) cudaEventDestroy(stage_ev[k]);
    }
    dev_free(cp_st);
    if (cp_fit_host) cudaFreeHost(cp_fit_host);
    for (auto e : cp_ev) cudaEventDestroy(e);
    for (auto e : cp_fork) cudaEventDestroy(e);
    for (auto e : cp_join) cudaEventDestroy(e);
    if (copy_stream) { cudaStreamSynchronize(copy_stream); cudaStreamDestroy(copy_stream); }
    if (side_stream) { cudaStreamSynchronize(side_stream); cudaStreamDestroy(side_stream); }
    if (ovl_stream) { cudaStreamSynchronize(ovl_stream); cudaStreamDestroy(ovl_stream); }
    if (ovl_fork) cudaEventDestroy(ovl_fork);
    if (ovl_join) cudaEventDestroy(ovl_join);
    if (ovl_tail) cudaEventDestroy(ovl_tail);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

// ----------------------------------------------------------------------------
//  geometry helpers (src/dynasor_preprocess.cpp:69-99)
// ----------------------------------------------------------------------------
static uint32_t round_up_pow2(uint32_t x) {
    if (x <= 1) return 1;
    uint32_t r = 1;
    while (r < x) r <<= 1;
    return r;
}
static int log2_ceil(uint32_t x) {
    int k = 0;
    while ((uint32_t(1) << k) < x) ++k;
    return k;
}
static uint32_t rows_per_shard(uint32_t I, int T) {
    if (I <= (uint32_t)T) return 1;
    uint32_t mn = I / ((uint32_t)T * 4u);
    mn = std::max(mn, 1u);
    mn = std::max(mn, 16u);
    mn = std::min(mn, 16384u);
    if (mn > I) mn = I;
    return round_up_pow2(mn);
}

// ----------------------------------------------------------------------------
//  layout from the device-memory budget (dyn_plan_storage,
//  src/dynasor_preprocess.cpp:951-1104): the same rule with device memory in
//  place of host RAM -- usable = 70% of free memory less a headroom of
//  max(2 GiB, 25% of total); NCopy when its footprint plus overhead fits,
//  else PingPong.
// ----------------------------------------------------------------------------
static int choose_layout(Plan& p) {
    size_t free_b = 0, total_b = 0;
    DGPU_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const double slab = (double)p.nnz * (4.0 + 4.0 * p.N) + 256.0 * (p.N + 1);
    double factors = 0.0;
    for (int n = 0; n < p.N; ++n)
        factors += (double)p.dims[n] * p.Rp * 4.0 * (p.precision == DGPU_PREC_BF16 ? 2.5 : 2.0);
    // partition scratch (chunk x bucket tables) and slack
    const double overhead = factors + 64.0 * 1024 * 1024 + 0.05 * slab;
    const double headroom = std::max(2.0 * (1ull << 30), 0.25 * (double)total_b);
    const double usable = 0.70 * (double)free_b;
    const double budget = usable > headroom ? usable - headroom : 0.0;
    const double ncopy_need = (double)(p.N + 1) * slab + overhead;
    p.layout = ncopy_need <= budget ? DGPU_LAYOUT_NCOPY : DGPU_LAYOUT_PINGPONG;
    return DGPU_OK;
}

// ----------------------------------------------------------------------------
//  device: per-mode shard histograms + index range check
// ----------------------------------------------------------------------------
struct Geom {
    uint32_t dims[kMaxModes];
    int      shift[kMaxModes];
    uint32_t binoff[kMaxModes];
};

__global__ void k_shard_counts(const __grid_constant__ SlabPtrs in, int N, uint64_t nnz, Geom g, uint32_t total,
                               int use_smem, unsigned long long* __restrict__ counts,
                               int* __restrict__ err)
{
    extern __shared__ uint32_t h[];
    if (use_smem) {
        for (uint32_t b = threadIdx.x; b < total; b += blockDim.x) h[b] = 0;
        __syncthreads();
    }
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        for (int n = 0; n < N; ++n) {
            const uint32_t r = in.idx[n][i];
            if (r >= g.dims[n]) {
                atomicExch(err, 1);
                continue;
            }
            const uint32_t bin = g.binoff[n] + (r >> g.shift[n]);
            if (use_smem) atomicAdd(&h[bin], 1u);
            else atomicAdd(&counts[bin], 1ull);
        }
    }
    if (use_smem) {
        __syncthreads();
        for (uint32_t b = threadIdx.x; b < total; b += blockDim.x)
            if (h[b]) atomicAdd(&counts[b], (unsigned long long)h[b]);
    }
}

// ----------------------------------------------------------------------------
//  host: LPT schedule and tiles
// ----------------------------------------------------------------------------
static void build_schedule(Plan& p) {
    p.sched.assign(p.N, std::vector<std::vector<uint32_t>>(p.T));
    for (int n = 0; n < p.N; ++n) {
        const uint64_t* cn = p.count[n].data();
        std::vector<uint32_t> order(p.K[n]);
        std::iota(order.begin(), order.end(), 0u);
        std::sort(order.begin(), order.end(),
                  [&](uint32_t a, uint32_t b) { return cn[a] > cn[b]; });
        using QE = std::pair<uint64_t, int>;
        std::priority_queue<QE, std::vector<QE>, std::greater<QE>> heap;
        for (int t = 0; t < p.T; ++t) heap.push({0ull, t});
        for (uint32_t s : order) {
            if (cn[s] == 0) continue;
            const QE top = heap.top();
            heap.pop();
            p.sched[n][top.second].push_back(s);
            heap.push({top.first + cn[s], top.second});
        }
    }
}

static void build_tiles(Plan& p) {
    p.tiles_h.assign(p.N, {});
    for (int n = 0; n < p.N; ++n) {
        auto& v = p.tiles_h[n];
        for (int t = 0; t < p.T; ++t)
            for (uint32_t s : p.sched[n][t]) {
                const uint64_t b = p.sbeg[n][s], e = p.send[n][s];
                for (uint64_t x = b; x < e; x += kTile) {
                    Tile tl;
                    tl.begin = (uint32_t)x;
                    tl.count = (uint32_t)std::min<uint64_t>(kTile, e - x);
                    tl.shard = s;
                    tl.seg_first = 0;
                    v.push_back(tl);
                }
            }
    }
}

static int upload_tiles(Plan& p, const std::vector<Tile>& h, Tile** d) {
    DGPU_TRY(dev_alloc(p, (void**)d, std::max<size_t>(1, h.size()) * sizeof(Tile)));
    if (!h.empty())
        DGPU_CUDA(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(Tile),
                                  cudaMemcpyHostToDevice, p.stream));
    return DGPU_OK;
}

// Tiles of mode n in slab order (shard 0, 1, ...) with their segment
// bookkeeping, for the per-shard fiber sort.
static int build_fiber_tiles(Plan& p, int n) {
    std::vector<Tile> v;
    std::vector<uint32_t> seg_of, base(p.K[n], 0);
    for (uint32_t s = 0; s < p.K[n]; ++s) {
        const uint64_t b = p.sbeg[n][s], e = p.send[n][s];
        base[s] = (uint32_t)b;
        const uint32_t first = (uint32_t)v.size();
        for (uint64_t x = b; x < e; x += kTile) {
            Tile tl;
            tl.begin = (uint32_t)x;
            tl.count = (uint32_t)std::min<uint64_t>(kTile, e - x);
            tl.shard = s;
            tl.seg_first = first;
            v.push_back(tl);
            seg_of.push_back(s);
        }
    }
    return build_partlist(p, v, seg_of, base, p.fib[n], nullptr);
}

// ----------------------------------------------------------------------------
//  plan creation
// ----------------------------------------------------------------------------
// Scalars, stream and tuning knobs shared by both ways of building a plan.
static int plan_init(Plan& p, int N, uint64_t nnz, const uint32_t* dims, const dgpu_plan_opts& o) {
    p.N = N;
    p.nnz = nnz;
    p.T = o.threads;
    p.R = o.rank;
    p.Rp = (o.rank + 15) / 16 * 16;
    p.layout = o.layout;
    p.fiber = o.fiber ? 1 : 0;
    p.precision = o.precision;
    p.accum = o.accum;
    p.device = o.device;
    DGPU_CUDA(cudaSetDevice(p.device));
    if (!p.stream) {
        DGPU_CUDA(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking));
        p.own_stream = true;
    }
    DGPU_CUDA(cudaDeviceGetAttribute(&p.sms, cudaDevAttrMultiProcessorCount, p.device));
    // digit widths of the LSD partition passes (tuning knobs; the permutation
    // does not depend on them)
    if (const char* e = std::getenv("DGPU_SORT_DIGIT_BITS")) p.sort_digit_bits = std::atoi(e);
    if (const char* e = std::getenv("DGPU_FIBER_DIGIT_BITS")) p.fiber_digit_bits = std::atoi(e);
    if (const char* e = std::getenv("DGPU_MTTKRP_KERNEL")) p.mttkrp_kernel = std::atoi(e) == 1 ? 1 : 0;
    if (const char* e = std::getenv("DGPU_RANK_TILE")) p.rank_tile = std::atoi(e);
    if (const char* e = std::getenv("DGPU_OVERLAP")) p.overlap = std::atoi(e);
    if (const char* e = std::getenv("DGPU_REMAP_CTAS")) p.remap_ctas = std::max(1, std::atoi(e));
    if (const char* e = std::getenv("DGPU_PART_CACHE")) p.part_cache = std::atoi(e) != 0 ? 1 : 0;
    if (const char* e = std::getenv("DGPU_PART_CACHE_CHECK")) p.part_cache_check = std::atoi(e) != 0 ? 1 : 0;
    if (const char* e = std::getenv("DGPU_PART_REPLAY")) p.part_replay = std::atoi(e) != 0 ? 1 : 0;
    for (int n = 0; n < N; ++n) p.dims[n] = dims[n];
    return DGPU_OK;
}

// Shard geometry of mode n for `mn` (a power of two) rows per shard, and the
// kernel class from the average fiber length (src/dynasor_preprocess.cpp:
// 2087-2095).
static void plan_mode_geometry(Plan& p, int n, uint32_t mn) {
    p.mn[n] = mn;
    p.shift[n] = log2_ceil(mn);
    p.K[n] = (p.dims[n] + mn - 1) / mn;
    if (p.K[n] == 0) p.K[n] = 1;
    p.afl[n] = (double)p.nnz / (double)std::max<uint32_t>(1u, p.dims[n]);
    p.kclass[n] = p.afl[n] >= 32.0 ? 2 : (p.afl[n] >= 8.0 ? 1 : 0);
}

// Slabs: PingPong keeps primary + scratch; NCopy keeps N copies (+1 scratch
// while sorting).
static int plan_alloc_slabs(Plan& p) {
    const int nslab = (p.layout == DGPU_LAYOUT_NCOPY) ? std::max(p.N + 1, 2) : 2;
    if (nslab > kMaxModes) {
        set_error("NCopy with %d modes needs %d slabs (max %d)", p.N, nslab, kMaxModes);
        return DGPU_ERR_ARG;
    }
    for (int s = 0; s < nslab; ++s) DGPU_TRY(slab_alloc(p, p.slab[s]));
    DGPU_TRY(dev_alloc(p, (void**)&p.err_flag, sizeof(int)));
    DGPU_CUDA(cudaMemsetAsync(p.err_flag, 0, sizeof(int), p.stream));
    DGPU_TRY(dev_alloc(p, (void**)&p.part_ctr, sizeof(uint32_t)));
    return DGPU_OK;
}

// Per-mode shard histograms of slab `s` on the device (any element order),
// with every index checked against its mode size.
static int device_shard_counts(Plan& p, const Slab& s, std::vector<std::vector<uint64_t>>& out) {
    Geom g{};
    uint32_t total = 0;
    for (int n = 0; n < p.N; ++n) {
        g.dims[n] = p.dims[n];
        g.shift[n] = p.shift[n];
        g.binoff[n] = total;
        total += p.K[n];
    }
    unsigned long long* counts_d = nullptr;
    DGPU_TRY(dev_alloc(p, (void**)&counts_d, (size_t)total * 8));
    DGPU_CUDA(cudaMemsetAsync(counts_d, 0, (size_t)total * 8, p.stream));
    DGPU_CUDA(cudaMemsetAsync(p.err_flag, 0, sizeof(int), p.stream));
    const int use_smem = total <= 12288 ? 1 : 0;
    const unsigned blocks =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((p.nnz + 255) / 256, 148 * 8));
    k_shard_counts<<<blocks, 256, use_smem ? total * 4 : 0, p.stream>>>(
        slab_in(s, p.N), p.N, p.nnz, g, total, use_smem, counts_d, p.err_flag);
    DGPU_CUDA(cudaGetLastError());
    std::vector<unsigned long long> counts_h(total);
    int err_h = 0;
    DGPU_CUDA(cudaMemcpyAsync(counts_h.data(), counts_d, (size_t)total * 8,
                              cudaMemcpyDeviceToHost, p.stream));
    DGPU_CUDA(cudaMemcpyAsync(&err_h, p.err_flag, sizeof(int), cudaMemcpyDeviceToHost, p.stream));
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    dev_free(counts_d);
    p.device_bytes -= (size_t)total * 8;
    DGPU_CUDA(cudaMemsetAsync(p.err_flag, 0, sizeof(int), p.stream));
    if (err_h) {
        set_error("plan: an index is out of range of its mode size");
        return DGPU_ERR_INDEX;
    }
    out.assign(p.N, {});
    for (int n = 0; n < p.N; ++n)
        out[n].assign(counts_h.begin() + g.binoff[n], counts_h.begin() + g.binoff[n] + p.K[n]);
    return DGPU_OK;
}

// The MTTKRP's CTA tiles of mode n: consecutive processing-order tiles of
// one shard merged up to kRunTileMerge x kTile nonzeros (3-mode plans).  A
// longer slice per lane group cuts the row runs its ends share with
// neighbours (each flushed by an atomic) and the CTAs' start-up; measured on
// the 3-mode rank-32 Zipf tensor, MTTKRP per sweep: 4096-nonzero CTAs 3.31 ms
// (FP32) / 2.71 ms (BF16), 8192 3.20 / 2.55, 16384 3.31 ms FP32, and 2048
// (a tile split in two) 3.70 ms.  On the 4-mode rank-64 tensor merged pairs
// measured within 0.6% (NCopy sweep 27.3 -> 27.1 ms FP32, 20.6 ms BF16), so
// 4-mode plans keep kTile CTAs.  The partition passes keep kTile tiles.
constexpr uint32_t kRunTileMerge = 2;

static int upload_run_tiles(Plan& p, int n) {
    dev_free(p.run_tiles_d[n]);
    p.run_tiles_d[n] = nullptr;
    p.run_tiles_n[n] = 0;
    if (p.N != 3) return DGPU_OK;
    std::vector<Tile> m;
    for (const Tile& t : p.tiles_h[n]) {
        if (!m.empty() && m.back().shard == t.shard && m.back().begin + m.back().count == t.begin &&
            m.back().count + t.count <= kRunTileMerge * kTile)
            m.back().count += t.count;
        else
            m.push_back(t);
    }
    DGPU_TRY(upload_tiles(p, m, &p.run_tiles_d[n]));
    p.run_tiles_n[n] = (uint32_t)m.size();
    return DGPU_OK;
}

// The MTTKRP of mode n over its CTA tiles (the merged ones for the row-run
// kernel; the TMA gather kernel cuts tiles of at most kTile nonzeros).
static int launch_mttkrp_run(Plan& p, int n, const Slab& in) {
    if (p.run_tiles_d[n] && p.mttkrp_kernel != 1 && mttkrp_scheme(p, n) == DGPU_ACCUM_ROWRUN)
        return launch_mttkrp(p, n, in, p.run_tiles_d[n], p.run_tiles_n[n]);
    return launch_mttkrp(p, n, in, p.tiles_d[n], (uint32_t)p.tiles_h[n].size());
}

// Tiles, partition lists and fiber tile lists from the shard tables and the
// schedule.
static int plan_tables(Plan& p) {
    build_tiles(p);
    static const std::vector<uint32_t> kNone;
    for (int n = 0; n < p.N; ++n) {
        DGPU_TRY(upload_tiles(p, p.tiles_h[n], &p.tiles_d[n]));
        DGPU_TRY(build_partlist(p, p.tiles_h[n], kNone, kNone, p.proc[n], p.tiles_d[n]));
        DGPU_TRY(upload_run_tiles(p, n));
    }
    for (int n = 0; n < p.N; ++n)
        if (p.fiber && p.kclass[n] == 2) DGPU_TRY(build_fiber_tiles(p, n));
    std::vector<Tile> id;
    for (uint64_t x = 0; x < p.nnz; x += kTile) {
        Tile tl;
        tl.begin = (uint32_t)x;
        tl.count = (uint32_t)std::min<uint64_t>(kTile, p.nnz - x);
        tl.shard = 0;
        tl.seg_first = 0;
        id.push_back(tl);
    }
    return build_partlist(p, id, kNone, kNone, p.ident, nullptr);
}

int plan_rebuild_partlists(Plan& p) {
    static const std::vector<uint32_t> kNone;
    // graphs captured over the old lists must not run again: drop this
    // plan's, and bump the generation that every cached key carries (a
    // batch graph kept on another plan then no longer matches)
    ++p.tables_gen;
    ++p.lists_gen;                               // kept partition tables no longer match
    if (p.cp_loop_exec) { cudaGraphExecDestroy(p.cp_loop_exec); p.cp_loop_exec = nullptr; }
    if (p.cp_batch_exec) { cudaGraphExecDestroy(p.cp_batch_exec); p.cp_batch_exec = nullptr; }
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    for (int n = 0; n < p.N; ++n) {
        if (p.tiles_h[n].empty()) continue;
        DGPU_TRY(build_partlist(p, p.tiles_h[n], kNone, kNone, p.proc[n], p.tiles_d[n]));
        if (p.fib[n].chunks) DGPU_TRY(build_fiber_tiles(p, n));
    }
    if (!p.ident.chunks) return DGPU_OK;
    std::vector<Tile> id;
    for (uint64_t x = 0; x < p.nnz; x += kTile) {
        Tile tl;
        tl.begin = (uint32_t)x;
        tl.count = (uint32_t)std::min<uint64_t>(kTile, p.nnz - x);
        tl.shard = 0;
        tl.seg_first = 0;
        id.push_back(tl);
    }
    return build_partlist(p, id, kNone, kNone, p.ident, nullptr);
}

static int plan_factors(Plan& p) {
    for (int n = 0; n < p.N; ++n) {
        const size_t fb = (size_t)p.dims[n] * p.Rp * sizeof(float);
        DGPU_TRY(dev_alloc(p, (void**)&p.Y[n], fb));
        DGPU_TRY(dev_alloc(p, (void**)&p.Yhat[n], fb));
        DGPU_CUDA(cudaMemsetAsync(p.Y[n], 0, fb, p.stream));
        DGPU_CUDA(cudaMemsetAsync(p.Yhat[n], 0, fb, p.stream));
        if (p.precision == DGPU_PREC_BF16) {
            DGPU_TRY(dev_alloc(p, (void**)&p.Yb[n], fb / 2));
            DGPU_CUDA(cudaMemsetAsync(p.Yb[n], 0, fb / 2, p.stream));
        }
        p.yb_stale[n] = true;
    }
    DGPU_TRY(dev_alloc(p, (void**)&p.lambda, (size_t)p.Rp * sizeof(float)));
    return DGPU_OK;
}

int plan_build(Plan& p, const dgpu_tensor_desc& t, const dgpu_plan_opts& o) {
    DGPU_TRY(plan_init(p, t.num_modes, t.nnz, t.mode_size, o));
    // geometry
    for (int n = 0; n < p.N; ++n) {
        const uint32_t mn = (o.mn_target && o.mn_target[n] > 0) ? round_up_pow2(o.mn_target[n])
                                                                : rows_per_shard(p.dims[n], p.T);
        plan_mode_geometry(p, n, mn);
    }
    if (p.layout == DGPU_LAYOUT_AUTO) DGPU_TRY(choose_layout(p));
    DGPU_TRY(plan_alloc_slabs(p));

    // input COO -> slab[1] (the reference's loader order)
    const int in_slab = 1;
    DGPU_CUDA(cudaMemcpyAsync(p.slab[in_slab].vals, t.vals, p.nnz * sizeof(float),
                              cudaMemcpyHostToDevice, p.stream));
    for (int n = 0; n < p.N; ++n)
        DGPU_CUDA(cudaMemcpyAsync(p.slab[in_slab].idx[n], t.idx[n], p.nnz * sizeof(uint32_t),
                                  cudaMemcpyHostToDevice, p.stream));

    // shard histograms on the device -> shard tables, schedule, tiles
    DGPU_TRY(device_shard_counts(p, p.slab[in_slab], p.count));
    p.sbeg.assign(p.N, {});
    p.send.assign(p.N, {});
    for (int n = 0; n < p.N; ++n) {
        p.sbeg[n].resize(p.K[n]);
        p.send[n].resize(p.K[n]);
        uint64_t c = 0;
        for (uint32_t s = 0; s < p.K[n]; ++s) {
            p.sbeg[n][s] = c;
            c += p.count[n][s];
            p.send[n][s] = c;
        }
    }
    build_schedule(p);
    DGPU_TRY(plan_tables(p));

    if (p.layout == DGPU_LAYOUT_MORTON) {
        // keys + values replace the slabs (the shard tables above stay for
        // plan queries only)
        DGPU_TRY(morton_build(p, in_slab));
        p.cur = 0;
        p.next_mode = 0;
        DGPU_TRY(plan_factors(p));
        DGPU_TRY(sync_checked(p));
        return DGPU_OK;
    }

    // stable scatter of the input order into mode-0 shard order
    int res = 0;
    DGPU_TRY(stable_sort_pingpong(p, in_slab, 0, p.ident, 0, p.shift[0], p.K[0], &res));
    p.cur = res;
    p.next_mode = 0;
    p.pp_transitions = 0;

    if (p.layout == DGPU_LAYOUT_NCOPY) {
        // copy 0 lives in slab[0]; copy k = remap of copy k-1 by the mode
        // (k-1) processing order, keyed by the mode-k shard.  The spare
        // slab p.N is the LSD intermediate.
        if (p.cur != 0) {
            DGPU_CUDA(cudaMemcpyAsync(p.slab[0].raw, p.slab[p.cur].raw, p.slab[0].bytes,
                                      cudaMemcpyDeviceToDevice, p.stream));
        }
        for (int k = 1; k < p.N; ++k) {
            DGPU_CUDA(cudaMemcpyAsync(p.slab[k].raw, p.slab[k - 1].raw, p.slab[k].bytes,
                                      cudaMemcpyDeviceToDevice, p.stream));
            int r = 0;
            DGPU_TRY(stable_sort_pingpong(p, k, p.N, p.proc[k - 1], k, p.shift[k], p.K[k], &r));
            if (r != k)
                DGPU_CUDA(cudaMemcpyAsync(p.slab[k].raw, p.slab[r].raw, p.slab[k].bytes,
                                          cudaMemcpyDeviceToDevice, p.stream));
        }
        if (p.fiber) {
            for (int k = 0; k < p.N; ++k) {
                if (p.kclass[k] != 2) continue;
                int r = 0;
                DGPU_TRY(fiber_sort(p, k, k, p.N, &r));
                if (r != k)
                    DGPU_CUDA(cudaMemcpyAsync(p.slab[k].raw, p.slab[r].raw, p.slab[k].bytes,
                                              cudaMemcpyDeviceToDevice, p.stream));
            }
        }
    }
    DGPU_TRY(plan_factors(p));
    DGPU_TRY(sync_checked(p));
    return DGPU_OK;
}

// ----------------------------------------------------------------------------
//  plan from a .dnp image (runtime-only mode, src/dynasor_dnp.cpp:719-803):
//  the saved slab(s), shard tables and schedule are used as they are; the
//  device checks every index range, the per-shard counts, the shard order of
//  the processing slab(s) and, on fiber-sorted NCopy copies, the row order.
// ----------------------------------------------------------------------------
__global__ void k_check_order(const uint32_t* __restrict__ idx, const Tile* __restrict__ tiles,
                              int shift, const uint64_t* __restrict__ sbeg, int rows_sorted,
                              int* __restrict__ err)
{
    const Tile tl = tiles[blockIdx.x];
    for (uint32_t j = threadIdx.x; j < tl.count; j += blockDim.x) {
        const uint64_t i = (uint64_t)tl.begin + j;
        const uint32_t r = idx[i];
        if ((r >> shift) != tl.shard) atomicOr(err, 0x400);
        if (rows_sorted && i > sbeg[tl.shard] && idx[i - 1] > r) atomicOr(err, 0x800);
    }
}

static int check_order(Plan& p, int n, const Slab& s, int rows_sorted) {
    const uint32_t nt = (uint32_t)p.tiles_h[n].size();
    if (nt == 0) return DGPU_OK;
    uint64_t* sb = nullptr;
    DGPU_TRY(dev_alloc(p, (void**)&sb, (size_t)p.K[n] * 8));
    DGPU_CUDA(cudaMemcpyAsync(sb, p.sbeg[n].data(), (size_t)p.K[n] * 8, cudaMemcpyHostToDevice,
                              p.stream));
    DGPU_CUDA(cudaMemsetAsync(p.err_flag, 0, sizeof(int), p.stream));
    k_check_order<<<nt, 256, 0, p.stream>>>(s.idx[n], p.tiles_d[n], p.shift[n], sb, rows_sorted,
                                             p.err_flag);
    DGPU_CUDA(cudaGetLastError());
    int err_h = 0;
    DGPU_CUDA(cudaMemcpyAsync(&err_h, p.err_flag, sizeof(int), cudaMemcpyDeviceToHost, p.stream));
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    dev_free(sb);
    p.device_bytes -= (size_t)p.K[n] * 8;
    DGPU_CUDA(cudaMemsetAsync(p.err_flag, 0, sizeof(int), p.stream));
    if (err_h & 0x400) {
        set_error("dnp: slab %s is not in mode-%d shard order", p.layout == DGPU_LAYOUT_NCOPY ?
                  "copy" : "(PingPong)", n);
        return DGPU_ERR_IO;
    }
    if (err_h & 0x800) {
        set_error("dnp: NCopy copy %d is flagged fiber-sorted but its rows are not sorted", n);
        return DGPU_ERR_IO;
    }
    return DGPU_OK;
}

// A Morton file: keys and values are uploaded as they are and checked on
// the device (decode within range, re-encode to the same key, ascending);
// the decoded nonzeros give the shard tables for plan queries, then the
// slabs are released.
static int plan_build_dnp_morton(Plan& p, const DnpImage& img, const dgpu_plan_opts& o) {
    dgpu_plan_opts oo = o;
    oo.threads = img.threads;
    oo.layout = DGPU_LAYOUT_MORTON;
    DGPU_TRY(plan_init(p, img.N, img.nnz, img.dims, oo));
    uint64_t seen = 0;
    for (int n = 0; n < p.N; ++n) {
        const int pc = __builtin_popcountll(img.mmask[n]);
        if (pc == 0 || pc > 32 || pc != img.mbits[n] || (img.mmask[n] & seen)) {
            set_error("dnp: Morton mask of mode %d (%d bits, %u stated) is empty, too wide or "
                      "overlaps another mode's", n, pc, (unsigned)img.mbits[n]);
            return DGPU_ERR_IO;
        }
        seen |= img.mmask[n];
        p.mmask[n] = img.mmask[n];
        p.mbits[n] = img.mbits[n];
        plan_mode_geometry(p, n, rows_per_shard(p.dims[n], p.T));
    }
    DGPU_TRY(plan_alloc_slabs(p));
    DGPU_TRY(dev_alloc(p, (void**)&p.mkeys, p.nnz * sizeof(uint64_t)));
    DGPU_TRY(dev_alloc(p, (void**)&p.mvals, p.nnz * sizeof(float)));
    DGPU_CUDA(cudaMemcpyAsync(p.mkeys, img.mkeys.data(), p.nnz * sizeof(uint64_t),
                              cudaMemcpyHostToDevice, p.stream));
    DGPU_CUDA(cudaMemcpyAsync(p.mvals, img.mvals.data(), p.nnz * sizeof(float),
                              cudaMemcpyHostToDevice, p.stream));
    DGPU_TRY(morton_check_decode(p, 1));
    DGPU_TRY(device_shard_counts(p, p.slab[1], p.count));
    p.sbeg.assign(p.N, {});
    p.send.assign(p.N, {});
    for (int n = 0; n < p.N; ++n) {
        p.sbeg[n].resize(p.K[n]);
        p.send[n].resize(p.K[n]);
        uint64_t c = 0;
        for (uint32_t s = 0; s < p.K[n]; ++s) {
            p.sbeg[n][s] = c;
            c += p.count[n][s];
            p.send[n][s] = c;
        }
    }
    build_schedule(p);
    DGPU_TRY(plan_tables(p));
    DGPU_TRY(sync_checked(p));
    free_slabs(p);
    p.cur = 0;
    p.next_mode = 0;
    p.pp_transitions = 0;
    DGPU_TRY(plan_factors(p));
    DGPU_TRY(sync_checked(p));
    return DGPU_OK;
}

int plan_build_dnp(Plan& p, const DnpImage& img, const dgpu_plan_opts& o) {
    if (img.layout == DGPU_LAYOUT_MORTON) return plan_build_dnp_morton(p, img, o);
    dgpu_plan_opts oo = o;
    oo.threads = img.threads;
    oo.layout = img.layout;
    if (img.layout == DGPU_LAYOUT_NCOPY) {
        // the copies decide: fiber-sorted DenseFiber copies, or none
        bool any = false;
        for (int k = 0; k < img.N; ++k) any = any || img.fiber_sorted[k];
        oo.fiber = any ? 1 : 0;
    }
    DGPU_TRY(plan_init(p, img.N, img.nnz, img.dims, oo));
    for (int n = 0; n < p.N; ++n) {
        const uint32_t mn = img.mn[n];
        if (mn == 0 || (mn & (mn - 1)) != 0) {
            set_error("dnp: mode %d has %u rows per shard (not a power of two)", n, mn);
            return DGPU_ERR_IO;
        }
        plan_mode_geometry(p, n, mn);
        if (p.K[n] != img.K[n] || p.shift[n] != img.shift[n]) {
            set_error("dnp: mode %d shard geometry (K %u, shift %d) does not match its size %u "
                      "and %u rows per shard", n, img.K[n], img.shift[n], p.dims[n], mn);
            return DGPU_ERR_IO;
        }
        if (img.kclass[n] > 2) {
            set_error("dnp: mode %d kernel class %u unknown", n, img.kclass[n]);
            return DGPU_ERR_IO;
        }
        p.afl[n] = img.afl[n];
        p.kclass[n] = (int)img.kclass[n];
        if (img.layout == DGPU_LAYOUT_NCOPY &&
            (img.fiber_sorted[n] != 0) != (p.fiber && p.kclass[n] == 2)) {
            set_error("dnp: NCopy copy %d fiber-sorted flag %d does not match its kernel class %d",
                      n, (int)img.fiber_sorted[n], p.kclass[n]);
            return DGPU_ERR_IO;
        }
    }
    // shard tables: contiguous ranges covering the slab
    p.sbeg = img.sbeg;
    p.send = img.send;
    p.count.assign(p.N, {});
    for (int n = 0; n < p.N; ++n) {
        if (p.sbeg[n].size() != p.K[n] || p.send[n].size() != p.K[n]) {
            set_error("dnp: mode %d shard table size differs from %u shards", n, p.K[n]);
            return DGPU_ERR_IO;
        }
        uint64_t c = 0;
        p.count[n].resize(p.K[n]);
        for (uint32_t s = 0; s < p.K[n]; ++s) {
            if (p.sbeg[n][s] != c || p.send[n][s] < c) {
                set_error("dnp: mode %d shard %u range [%llu,%llu) is not contiguous", n, s,
                          (unsigned long long)p.sbeg[n][s], (unsigned long long)p.send[n][s]);
                return DGPU_ERR_IO;
            }
            p.count[n][s] = p.send[n][s] - c;
            c = p.send[n][s];
        }
        if (c != p.nnz) {
            set_error("dnp: mode %d shard ranges cover %llu of %llu nonzeros", n,
                      (unsigned long long)c, (unsigned long long)p.nnz);
            return DGPU_ERR_IO;
        }
    }
    // schedule: every non-empty shard exactly once, empty ones at most once
    p.sched = img.sched;
    for (int n = 0; n < p.N; ++n) {
        std::vector<uint8_t> seen(p.K[n], 0);
        if ((int)p.sched[n].size() != p.T) {
            set_error("dnp: mode %d schedule has %zu thread lists, expected %d", n,
                      p.sched[n].size(), p.T);
            return DGPU_ERR_IO;
        }
        for (const auto& lst : p.sched[n])
            for (uint32_t s : lst) {
                if (s >= p.K[n] || seen[s]) {
                    set_error("dnp: mode %d schedule names shard %u %s", n, s,
                              s >= p.K[n] ? "out of range" : "twice");
                    return DGPU_ERR_IO;
                }
                seen[s] = 1;
            }
        for (uint32_t s = 0; s < p.K[n]; ++s)
            if (!seen[s] && p.count[n][s]) {
                set_error("dnp: mode %d schedule omits non-empty shard %u", n, s);
                return DGPU_ERR_IO;
            }
    }
    DGPU_TRY(plan_alloc_slabs(p));
    const int ncopies = (img.layout == DGPU_LAYOUT_NCOPY) ? p.N : 1;
    for (int k = 0; k < ncopies; ++k) {
        Slab& d = p.slab[k];
        DGPU_CUDA(cudaMemcpyAsync(d.vals, img.vals[k].data(), p.nnz * sizeof(float),
                                  cudaMemcpyHostToDevice, p.stream));
        for (int m = 0; m < p.N; ++m)
            DGPU_CUDA(cudaMemcpyAsync(d.idx[m], img.idx[k][m].data(), p.nnz * sizeof(uint32_t),
                                      cudaMemcpyHostToDevice, p.stream));
        // index ranges and shard counts of every copy
        std::vector<std::vector<uint64_t>> cnt;
        DGPU_TRY(device_shard_counts(p, d, cnt));
        for (int n = 0; n < p.N; ++n)
            if (cnt[n] != p.count[n]) {
                set_error("dnp: %s %d holds shard counts of mode %d that differ from the shard "
                          "table", ncopies > 1 ? "copy" : "slab", k, n);
                return DGPU_ERR_IO;
            }
    }
    DGPU_TRY(plan_tables(p));
    if (img.layout == DGPU_LAYOUT_NCOPY) {
        for (int k = 0; k < p.N; ++k) DGPU_TRY(check_order(p, k, p.slab[k], img.fiber_sorted[k]));
    } else {
        DGPU_TRY(check_order(p, 0, p.slab[0], 0));
    }
    p.cur = 0;
    p.next_mode = 0;
    DGPU_TRY(plan_factors(p));
    DGPU_TRY(sync_checked(p));
    return DGPU_OK;
}

// One mode of the PingPong sweep: fiber sort (DenseFiber modes), MTTKRP,
// device remap for mode n+1.  src/dynasor.cpp:352-539.
// The PingPong mode with two hooks for callers that stream factors in and
// Yhat out: the MTTKRP waits for `waits` (the fiber sort before it needs no
// factor), and `after_mttkrp` is recorded once Yhat[n] is complete (the
// remap after it does not touch Yhat).
// One PingPong mode.  `after` (optional) enqueues work that needs this
// mode's Yhat but not the remapped slab (a CP-ALS factor update): it runs
// right after the MTTKRP on the MTTKRP's stream.
static int mode_pingpong_impl(Plan& p, int n, const cudaEvent_t* waits, int nwaits,
                              cudaEvent_t after_mttkrp, const std::function<int()>* after) {
    if (n != p.next_mode) {
        set_error("mttkrp_mode(%d): the slab is remapped for mode %d; modes must run in "
                  "order 0..N-1", n, p.next_mode);
        return DGPU_ERR_ORDER;
    }
    // the step's partition passes may use kept offset tables (stable_partition)
    struct PcScope {
        Plan& p;
        PcScope(Plan& q, int n) : p(q) { p.pc_mode = q.part_cache ? n : -1; }
        ~PcScope() { p.pc_mode = -1; p.pc_slot = nullptr; }
    } pc_scope(p, n);
    const int other = 1 - p.cur;
    if (p.fiber && p.kclass[n] == 2) {
        int r = 0;
        DGPU_TRY(fiber_sort(p, n, p.cur, other, &r));
        p.cur = r;
    }
    {
        const size_t yb = (size_t)p.dims[n] * p.Rp * sizeof(float);
        LaunchTimer t(p, KK_ZERO, (double)yb);
        DGPU_CUDA(cudaMemsetAsync(p.Yhat[n], 0, yb, p.stream));
    }
    for (int k = 0; k < nwaits; ++k) DGPU_CUDA(cudaStreamWaitEvent(p.stream, waits[k], 0));
    const int nm = (n + 1) % p.N;
    int r = 0;
    // overlap needs a one-pass remap: a second LSD pass would write back
    // into the slab the MTTKRP is reading
    const int digit = std::max(1, std::min(kDigitBits, p.sort_digit_bits));
    const bool one_pass = (uint64_t)p.K[nm] <= ((uint64_t)1 << digit);
    if (p.overlap == 0 || p.timing || (!one_pass && p.overlap != 2)) {
        DGPU_TRY(pingpong_drain(p));
        DGPU_TRY(launch_mttkrp_run(p, n, p.slab[p.cur]));
        if (after_mttkrp) DGPU_CUDA(cudaEventRecord(after_mttkrp, p.stream));
        if (after) DGPU_TRY((*after)());
        DGPU_TRY(stable_sort_pingpong(p, p.cur, 1 - p.cur, p.proc[n], nm, p.shift[nm], p.K[nm], &r));
    } else {
        // The MTTKRP and the remap both only read the live slab (the remap
        // writes the other one), so the MTTKRP runs on ovl_stream beside the
        // remap on the plan stream.  Each kernel alone fills the SMs'
        // registers.  Overlap 1 launches the MTTKRP first and the remap's
        // CTAs start as its last CTAs drain (measured 9.72 -> 9.61 ms per
        // sweep on the 64.7M-nonzero tensor, ranked passes).  Overlap 2
        // launches the remap's first pass first at remap_ctas CTAs per SM
        // when it is replayed, so the MTTKRP fills the rest of every SM
        // beside it (7.64 -> 7.38 ms, replayed passes).  The plan stream
        // waits for the MTTKRP before any pass that rewrites the slab it
        // reads (the next mode's fiber sort, a later LSD pass of the remap);
        // `after` stays on ovl_stream, beside the remap and the next fiber
        // sort, until pingpong_drain.
        if (!p.ovl_stream) {
            DGPU_CUDA(cudaStreamCreateWithFlags(&p.ovl_stream, cudaStreamNonBlocking));
            DGPU_CUDA(cudaEventCreateWithFlags(&p.ovl_fork, cudaEventDisableTiming));
            DGPU_CUDA(cudaEventCreateWithFlags(&p.ovl_join, cudaEventDisableTiming));
            DGPU_CUDA(cudaEventCreateWithFlags(&p.ovl_tail, cudaEventDisableTiming));
        }
        DGPU_CUDA(cudaEventRecord(p.ovl_fork, p.stream));
        DGPU_CUDA(cudaStreamWaitEvent(p.ovl_stream, p.ovl_fork, 0));
        const cudaStream_t main = p.stream;
        struct Restore {
            Plan& p;
            cudaStream_t s;
            ~Restore() { p.stream = s; p.replay_cap = 0; }
        } restore{p, main};
        // DGPU_OVERLAP=2: the remap's first pass is launched first with at
        // most remap_ctas CTAs per SM (when it is replayed), so the MTTKRP
        // launched next beside it fills the rest of every SM; later passes
        // rewrite the slab the MTTKRP reads and wait for it
        int r0 = 0;
        if (p.overlap == 2) {
            p.replay_cap = p.remap_ctas;
            DGPU_TRY(stable_sort_pingpong(p, p.cur, 1 - p.cur, p.proc[n], nm, p.shift[nm], p.K[nm],
                                          &r0, 0, 1));
            p.replay_cap = 0;
        }
        p.stream = p.ovl_stream;
        DGPU_TRY(launch_mttkrp_run(p, n, p.slab[p.cur]));
        if (after_mttkrp) DGPU_CUDA(cudaEventRecord(after_mttkrp, p.stream));
        DGPU_CUDA(cudaEventRecord(p.ovl_join, p.stream));
        if (after) {
            DGPU_TRY((*after)());
            DGPU_CUDA(cudaEventRecord(p.ovl_tail, p.stream));
            p.ovl_pending = true;
        }
        p.stream = main;
        if (p.overlap == 2) {
            DGPU_CUDA(cudaStreamWaitEvent(main, p.ovl_join, 0));
            DGPU_TRY(stable_sort_pingpong(p, r0, 1 - r0, p.proc[n], nm, p.shift[nm], p.K[nm], &r, 1));
        } else {
            DGPU_TRY(stable_sort_pingpong(p, p.cur, 1 - p.cur, p.proc[n], nm, p.shift[nm], p.K[nm],
                                          &r));
            DGPU_CUDA(cudaStreamWaitEvent(main, p.ovl_join, 0));
        }
    }
    p.cur = r;
    p.next_mode = nm;
    ++p.pp_transitions;
    return DGPU_OK;
}

int pingpong_drain(Plan& p) {
    if (p.ovl_pending) {
        DGPU_CUDA(cudaStreamWaitEvent(p.stream, p.ovl_tail, 0));
        p.ovl_pending = false;
    }
    return DGPU_OK;
}

int mode_pingpong_staged(Plan& p, int n, const cudaEvent_t* waits, int nwaits,
                         cudaEvent_t after_mttkrp) {
    return mode_pingpong_impl(p, n, waits, nwaits, after_mttkrp, nullptr);
}

int mode_pingpong_then(Plan& p, int n, const std::function<int()>& after) {
    return mode_pingpong_impl(p, n, nullptr, 0, nullptr, &after);
}

int mode_pingpong(Plan& p, int n) { return mode_pingpong_staged(p, n, nullptr, 0, nullptr); }

int mode_ncopy(Plan& p, int n) {
    {
        const size_t yb = (size_t)p.dims[n] * p.Rp * sizeof(float);
        LaunchTimer t(p, KK_ZERO, (double)yb);
        DGPU_CUDA(cudaMemsetAsync(p.Yhat[n], 0, yb, p.stream));
    }
    DGPU_TRY(launch_mttkrp_run(p, n, p.slab[n]));
    p.next_mode = (n + 1) % p.N;
    return DGPU_OK;
}

}  // namespace dgpu
