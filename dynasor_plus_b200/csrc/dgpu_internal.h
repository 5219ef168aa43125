// ============================================================================
//  dgpu_internal.h -- shared declarations of libdynasor_b200.so.
//
//  Device data layout of a plan (all in HBM):
//
//    slab[s]   s in {0,1} (PingPong) or {0..N-1} (NCopy):
//              one cudaMalloc holding [vals f32 | idx[0] u32 | ... | idx[N-1]]
//              each column 256 B aligned.  The SoA order matches the
//              reference's Tensor (include/dynasor_common.h:345-352).
//    Y[n], Yhat[n]      I_n x Rp FP32 row-major, padding columns zero.
//    Yb[n]              I_n x Rp BF16 mirror of Y[n] for BF16 gathers.
//    tiles[n]           work tiles of mode n in the reference's processing
//                       order (LPT worker, shard list, slab position).
//    part_cnt / part_off  per-(bucket, tile) counts and offsets of the
//                       stable counting sort that implements the remap.
// ============================================================================
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dynasor_b200.h"

namespace dgpu {

constexpr int kMaxModes = DGPU_MAX_MODES;

// Elements per work tile (one CTA of the MTTKRP / partition kernels).
constexpr uint32_t kTile = 4096;
// Largest bucket count one partition pass handles; larger keys are split
// into least-significant-digit passes of this many buckets.
constexpr uint32_t kMaxBuckets = 2048;
constexpr int kDigitBits = 11;   // log2(kMaxBuckets)
constexpr int kDefaultDigitBits = 8;

// ----------------------------------------------------------------------------
//  Error plumbing (thread-local last error, status codes, no exit()).
// ----------------------------------------------------------------------------
void set_error(const char* fmt, ...);
const char* last_error();

#define DGPU_CUDA(call)                                                        \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            ::dgpu::set_error("%s failed: %s (%s:%d)", #call,                  \
                              cudaGetErrorString(e_), __FILE__, __LINE__);     \
            return DGPU_ERR_CUDA;                                              \
        }                                                                      \
    } while (0)

#define DGPU_TRY(expr)                                                         \
    do {                                                                       \
        int rc_ = (expr);                                                      \
        if (rc_ != DGPU_OK) return rc_;                                        \
    } while (0)

// One work tile: `count` consecutive slab positions starting at `begin`,
// all inside super-shard `shard` of the tile table's mode.  For segmented
// partitions (one independent counting sort per shard) `seg_first` is the
// index of the first tile of the same shard in the tile array.
struct Tile {
    uint32_t begin;
    uint32_t count;
    uint32_t shard;
    uint32_t seg_first;
};

// A chunk: consecutive entries [tile_begin, tile_end) of a tile list, all in
// one segment.  One CTA of the partition kernels handles one chunk.
struct Chunk {
    uint32_t tile_begin;
    uint32_t tile_end;
    uint32_t seg;
    uint32_t contiguous;        // 1: the tiles are consecutive slab ranges
};

// A segment: chunks [chunk_begin, chunk_end) sorted as one independent
// counting sort whose output starts at slab position `base`.
struct Seg {
    uint32_t chunk_begin;
    uint32_t chunk_end;
    uint32_t base;
    uint32_t pad;
};

// A tile list prepared for the chunked partition (device arrays).
struct PartList {
    Tile*     tiles = nullptr;
    uint32_t  ntiles = 0;
    Chunk*    chunks = nullptr;
    uint32_t  nchunks = 0;
    Seg*      segs = nullptr;
    uint32_t  nsegs = 0;
    uint32_t* order = nullptr;    // chunk ids, largest first: the scatter's work queue
    bool      own_tiles = false;
    // the scatter's windows in list order (a window never crosses a tile):
    // {first slab position, offset in list order, element count, 0}, and
    // each tile's offset in list order
    uint4*    wins = nullptr;
    uint32_t  nwin = 0;
    uint32_t* tile_pre = nullptr;
    uint32_t* tile_wb = nullptr;  // each tile's first window
    uint64_t  total = 0;          // elements listed
};

// Offset tables of one partition pass of the PingPong sweep, kept for the
// next sweep.  After the slab has gone through one full cycle of modes its
// arrangement is a function of the coordinates alone (every mode's shard and
// row key plus the schedule order break all ties), so each pass of a later
// cycle sees the same arrangement and produces the same per-(chunk, bucket)
// offsets; the reference likewise builds its remap cursor table once, at
// preprocessing.  Valid while the pass runs with the same list, key and
// bucket count.
constexpr int kPartCachePasses = 4;            // LSD passes per sort kept
struct PartCacheSlot {
    uint32_t*       off = nullptr;             // [chunks x buckets] in-segment prefixes
    uint32_t*       base = nullptr;            // [segments x buckets] bucket starts
    size_t          off_cap = 0, base_cap = 0; // entries allocated
    const PartList* list = nullptr;
    uint64_t        lists_gen = 0;
    int             key_mode = -1, shift = -1;
    uint32_t        mask = 0, nb = 0;
    bool            valid = false;
    // the pass recorded: for each slot of a window's bucket-ordered staging
    // (list order), the window index of the element staged there, and per
    // window and bucket the destination of the window's slot 0 of that
    // bucket (slot i of bucket b goes to tab[window][b] + i); a pass with a
    // recording is replayed without ranking
    uint16_t*       inv = nullptr;
    uint32_t*       tab = nullptr;
    size_t          inv_cap = 0, tab_cap = 0;  // entries allocated
    bool            replay = false;
};

// SoA slab on the device.
struct Slab {
    void*     raw = nullptr;
    size_t    bytes = 0;
    float*    vals = nullptr;
    uint32_t* idx[kMaxModes] = {nullptr};
};

// Device pointer bundle passed by value to kernels.
struct SlabPtrs {
    const float*    vals;
    const uint32_t* idx[kMaxModes];
};
struct SlabOut {
    float*    vals;
    uint32_t* idx[kMaxModes];
};

// Kernel classes tracked by the optional per-launch CUDA-event timer.
enum KernelKind : int {
    KK_MTTKRP = 0,       // mode-n MTTKRP
    KK_PART_HIST = 1,    // remap / shard sort partition: per-chunk histograms
    KK_PART_SCAN = 2,    // remap / shard sort partition: exclusive scans
    KK_PART_SCATTER = 3, // remap / shard sort partition: stable scatter
    KK_ZERO = 4,         // Yhat zeroing
    KK_LINALG = 5,       // CP-ALS dense kernels
    KK_FIB_HIST = 6,     // fiber sort partition: histograms
    KK_FIB_SCAN = 7,     // fiber sort partition: scans
    KK_FIB_SCATTER = 8,  // fiber sort partition: scatter
    KK_COUNT = 9
};

struct TimedLaunch {
    int         kind;
    cudaEvent_t a, b;
    double      bytes;    // algorithmic bytes of the launch
};

// A number no other plan of this process has had (plan.cu): keys of cached
// graphs that span several plans name their plans by it, so a graph built
// for a plan that has since been destroyed can never match a new plan that
// reuses its address.
uint64_t next_plan_serial();

// Words of a cached CP-ALS loop graph's key (cpals.cu, CpSession::loop_key).
constexpr int kLoopKeyWords = 13;

struct Plan {
    uint64_t                 serial = next_plan_serial();
    // ---- per-launch timing (dgpu_plan_set_timing) -----------------------
    bool                     timing = false;
    std::vector<TimedLaunch> pending;
    std::vector<cudaEvent_t> event_pool;
    double                   t_ms[KK_COUNT] = {};
    double                   t_bytes[KK_COUNT] = {};
    uint64_t                 t_launches[KK_COUNT] = {};

    // ---- geometry ----------------------------------------------------
    int       N = 0;
    uint64_t  nnz = 0;
    int       T = 1;
    int       R = 0, Rp = 0;
    int       layout = DGPU_LAYOUT_PINGPONG;
    int       fiber = 1;
    int       precision = DGPU_PREC_FP32;
    int       accum = DGPU_ACCUM_AUTO;
    int       device = 0;
    uint32_t  dims[kMaxModes] = {};
    uint32_t  mn[kMaxModes] = {};
    int       shift[kMaxModes] = {};
    uint32_t  K[kMaxModes] = {};
    int       kclass[kMaxModes] = {};
    double    afl[kMaxModes] = {};

    // ---- host plan tables ---------------------------------------------
    std::vector<std::vector<uint64_t>> count;   // [n][s]
    std::vector<std::vector<uint64_t>> sbeg;    // [n][s]
    std::vector<std::vector<uint64_t>> send;    // [n][s]
    std::vector<std::vector<std::vector<uint32_t>>> sched;  // [n][tid]
    std::vector<std::vector<Tile>> tiles_h;     // [n] processing order

    // ---- device state -------------------------------------------------
    cudaStream_t stream = nullptr;
    bool         own_stream = false;
    cudaStream_t copy_stream = nullptr;         // host transfers overlapping the sweep
    cudaStream_t side_stream = nullptr;         // CP-ALS solves overlapping the MTTKRP
    cudaStream_t ovl_stream = nullptr;          // PingPong: MTTKRP beside the remap
    cudaEvent_t  ovl_fork = nullptr, ovl_join = nullptr, ovl_tail = nullptr;
    bool         ovl_pending = false;           // work after ovl_tail's record not yet joined
    // 0: MTTKRP then remap on the plan stream; 1: MTTKRP launched first on a
    // second stream beside the remap; 2 (default): the remap's first pass
    // launched first at remap_ctas CTAs per SM, the MTTKRP beside it
    int          overlap = 2;
    int          remap_ctas = 1;                // overlap 2: remap CTAs per SM beside the MTTKRP
    int          replay_cap = 0;                // > 0: replayed passes run at most this many CTAs per SM
    Slab         slab[kMaxModes];               // 2 for PingPong, N for NCopy
    int          cur = 0;                       // PingPong: live slab index
    int          next_mode = 0;                 // PingPong: mode the slab is sorted for
    Tile*        tiles_d[kMaxModes] = {nullptr};   // mode n tiles, processing order
    // the MTTKRP's CTA tiles: processing-order tiles of one shard merged
    // in pairs for 3-mode plans (rowrun_tiles in plan.cu), else tiles_d
    Tile*        run_tiles_d[kMaxModes] = {nullptr};
    uint32_t     run_tiles_n[kMaxModes] = {0};
    PartList     proc[kMaxModes];               // remap of mode n (global, processing order)
    PartList     fib[kMaxModes];                // fiber sort of mode n (segmented by shard)
    PartList     ident;                         // identity order over [0, nnz) (global)
    int          sms = 148;                     // SM count of the device
    int          part_fiber = 0;                // 1 while a fiber-sort partition runs (timing class)
    int          rank_tile = 0;                 // MTTKRP columns per slab pass (0: tuned)
    int          tile_for[kMaxModes] = {};      // tuned columns per slab pass, per mode
    // Widest LSD digit of shard sorts / remaps and of fiber sorts.  Above ~8
    // bits a pass writes runs of a few elements per bucket and window, which
    // costs more (uncoalesced stores, partial-sector DRAM writes) than a
    // second pass with narrow digits.
    int          sort_digit_bits = kDefaultDigitBits;
    int          fiber_digit_bits = kDefaultDigitBits;
    // Chunk sizes of the partition passes and the MTTKRP grid target; the
    // defaults were measured on the 64.7M-nonzero 3-mode tensor and
    // dgpu_plan_autotune picks per plan.  Neither changes any permutation.
    int          chunks_per_sm = 4;             // global (remap) partition: chunks per SM
    int          seg_chunk_tiles = 16;          // segmented (fiber) partition: tiles per chunk
    int          mttkrp_ctas_per_sm = 4;        // tiles are split until this many CTAs per SM
    // MTTKRP gathers: 0 per-lane loads (mttkrp.cu, any shape), 1 the TMA
    // engine's tile::gather4 into a shared-memory ring (mttkrp_tma.cu;
    // 3 and 4 modes, Rp 16/32/64, whole rows)
    int          mttkrp_kernel = 0;
    float*       Y[kMaxModes] = {nullptr};
    float*       Yhat[kMaxModes] = {nullptr};
    __nv_bfloat16* Yb[kMaxModes] = {nullptr};
    bool         yb_stale[kMaxModes] = {};
    // Under BF16 precision, the mode whose MTTKRP still gathers FP32 rows
    // (-1: none).  CP-ALS sets it to the last mode for the length of a run:
    // that mode's Yhat gives the fit's <X, M> term, and BF16-rounded gathers
    // there move the fit by up to ~2e-4 on small, well-fitted tensors.
    int          fp32_gather_mode = -1;
    bool         gather_fp32_all = false;       // every mode gathers FP32 (gradient path)
    float*       grad_buf = nullptr;            // CP-OPT gradients of all modes
    size_t       grad_cap = 0;                  // floats in grad_buf
    float*       model_buf = nullptr;           // CP-OPT model values at the nonzeros
    size_t       model_cap = 0;                 // floats in model_buf
    // two pinned chunks that copies to pageable host memory go through
    void*        stage_host[2] = {nullptr, nullptr};
    size_t       stage_cap = 0;                 // bytes of each chunk
    cudaEvent_t  stage_ev[2] = {nullptr, nullptr};
    uint32_t*    part_cnt = nullptr;            // [chunks x buckets] counts
    uint32_t*    part_off = nullptr;            // [chunks x buckets] in-segment prefixes
    size_t       part_cap = 0;                  // entries of each
    uint32_t*    part_base = nullptr;           // [segments x buckets] bucket starts
    size_t       part_base_cap = 0;
    // PingPong partition passes: offset tables kept per (mode, fiber sort 0 /
    // remap 1, LSD pass) once the slab is past its first cycle (see
    // PartCacheSlot); DGPU_PART_CACHE=0 turns this off and
    // DGPU_PART_CACHE_CHECK=1 recomputes every kept table and flags a
    // difference (device fault flag 0x1000)
    PartCacheSlot pcache[kMaxModes][2][kPartCachePasses];
    int          part_cache = 1;
    int          part_cache_check = 0;
    int          part_replay = 1;               // DGPU_PART_REPLAY=0: kept tables only, no recording
    uint64_t     pp_transitions = 0;            // PingPong modes run since the slab was set
    uint64_t     lists_gen = 0;                 // bumped when partition lists are rebuilt
    uint64_t     pc_uncached = 0;               // PingPong passes that computed their tables
    int          pc_mode = -1;                  // mode of the running PingPong step (-1: none)
    PartCacheSlot* pc_slot = nullptr;           // slot of the next stable_partition call
    int*         err_flag = nullptr;            // device-side fault flag
    uint32_t*    part_ctr = nullptr;            // work-queue counter of the partition scatter
    float*       lambda = nullptr;              // [Rp]
    double*      la_work = nullptr;             // CP-ALS R x R scratch (FP64)
    size_t       la_work_cap = 0;
    float*       la_f32 = nullptr;              // FP32 scratch (Grams etc.)
    size_t       la_f32_cap = 0;
    uint64_t     device_bytes = 0;
    // CP-ALS state kept across cpals calls on this plan: the pinned fit
    // buffer, the device loop's state array, timing / fork-join events, and
    // the device-loop graph of the last run with the key it was captured for
    // (options, norm, live slab and the buffers it reads)
    double*      cp_fit_host = nullptr;         // pinned [4]
    double*      cp_st = nullptr;               // device loop state
    size_t       cp_st_bytes = 0;
    std::vector<cudaEvent_t> cp_ev, cp_fork, cp_join;
    cudaGraphExec_t cp_loop_exec = nullptr;
    uint64_t     cp_loop_key[kLoopKeyWords] = {};
    // bumped whenever the partition lists are rebuilt or a launch knob
    // changes (dgpu_plan_autotune): part of every cached loop graph's key
    uint64_t     tables_gen = 0;
    // the device loops of a multi-tensor batch led by this plan (the first
    // of the batch): one graph of parallel WHILE nodes, kept with its key
    // (every plan's serial and loop key) for a later call on the same plans
    cudaGraphExec_t cp_batch_exec = nullptr;
    std::vector<uint64_t> cp_batch_key;
    double       cp_tnorm2 = -1.0;              // ||T||^2 once computed (< 0: not yet)
    double       cp_mttkrp_frac = 0.5;          // MTTKRP share of an iteration, last measured
    // Morton layout: sorted keys and their values (the slabs are freed once
    // they are built), per-mode masks and bit counts
    uint64_t*    mkeys = nullptr;
    float*       mvals = nullptr;
    uint64_t     mmask[kMaxModes] = {};
    uint8_t      mbits[kMaxModes] = {};

    ~Plan();
};

// ---- optional launch timing ------------------------------------------------
// Brackets one launch with CUDA events on the plan stream when timing is on.
struct LaunchTimer {
    Plan&       p;
    int         kind;
    double      bytes;
    cudaEvent_t a = nullptr;
    LaunchTimer(Plan& pl, int k, double b);
    ~LaunchTimer();
};
int timing_collect(Plan& p);

// Synchronises the plan stream and reads the device fault flag (bounded
// waits that gave up, out-of-range keys); a raised flag is cleared and
// reported as DGPU_ERR_DEVICE.
int sync_checked(Plan& p);

// PingPong: makes the plan stream wait for work that a chained mode left on
// ovl_stream (plan.cu, mode_pingpong_then).
int pingpong_drain(Plan& p);

// ---- Morton layout (morton.cu) -------------------------------------------
// Key bit positions of each mode's index bits, LSB first: decoding is pext
// of the key by the mode's mask, encoding pdep (src/dynasor_morton.cpp:43-81).
struct MortonDec {
    uint8_t pos[kMaxModes][32];
    uint8_t bits[kMaxModes];
};
// The reference's bit plan (src/dynasor_morton.cpp:99-134): b_n =
// ceil(log2 I_n) (>= 1), bits handed out LSB-first round-robin over the
// modes that still need bits.  False when sum b_n > 64.
bool morton_plan(int N, const uint32_t* dims, uint64_t* mask, uint8_t* bits);
MortonDec morton_decoder(const Plan& p);
// Morton keys from slab[src] (COO in any order), sorted, into p.mkeys /
// p.mvals; frees the slabs.
int morton_build(Plan& p, int src);
// p.mkeys / p.mvals already hold keys and values (e.g. read from a file):
// check every key (decodes within range, re-encodes to itself, ascending)
// and decode them into slab `dst` (vals + indices).
int morton_check_decode(Plan& p, int dst);
// Releases every slab of the plan (Morton plans keep keys and values only).
void free_slabs(Plan& p);

// ---- .dnp processed-tensor image (src/dynasor_dnp.cpp) ---------------------
// Host copy of everything one .dnp file holds for the PingPong and NCopy
// layouts.  `copies` slabs: 1 for PingPong, N for NCopy.
struct DnpImage {
    int      layout = DGPU_LAYOUT_PINGPONG;      // DGPU_LAYOUT_PINGPONG / NCOPY
    int      N = 0;
    uint64_t nnz = 0;
    uint32_t dims[kMaxModes] = {};
    int      threads = 0;
    double   tnorm_sq = 0.0;
    uint32_t K[kMaxModes] = {};
    uint32_t mn[kMaxModes] = {};
    int32_t  shift[kMaxModes] = {};
    uint32_t shard_size = 0;
    double   afl[kMaxModes] = {};
    uint32_t kclass[kMaxModes] = {};
    int8_t   inplace_mode = 0;
    uint64_t remap_stride = 0;
    std::vector<uint64_t> touched_count;                      // [n]
    std::vector<std::vector<uint8_t>> touched;                // [n][ceil(I_n/8)]
    std::vector<std::vector<uint64_t>> sbeg, send;            // [n][s]
    std::vector<std::vector<std::vector<uint32_t>>> sched;    // [n][tid]
    std::vector<std::vector<uint64_t>> cursor;                // [n][tid * stride + s']
    uint8_t  fiber_sorted[kMaxModes] = {};
    uint8_t  csr[kMaxModes] = {};
    std::vector<float> vals[kMaxModes];                       // [copy][nnz]
    std::vector<uint32_t> idx[kMaxModes][kMaxModes];          // [copy][mode][nnz]
    std::vector<uint64_t> rowptr[kMaxModes];                  // [copy][I_k + 1] when csr[k]
    uint64_t mmask[kMaxModes] = {};                           // Morton files
    uint8_t  mbits[kMaxModes] = {};
    std::vector<uint64_t> mkeys;
    std::vector<float> mvals;
};
// A plan that uses the image's slabs, shard tables and schedule as they are.
int plan_build_dnp(Plan& p, const DnpImage& img, const dgpu_plan_opts& o);

// ---- device memory helpers ----------------------------------------------
int  dev_alloc(Plan& p, void** ptr, size_t bytes);
void dev_free(void* ptr);
int  slab_alloc(Plan& p, Slab& s);
SlabPtrs slab_in(const Slab& s, int N);
SlabOut  slab_out(const Slab& s, int N);

// ---- kernels launched from host code (defined in .cu files) -------------
// Per-mode shard histograms of the input COO (flat, sum of K_n bins) and
// an out-of-range index check.
int launch_shard_counts(Plan& p, const Slab& s, uint64_t* counts_d, size_t total_bins);

// Stable partition: the elements listed by `tiles` (processing order) are
// written to `out` ordered by key = (idx[key_mode] >> key_shift) & key_mask
// (buckets < nb <= kMaxBuckets), each bucket starting at `base_off` +
// (elements of all smaller buckets), stably.  Uses p.part_cnt/part_off.
// The list's segments are sorted independently (a global list has one).
int stable_partition(Plan& p, const Slab& in, const PartList& list,
                     int key_mode, int key_shift, uint32_t key_mask, uint32_t nb,
                     const Slab& out);
// Fiber sort of mode n (stable sort of every mode-n shard by row) from
// slab[src] ping-ponging with slab[other]; *result = slab holding it.
int fiber_sort(Plan& p, int n, int src, int other, int* result);
// Build the chunk/segment tables of a tile list.  `seg_of_tile` (host, may
// be empty) gives each tile's segment and `seg_base` each segment's output
// start; empty means one global segment starting at 0.
// Rebuilds every partition list of the plan with the current chunk sizes
// (plan.cu).
int plan_rebuild_partlists(Plan& p);
int build_partlist(Plan& p, const std::vector<Tile>& tiles,
                   const std::vector<uint32_t>& seg_of_tile,
                   const std::vector<uint32_t>& seg_base, PartList& out, Tile* shared_tiles);
void free_partlist(PartList& l);
// Stable sort of the sequence listed by `first` (a global list) over slab[a]
// by the key (idx[key_mode] >> key_shift) < key_limit, any key range: one
// partition pass per least-significant digit (later passes in slab order),
// ping-ponging between slab[a] and slab[b]; *result receives the slab index
// that holds the sorted data.
// Passes [k0, k1) only (k1 < 0: to the last) -- the remap split around the
// MTTKRP launched beside it.
int stable_sort_pingpong(Plan& p, int a, int b, const PartList& first,
                         int key_mode, int key_shift, uint64_t key_limit, int* result,
                         int k0 = 0, int k1 = -1);

// MTTKRP of mode n over the tiles of the slab `in` into p.Yhat[n].
int launch_mttkrp(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles);
int mttkrp_scheme(const Plan& p, int n);   // DGPU_ACCUM_ROWRUN or DGPU_ACCUM_PRIVATE
// All-modes pass over the plan's live nonzeros (SoA slab or Morton keys).
int launch_mttkrp_all_modes(Plan& p);
// Values array of the live nonzeros (any order).
const float* live_vals(const Plan& p);

// MTTKRP with TMA row gathers (mttkrp_tma.cu): whether the plan's shape has
// a variant for `cols` columns per pass, and the launch.
bool gather_supported(const Plan& p, int cols);
int launch_mttkrp_gather(Plan& p, int n, const Slab& in, const Tile* tiles, uint32_t ntiles,
                         bool bf, int wl, int rows_contiguous);

// FP32 -> BF16 factor mirror.
int launch_to_bf16(Plan& p, int n);
// bytes from device memory to host memory the caller may not have pinned:
// chunk k+1 is copied to one of the plan's two pinned chunks while the host
// moves chunk k out of the other; waits for the plan stream (extras.cu)
int copy_to_host_staged(Plan& p, void* host, const void* dev, size_t bytes);

// Dense CP-ALS pieces.
int cp_tensor_norm(Plan& p, const float* vals, double* out);
int launch_model_values(Plan& p, float* out);
int cpopt_gradient(Plan& p, float* const* grad_host);

}  // namespace dgpu
