// ============================================================================
//  api.cu -- the extern "C" boundary of libdynasor_b200.so.
//
//  Every entry point validates its arguments, returns a DGPU_* status and
//  records a one-line message for dgpu_last_error().  No exit(), no
//  exceptions across the boundary.
// ============================================================================
#include "dgpu_internal.h"

#include <chrono>
#include <cstring>
#include <new>
#include <vector>

namespace dgpu {
int plan_build(Plan& p, const dgpu_tensor_desc& t, const dgpu_plan_opts& o);
int mode_pingpong(Plan& p, int n);
int mode_pingpong_staged(Plan& p, int n, const cudaEvent_t* waits, int nwaits,
                         cudaEvent_t after_mttkrp);
int mode_ncopy(Plan& p, int n);
int cpals_run(Plan& p, const dgpu_cp_options& o, dgpu_cp_result& r, double* fit_history);
int cpals_multistart_run(Plan& p, int K, const dgpu_cp_options& o, dgpu_cp_result* res,
                         double* fit_history);
int cpals_batch_run(Plan* const* plans, int count, const dgpu_cp_options& o,
                    dgpu_cp_result* res, double* fit_history);
}  // namespace dgpu

using namespace dgpu;

#define API_GUARD(p)                                                           \
    do {                                                                       \
        if (!(p)) {                                                            \
            set_error("%s: null plan", __func__);                              \
            return DGPU_ERR_ARG;                                               \
        }                                                                      \
        cudaError_t e_ = cudaSetDevice((p)->device);                           \
        if (e_ != cudaSuccess) {                                               \
            set_error("%s: cudaSetDevice: %s", __func__, cudaGetErrorString(e_)); \
            return DGPU_ERR_CUDA;                                              \
        }                                                                      \
    } while (0)

#define MODE_GUARD(p, n)                                                       \
    do {                                                                       \
        if ((n) < 0 || (n) >= (p)->N) {                                        \
            set_error("%s: mode %d out of range [0,%d)", __func__, (n), (p)->N); \
            return DGPU_ERR_ARG;                                               \
        }                                                                      \
    } while (0)

extern "C" {

const char* dgpu_last_error(void) { return last_error(); }

int dgpu_version(void) { return 0x000100; }

int dgpu_device_count(int* count) {
    if (!count) { set_error("dgpu_device_count: null"); return DGPU_ERR_ARG; }
    *count = 0;
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        set_error("cudaGetDeviceCount: %s", cudaGetErrorString(e));
        return DGPU_ERR_CUDA;
    }
    return DGPU_OK;
}

void dgpu_plan_opts_default(dgpu_plan_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->threads = 1;
    o->rank = 16;
    o->layout = DGPU_LAYOUT_PINGPONG;
    o->fiber = 1;
    o->precision = DGPU_PREC_FP32;
    o->device = 0;
    o->mn_target = nullptr;
}

int dgpu_plan_create(const dgpu_tensor_desc* t, const dgpu_plan_opts* o, dgpu_plan** out) {
    if (!t || !o || !out) { set_error("dgpu_plan_create: null argument"); return DGPU_ERR_ARG; }
    *out = nullptr;
    if (t->num_modes < 2 || t->num_modes > DGPU_MAX_MODES) {
        set_error("dgpu_plan_create: num_modes %d outside [2,%d]", t->num_modes, DGPU_MAX_MODES);
        return t->num_modes <= 0 ? DGPU_ERR_EMPTY : DGPU_ERR_ARG;
    }
    if (t->nnz == 0) { set_error("dgpu_plan_create: empty tensor (nnz = 0)"); return DGPU_ERR_EMPTY; }
    if (t->nnz >= 0xffffffffull) {
        set_error("dgpu_plan_create: nnz %llu exceeds the 32-bit slab positions",
                  (unsigned long long)t->nnz);
        return DGPU_ERR_ARG;
    }
    if (!t->mode_size || !t->vals || !t->idx) {
        set_error("dgpu_plan_create: null tensor array"); return DGPU_ERR_ARG;
    }
    for (int n = 0; n < t->num_modes; ++n) {
        if (!t->idx[n]) { set_error("dgpu_plan_create: idx[%d] is null", n); return DGPU_ERR_ARG; }
        if (t->mode_size[n] == 0) {
            set_error("dgpu_plan_create: mode %d has size 0", n); return DGPU_ERR_ARG;
        }
    }
    if (o->threads < 1) { set_error("dgpu_plan_create: threads %d < 1", o->threads); return DGPU_ERR_ARG; }
    if (o->rank < 1 || o->rank > 1024) {
        set_error("dgpu_plan_create: rank %d outside [1,1024]", o->rank); return DGPU_ERR_ARG;
    }
    if (o->layout != DGPU_LAYOUT_PINGPONG && o->layout != DGPU_LAYOUT_NCOPY &&
        o->layout != DGPU_LAYOUT_MORTON && o->layout != DGPU_LAYOUT_AUTO) {
        set_error("dgpu_plan_create: unknown layout %d", o->layout); return DGPU_ERR_ARG;
    }
    if (o->precision != DGPU_PREC_FP32 && o->precision != DGPU_PREC_BF16) {
        set_error("dgpu_plan_create: unknown precision %d", o->precision); return DGPU_ERR_ARG;
    }
    if (o->accum < DGPU_ACCUM_AUTO || o->accum > DGPU_ACCUM_PRIVATE) {
        set_error("dgpu_plan_create: unknown accumulation mode %d", o->accum); return DGPU_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("dgpu_plan_create: no CUDA device available");
        return DGPU_ERR_CUDA;
    }
    if (o->device < 0 || o->device >= ndev) {
        set_error("dgpu_plan_create: device %d outside [0,%d)", o->device, ndev);
        return DGPU_ERR_ARG;
    }
    Plan* p = new (std::nothrow) Plan();
    if (!p) { set_error("dgpu_plan_create: host OOM"); return DGPU_ERR_NOMEM; }
    const int rc = plan_build(*p, *t, *o);
    if (rc != DGPU_OK) {
        delete p;
        return rc;
    }
    *out = reinterpret_cast<dgpu_plan*>(p);
    return DGPU_OK;
}

int dgpu_plan_destroy(dgpu_plan* plan) {
    if (!plan) return DGPU_OK;
    delete reinterpret_cast<Plan*>(plan);
    return DGPU_OK;
}

int dgpu_plan_get_info(const dgpu_plan* plan, dgpu_plan_info* info) {
    const Plan* p = reinterpret_cast<const Plan*>(plan);
    if (!p || !info) { set_error("dgpu_plan_get_info: null argument"); return DGPU_ERR_ARG; }
    std::memset(info, 0, sizeof(*info));
    info->num_modes = p->N;
    info->nnz = p->nnz;
    info->rank = p->R;
    info->rank_padded = p->Rp;
    info->threads = p->T;
    for (int n = 0; n < p->N; ++n) {
        info->mode_size[n] = p->dims[n];
        info->mn[n] = p->mn[n];
        info->mn_shift[n] = p->shift[n];
        info->shards_per_mode[n] = p->K[n];
        info->kernel_class[n] = p->kclass[n];
        info->avg_fiber_len[n] = p->afl[n];
        info->tiles[n] = (uint32_t)p->tiles_h[n].size();
    }
    info->next_mode = p->next_mode;
    info->device_bytes = p->device_bytes;
    info->layout = p->layout;
    return DGPU_OK;
}

int dgpu_plan_set_stream(dgpu_plan* plan, void* stream) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    DGPU_CUDA(cudaStreamSynchronize(p->stream));
    if (p->own_stream) cudaStreamDestroy(p->stream);
    p->own_stream = false;
    p->stream = static_cast<cudaStream_t>(stream);
    return DGPU_OK;
}

int dgpu_plan_sync(dgpu_plan* plan) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    DGPU_TRY(sync_checked(*p));
    return DGPU_OK;
}

int dgpu_plan_set_timing(dgpu_plan* plan, int enable) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    DGPU_TRY(timing_collect(*p));
    p->timing = enable != 0;
    return DGPU_OK;
}

int dgpu_plan_get_timing(dgpu_plan* plan, dgpu_kernel_timing* out, int max, int* count,
                         int reset) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    if (!count || (max > 0 && !out)) { set_error("dgpu_plan_get_timing: null"); return DGPU_ERR_ARG; }
    DGPU_TRY(timing_collect(*p));
    static const char* names[KK_COUNT] = {"mttkrp", "part_hist", "part_scan", "part_scatter",
                                          "zero", "linalg", "fiber_hist", "fiber_scan",
                                          "fiber_scatter"};
    int k = 0;
    for (int i = 0; i < KK_COUNT && k < max; ++i) {
        std::memset(&out[k], 0, sizeof(out[k]));
        std::strncpy(out[k].name, names[i], sizeof(out[k].name) - 1);
        out[k].launches = p->t_launches[i];
        out[k].total_ms = p->t_ms[i];
        out[k].bytes = p->t_bytes[i];
        ++k;
    }
    *count = k;
    if (reset)
        for (int i = 0; i < KK_COUNT; ++i) p->t_ms[i] = p->t_bytes[i] = 0, p->t_launches[i] = 0;
    return DGPU_OK;
}

int dgpu_plan_shards(const dgpu_plan* plan, int n, uint64_t* begin, uint64_t* end) {
    const Plan* p = reinterpret_cast<const Plan*>(plan);
    if (!p || !begin || !end) { set_error("dgpu_plan_shards: null argument"); return DGPU_ERR_ARG; }
    MODE_GUARD(p, n);
    std::memcpy(begin, p->sbeg[n].data(), p->K[n] * sizeof(uint64_t));
    std::memcpy(end, p->send[n].data(), p->K[n] * sizeof(uint64_t));
    return DGPU_OK;
}

int dgpu_plan_schedule(const dgpu_plan* plan, int n, uint32_t* counts, uint32_t* flat,
                       uint32_t* n_listed) {
    const Plan* p = reinterpret_cast<const Plan*>(plan);
    if (!p || !counts || !flat || !n_listed) {
        set_error("dgpu_plan_schedule: null argument"); return DGPU_ERR_ARG;
    }
    MODE_GUARD(p, n);
    uint32_t k = 0;
    for (int t = 0; t < p->T; ++t) {
        counts[t] = (uint32_t)p->sched[n][t].size();
        for (uint32_t s : p->sched[n][t]) flat[k++] = s;
    }
    *n_listed = k;
    return DGPU_OK;
}

int dgpu_upload_factor(dgpu_plan* plan, int n, const float* Y) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    MODE_GUARD(p, n);
    if (!Y) { set_error("dgpu_upload_factor: null"); return DGPU_ERR_ARG; }
    DGPU_CUDA(cudaMemcpyAsync(p->Y[n], Y, (size_t)p->dims[n] * p->Rp * sizeof(float),
                              cudaMemcpyHostToDevice, p->stream));
    p->yb_stale[n] = true;
    return DGPU_OK;
}

int dgpu_download_factor(dgpu_plan* plan, int n, float* Y) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    MODE_GUARD(p, n);
    if (!Y) { set_error("dgpu_download_factor: null"); return DGPU_ERR_ARG; }
    DGPU_CUDA(cudaMemcpyAsync(Y, p->Y[n], (size_t)p->dims[n] * p->Rp * sizeof(float),
                              cudaMemcpyDeviceToHost, p->stream));
    DGPU_TRY(sync_checked(*p));
    return DGPU_OK;
}

int dgpu_download_yhat(dgpu_plan* plan, int n, float* Yhat) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    MODE_GUARD(p, n);
    if (!Yhat) { set_error("dgpu_download_yhat: null"); return DGPU_ERR_ARG; }
    DGPU_CUDA(cudaMemcpyAsync(Yhat, p->Yhat[n], (size_t)p->dims[n] * p->Rp * sizeof(float),
                              cudaMemcpyDeviceToHost, p->stream));
    DGPU_TRY(sync_checked(*p));
    return DGPU_OK;
}

int dgpu_download_lambda(dgpu_plan* plan, float* lambda) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    if (!lambda) { set_error("dgpu_download_lambda: null"); return DGPU_ERR_ARG; }
    DGPU_CUDA(cudaMemcpyAsync(lambda, p->lambda, (size_t)p->R * sizeof(float),
                              cudaMemcpyDeviceToHost, p->stream));
    DGPU_CUDA(cudaStreamSynchronize(p->stream));
    return DGPU_OK;
}

int dgpu_factor_device_ptr(dgpu_plan* plan, int n, void** Y, void** Yhat) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    if (!p) { set_error("dgpu_factor_device_ptr: null plan"); return DGPU_ERR_ARG; }
    MODE_GUARD(p, n);
    if (Y) *Y = p->Y[n];
    if (Yhat) *Yhat = p->Yhat[n];
    p->yb_stale[n] = true;   // the caller may write Y[n] directly
    return DGPU_OK;
}

int dgpu_mttkrp_mode(dgpu_plan* plan, int n) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    MODE_GUARD(p, n);
    if (p->layout == DGPU_LAYOUT_MORTON) {
        set_error("dgpu_mttkrp_mode: a Morton plan runs the all-modes pass only "
                  "(dgpu_mttkrp_all_modes / dgpu_mttkrp_sweep)");
        return DGPU_ERR_ARG;
    }
    if (p->layout == DGPU_LAYOUT_NCOPY) return mode_ncopy(*p, n);
    return mode_pingpong(*p, n);
}

int dgpu_mttkrp_sweep(dgpu_plan* plan) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    // a sweep without factor updates computes every mode from the same
    // factors: on the Morton layout that is one all-modes pass
    if (p->layout == DGPU_LAYOUT_MORTON) return launch_mttkrp_all_modes(*p);
    for (int n = 0; n < p->N; ++n) {
        const int rc = (p->layout == DGPU_LAYOUT_NCOPY) ? mode_ncopy(*p, n) : mode_pingpong(*p, n);
        if (rc != DGPU_OK) return rc;
    }
    return DGPU_OK;
}

int dgpu_mttkrp_sweep_host(dgpu_plan* plan, const float* const* Y, float* const* Yhat,
                           double* secs) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    if (!Y || !Yhat) { set_error("dgpu_mttkrp_sweep_host: null"); return DGPU_ERR_ARG; }
    for (int n = 0; n < p->N; ++n)
        if (!Y[n] || !Yhat[n]) { set_error("dgpu_mttkrp_sweep_host: null factor %d", n); return DGPU_ERR_ARG; }
    if (p->next_mode != 0 && p->layout == DGPU_LAYOUT_PINGPONG) {
        set_error("dgpu_mttkrp_sweep_host: the slab is ordered for mode %d, a sweep starts at 0",
                  p->next_mode);
        return DGPU_ERR_ORDER;
    }
    if (p->layout == DGPU_LAYOUT_MORTON) {
        // one all-modes pass between the uploads and the downloads
        cudaEvent_t a = nullptr, b = nullptr;
        DGPU_CUDA(cudaEventCreate(&a));
        DGPU_CUDA(cudaEventCreate(&b));
        struct E { cudaEvent_t& a; cudaEvent_t& b; ~E() { cudaEventDestroy(a); cudaEventDestroy(b); } } eg{a, b};
        for (int w = 0; w < p->N; ++w) {
            DGPU_CUDA(cudaMemcpyAsync(p->Y[w], Y[w], (size_t)p->dims[w] * p->Rp * sizeof(float),
                                      cudaMemcpyHostToDevice, p->stream));
            p->yb_stale[w] = true;
        }
        DGPU_CUDA(cudaEventRecord(a, p->stream));
        DGPU_TRY(launch_mttkrp_all_modes(*p));
        DGPU_CUDA(cudaEventRecord(b, p->stream));
        for (int n = 0; n < p->N; ++n)
            DGPU_CUDA(cudaMemcpyAsync(Yhat[n], p->Yhat[n], (size_t)p->dims[n] * p->Rp * sizeof(float),
                                      cudaMemcpyDeviceToHost, p->stream));
        DGPU_TRY(sync_checked(*p));
        if (secs) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            *secs = ms * 1e-3;
        }
        return DGPU_OK;
    }
    // Transfers overlap the mode passes on a second stream: the factors mode 0
    // gathers go first (on PingPong plans while mode 0's fiber sort runs),
    // Y[0] (first needed by mode 1) streams in while mode 0 runs, and each
    // Yhat[n] streams out as soon as its MTTKRP is done (on PingPong plans
    // while the remap after it runs).  With pinned host buffers little of
    // the transfer time is exposed.
    if (!p->copy_stream) DGPU_CUDA(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
    const int N = p->N;
    std::vector<cudaEvent_t> up(N, nullptr), done(N, nullptr);
    cudaEvent_t e0 = nullptr, e1 = nullptr, start = nullptr;
    struct Ev {
        std::vector<cudaEvent_t>& a; std::vector<cudaEvent_t>& b; cudaEvent_t* c[3];
        ~Ev() {
            for (auto e : a) if (e) cudaEventDestroy(e);
            for (auto e : b) if (e) cudaEventDestroy(e);
            for (auto e : c) if (*e) cudaEventDestroy(*e);
        }
    } evg{up, done, {&e0, &e1, &start}};
    for (int n = 0; n < N; ++n) {
        DGPU_CUDA(cudaEventCreateWithFlags(&up[n], cudaEventDisableTiming));
        DGPU_CUDA(cudaEventCreateWithFlags(&done[n], cudaEventDisableTiming));
    }
    DGPU_CUDA(cudaEventCreate(&e0));
    DGPU_CUDA(cudaEventCreate(&e1));
    DGPU_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    // the copy stream starts after everything already queued on the plan stream
    DGPU_CUDA(cudaEventRecord(start, p->stream));
    DGPU_CUDA(cudaStreamWaitEvent(p->copy_stream, start, 0));
    for (int k = 1; k <= N; ++k) {
        const int w = k % N;                       // 1, 2, ..., N-1, then 0
        DGPU_CUDA(cudaMemcpyAsync(p->Y[w], Y[w], (size_t)p->dims[w] * p->Rp * sizeof(float),
                                  cudaMemcpyHostToDevice, p->copy_stream));
        DGPU_CUDA(cudaEventRecord(up[w], p->copy_stream));
        p->yb_stale[w] = true;
    }
    int rc = DGPU_OK;
    for (int n = 0; n < N && rc == DGPU_OK; ++n) {
        if (n == 0) DGPU_CUDA(cudaEventRecord(e0, p->stream));
        if (p->layout == DGPU_LAYOUT_NCOPY) {
            for (int w = 0; w < N; ++w)
                if (w != n) DGPU_CUDA(cudaStreamWaitEvent(p->stream, up[w], 0));
            rc = mode_ncopy(*p, n);
            if (rc != DGPU_OK) break;
            DGPU_CUDA(cudaEventRecord(done[n], p->stream));
        } else {
            // the fiber sort runs while the factors stream in; Yhat[n] streams
            // out while the remap runs
            std::vector<cudaEvent_t> waits;
            for (int w = 0; w < N; ++w)
                if (w != n) waits.push_back(up[w]);
            rc = mode_pingpong_staged(*p, n, waits.data(), (int)waits.size(), done[n]);
            if (rc != DGPU_OK) break;
        }
        DGPU_CUDA(cudaStreamWaitEvent(p->copy_stream, done[n], 0));
        DGPU_CUDA(cudaMemcpyAsync(Yhat[n], p->Yhat[n], (size_t)p->dims[n] * p->Rp * sizeof(float),
                                  cudaMemcpyDeviceToHost, p->copy_stream));
    }
    if (rc == DGPU_OK) DGPU_CUDA(cudaEventRecord(e1, p->stream));
    const cudaError_t ec = cudaStreamSynchronize(p->copy_stream);
    const int rs = sync_checked(*p);
    if (rc == DGPU_OK && ec != cudaSuccess) {
        set_error("dgpu_mttkrp_sweep_host: %s", cudaGetErrorString(ec));
        rc = DGPU_ERR_CUDA;
    }
    if (rc == DGPU_OK) rc = rs;
    if (rc == DGPU_OK && secs) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        *secs = ms * 1e-3;
    }
    return rc;
}

int dgpu_download_slab(dgpu_plan* plan, float* vals, uint32_t* const* idx) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    if (!vals || !idx) { set_error("dgpu_download_slab: null"); return DGPU_ERR_ARG; }
    for (int n = 0; n < p->N; ++n)
        if (!idx[n]) { set_error("dgpu_download_slab: idx[%d] null", n); return DGPU_ERR_ARG; }
    if (p->layout == DGPU_LAYOUT_MORTON) {
        // key order, indices decoded on the host (pext by each mode's mask)
        std::vector<uint64_t> keys(p->nnz);
        DGPU_CUDA(cudaMemcpyAsync(keys.data(), p->mkeys, p->nnz * sizeof(uint64_t),
                                  cudaMemcpyDeviceToHost, p->stream));
        DGPU_CUDA(cudaMemcpyAsync(vals, p->mvals, p->nnz * sizeof(float), cudaMemcpyDeviceToHost,
                                  p->stream));
        DGPU_TRY(sync_checked(*p));
        const MortonDec d = morton_decoder(*p);
        for (int n = 0; n < p->N; ++n)
            for (uint64_t i = 0; i < p->nnz; ++i) {
                uint32_t x = 0;
                for (int j = 0; j < d.bits[n]; ++j) x |= (uint32_t)((keys[i] >> d.pos[n][j]) & 1u) << j;
                idx[n][i] = x;
            }
        return DGPU_OK;
    }
    const Slab& s = (p->layout == DGPU_LAYOUT_NCOPY) ? p->slab[p->next_mode] : p->slab[p->cur];
    DGPU_CUDA(cudaMemcpyAsync(vals, s.vals, p->nnz * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    for (int n = 0; n < p->N; ++n) {
        if (!idx[n]) { set_error("dgpu_download_slab: idx[%d] null", n); return DGPU_ERR_ARG; }
        DGPU_CUDA(cudaMemcpyAsync(idx[n], s.idx[n], p->nnz * sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, p->stream));
    }
    DGPU_TRY(sync_checked(*p));
    return DGPU_OK;
}

int dgpu_plan_morton(dgpu_plan* plan, uint64_t* mask, uint8_t* bits, uint64_t* keys, float* vals) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    if (p->layout != DGPU_LAYOUT_MORTON) {
        set_error("dgpu_plan_morton: plan layout is not Morton"); return DGPU_ERR_NOT_BUILT;
    }
    for (int n = 0; n < p->N; ++n) {
        if (mask) mask[n] = p->mmask[n];
        if (bits) bits[n] = p->mbits[n];
    }
    if (keys)
        DGPU_CUDA(cudaMemcpyAsync(keys, p->mkeys, p->nnz * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                  p->stream));
    if (vals)
        DGPU_CUDA(cudaMemcpyAsync(vals, p->mvals, p->nnz * sizeof(float), cudaMemcpyDeviceToHost,
                                  p->stream));
    DGPU_TRY(sync_checked(*p));
    return DGPU_OK;
}

int dgpu_download_copy(dgpu_plan* plan, int k, float* vals, uint32_t* const* idx) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    MODE_GUARD(p, k);
    if (p->layout != DGPU_LAYOUT_NCOPY) {
        set_error("dgpu_download_copy: plan layout is not NCopy"); return DGPU_ERR_NOT_BUILT;
    }
    if (!vals || !idx) { set_error("dgpu_download_copy: null"); return DGPU_ERR_ARG; }
    const Slab& s = p->slab[k];
    DGPU_CUDA(cudaMemcpyAsync(vals, s.vals, p->nnz * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    for (int n = 0; n < p->N; ++n)
        DGPU_CUDA(cudaMemcpyAsync(idx[n], s.idx[n], p->nnz * sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, p->stream));
    DGPU_TRY(sync_checked(*p));
    return DGPU_OK;
}

void dgpu_cp_options_default(dgpu_cp_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->max_iters = 50;
    o->tol = 1e-4;
    o->seed = 42;
    o->ridge = 1e-10;
    o->kernel = DGPU_CP_GAUSS_SEIDEL;
    o->solve_fp64 = 1;
    o->use_init = 0;
    o->verbose = 0;
    o->graphs = 1;
}

namespace {
// BF16-gather CP-ALS gathers the last mode's rows in FP32: the last mode's
// Yhat gives the fit's <X, M> = sum_r lambda_r <Y[N-1][:, r], Yhat[N-1][:, r]>
// (src/dynasor_linalg.cpp:324-366), and a Yhat computed from BF16-rounded
// factors moves that term, and with it the fit, by up to ~2e-4 on small
// well-fitted tensors (FP64 CP-ALS with BF16-rounded gathers on a 20 x 25 x
// 30 rank-5 tensor; ~6e-6 with the last mode in FP32).  Set for the length
// of one run, reset on every exit path.
// DGPU_CP_AUTO: the compute plan's kernel (the reference's pick_auto rule,
// src/dynasor_preprocess.cpp:1252-1285); with verbose the plan banner is
// printed first, as the reference's driver prints dyn_print_compute_plan.
int resolve_kernel(Plan& p, dgpu_cp_options& o) {
    if (o.kernel != DGPU_CP_GAUSS_SEIDEL && o.kernel != DGPU_CP_JACOBI && o.kernel != DGPU_CP_AUTO) {
        set_error("cpals: unknown kernel %d", o.kernel);
        return DGPU_ERR_ARG;
    }
    if (o.kernel != DGPU_CP_AUTO) return DGPU_OK;
    dgpu_compute_plan cp;
    DGPU_TRY(dgpu_build_compute_plan(reinterpret_cast<dgpu_plan*>(&p), nullptr, &cp));
    o.kernel = cp.kernel;
    if (o.verbose) {
        char banner[1024];
        if (dgpu_format_compute_plan(&cp, "[plan]", banner, sizeof(banner)) == DGPU_OK)
            std::fputs(banner, stdout);
    }
    return DGPU_OK;
}

struct LastModeFp32 {
    std::vector<Plan*> ps;
    LastModeFp32(Plan* const* p, int count) : ps(p, p + count) {
        for (Plan* q : ps) q->fp32_gather_mode = q->N - 1;
    }
    ~LastModeFp32() {
        for (Plan* q : ps) q->fp32_gather_mode = -1;
    }
};
}  // namespace

int dgpu_cpals(dgpu_plan* plan, const dgpu_cp_options* opt, dgpu_cp_result* res,
               double* fit_history) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    if (!opt || !res) { set_error("dgpu_cpals: null argument"); return DGPU_ERR_ARG; }
    if (opt->max_iters < 0) { set_error("dgpu_cpals: max_iters < 0"); return DGPU_ERR_ARG; }
    dgpu_cp_options o = *opt;
    DGPU_TRY(resolve_kernel(*p, o));
    LastModeFp32 fp32_last(&p, 1);
    return cpals_run(*p, o, *res, fit_history);
}

int dgpu_cpals_batch(dgpu_plan* const* plans, int count, const dgpu_cp_options* opt,
                     dgpu_cp_result* res, double* fit_history) {
    if (!plans || !opt || !res || count < 1) {
        set_error("dgpu_cpals_batch: null argument or count < 1");
        return DGPU_ERR_ARG;
    }
    if (opt->max_iters < 0) { set_error("dgpu_cpals_batch: max_iters < 0"); return DGPU_ERR_ARG; }
    std::vector<Plan*> ps(count);
    for (int k = 0; k < count; ++k) {
        ps[k] = reinterpret_cast<Plan*>(plans[k]);
        if (!ps[k]) { set_error("dgpu_cpals_batch: plan %d is null", k); return DGPU_ERR_ARG; }
        if (ps[k]->device != ps[0]->device) {
            set_error("dgpu_cpals_batch: plans on different devices (%d, %d)", ps[0]->device,
                      ps[k]->device);
            return DGPU_ERR_ARG;
        }
        for (int j = 0; j < k; ++j)
            if (ps[j] == ps[k]) { set_error("dgpu_cpals_batch: plan %d repeated", k); return DGPU_ERR_ARG; }
    }
    Plan* p = ps[0];
    API_GUARD(p);
    // one kernel for the batch: DGPU_CP_AUTO must resolve alike on every plan
    dgpu_cp_options o = *opt;
    if (o.kernel == DGPU_CP_AUTO) {
        int kind = -1;
        for (int k = 0; k < count; ++k) {
            dgpu_cp_options ok = o;
            ok.verbose = 0;
            DGPU_TRY(resolve_kernel(*ps[k], ok));
            if (kind >= 0 && ok.kernel != kind) {
                set_error("dgpu_cpals_batch: the plans' compute plans choose different kernels; "
                          "pass DGPU_CP_GAUSS_SEIDEL or DGPU_CP_JACOBI");
                return DGPU_ERR_ARG;
            }
            kind = ok.kernel;
        }
        o.kernel = kind;
    }
    DGPU_TRY(resolve_kernel(*p, o));
    LastModeFp32 fp32_last(ps.data(), count);
    return cpals_batch_run(ps.data(), count, o, res, fit_history);
}

int dgpu_cpals_multistart(dgpu_plan* plan, int restarts, const dgpu_cp_options* opt,
                          dgpu_cp_result* res, double* fit_history) {
    Plan* p = reinterpret_cast<Plan*>(plan);
    API_GUARD(p);
    if (!opt || !res) { set_error("dgpu_cpals_multistart: null argument"); return DGPU_ERR_ARG; }
    if (p->layout == DGPU_LAYOUT_MORTON) {
        set_error("dgpu_cpals_multistart: runs on the PingPong and NCopy layouts");
        return DGPU_ERR_ARG;
    }
    if (opt->max_iters < 0) { set_error("dgpu_cpals_multistart: max_iters < 0"); return DGPU_ERR_ARG; }
    if (restarts < 1 || p->R % restarts != 0) {
        set_error("dgpu_cpals_multistart: the plan rank %d is not a multiple of %d restarts", p->R,
                  restarts);
        return DGPU_ERR_ARG;
    }
    if (p->R / restarts > 64) {
        set_error("dgpu_cpals_multistart: rank per restart %d exceeds 64", p->R / restarts);
        return DGPU_ERR_ARG;
    }
    dgpu_cp_options o = *opt;
    DGPU_TRY(resolve_kernel(*p, o));
    LastModeFp32 fp32_last(&p, 1);
    return cpals_multistart_run(*p, restarts, o, res, fit_history);
}

}  // extern "C"
