// ============================================================================
//  flycoo_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
//  A plain CPU restatement of the Dynasor+ hot path (single-threaded except
//  the FP64 CP-ALS, whose per-row sums and Gram blocks run under OpenMP in
//  an order that does not depend on the thread count), used
//  only as a checker by tests/, __graft_entry__.smoke() and the CPU-baseline
//  leg of bench.py.  The product library never links or calls it.
//
//  What it restates (reference file:line in brackets):
//    * pick_mn / shard geometry       [src/dynasor_preprocess.cpp:69-99, 2031-2048]
//    * per-mode shard counts and the stable mode-0 shard scatter
//                                     [src/dynasor_preprocess.cpp:113-281]
//    * greedy LPT schedule            [src/dynasor_preprocess.cpp:291-323]
//    * shard_begin/end + cursor table [src/dynasor_preprocess.cpp:332-463]
//    * kernel classification          [src/dynasor_preprocess.cpp:2087-2095]
//    * the remap permutation          [src/dynasor_kernel.cpp:220-227,
//                                      src/dynasor.cpp:428-536]
//    * the single-pass fiber sort     [src/dynasor_preprocess.cpp:471-521,
//                                      2225-2256]
//    * NCopy copy population          [src/dynasor_preprocess.cpp:541-593,
//                                      1740-1790]
//    * the per-nnz MTTKRP arithmetic  [src/dynasor_kernel.cpp:91-229]
//      both as the reference's own FP32 fold (fmaf, slab order) and in FP64
//    * CP-ALS (Gauss-Seidel) in FP64  [src/dynasor_cpals.cpp:42-396,
//                                      src/dynasor_linalg.cpp:47-402]
//    * the Morton bit plan, keys and key order
//                                     [src/dynasor_morton.cpp:43-134, 143-352]
//
//  The LPT sort uses std::sort with the same strict-weak ordering as the
//  reference, so shard order on count ties follows the same libstdc++
//  introsort; that is the one place where "the same library call" is the
//  specification.
// ============================================================================
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <queue>
#include <random>
#include <vector>

namespace {

constexpr int kMaxModes = 8;

uint32_t round_up_pow2(uint32_t x) {
    if (x <= 1) return 1;
    uint32_t r = 1;
    while (r < x) r <<= 1;
    return r;
}
int log2_ceil(uint32_t x) {
    int k = 0;
    while ((uint32_t(1) << k) < x) ++k;
    return k;
}

// Rows per super-shard for a mode of size I built for T workers.
uint32_t rows_per_shard(uint32_t I, int T) {
    if (I <= (uint32_t)T) return 1;
    uint32_t mn = I / ((uint32_t)T * 4u);
    if (mn < 1u) mn = 1u;
    if (mn < 16u) mn = 16u;
    if (mn > 16384u) mn = 16384u;
    if (mn > I) mn = I;
    return round_up_pow2(mn);
}

struct Slab {
    std::vector<float>                 v;
    std::vector<std::vector<uint32_t>> ix;
};

struct Oracle {
    int N = 0, T = 1;
    uint64_t nnz = 0;
    uint32_t dims[kMaxModes] = {};
    uint32_t mn[kMaxModes] = {};
    int      shift[kMaxModes] = {};
    uint32_t K[kMaxModes] = {};
    int      kclass[kMaxModes] = {};
    std::vector<std::vector<uint64_t>> count;        // [n][s]
    std::vector<std::vector<uint64_t>> sbeg, send;   // [n][s]
    std::vector<std::vector<std::vector<uint32_t>>> sched; // [n][tid] -> shards
    std::vector<std::vector<uint64_t>> cursor;       // [n][tid*stride + s']
    std::vector<size_t> stride;                      // [n]
    Slab cur;                                        // current primary slab
};

// Stable scatter of `src` positions listed in `order` into buckets.
void stable_bucket_scatter(const Slab& src, const std::vector<uint64_t>& order,
                           const std::vector<uint32_t>& bucket_of,
                           std::vector<uint64_t> start, Slab& dst, int N)
{
    for (uint64_t p = 0; p < order.size(); ++p) {
        const uint64_t i = order[p];
        const uint64_t d = start[bucket_of[p]]++;
        dst.v[d] = src.v[i];
        for (int w = 0; w < N; ++w) dst.ix[w][d] = src.ix[w][i];
    }
}

Slab make_slab(uint64_t nnz, int N) {
    Slab s;
    s.v.assign(nnz, 0.f);
    s.ix.assign(N, std::vector<uint32_t>(nnz, 0));
    return s;
}

} // namespace

extern "C" {

// ---------------------------------------------------------------------------
//  Build: geometry, counts, mode-0 stable shard sort, LPT, remap plan.
// ---------------------------------------------------------------------------
void* orc_create(int N, uint64_t nnz, const uint32_t* dims, const float* vals,
                 const uint32_t* const* idx, int threads)
{
    auto* o = new Oracle();
    o->N = N; o->T = threads; o->nnz = nnz;
    for (int n = 0; n < N; ++n) {
        o->dims[n]  = dims[n];
        o->mn[n]    = rows_per_shard(dims[n], threads);
        o->shift[n] = log2_ceil(o->mn[n]);
        o->K[n]     = (dims[n] + o->mn[n] - 1) / o->mn[n];
        if (o->K[n] == 0) o->K[n] = 1;
        const double afl = (double)nnz / (double)std::max<uint32_t>(1u, dims[n]);
        o->kclass[n] = afl >= 32.0 ? 2 : (afl >= 8.0 ? 1 : 0);
    }

    // Shard counts of every mode.
    o->count.assign(N, {});
    for (int n = 0; n < N; ++n) {
        o->count[n].assign(o->K[n], 0);
        for (uint64_t i = 0; i < nnz; ++i) o->count[n][idx[n][i] >> o->shift[n]]++;
    }
    o->sbeg.assign(N, {}); o->send.assign(N, {});
    for (int n = 0; n < N; ++n) {
        uint64_t c = 0;
        o->sbeg[n].resize(o->K[n]); o->send[n].resize(o->K[n]);
        for (uint32_t s = 0; s < o->K[n]; ++s) {
            o->sbeg[n][s] = c; c += o->count[n][s]; o->send[n][s] = c;
        }
    }

    // Stable scatter of the input order into mode-0 shard order.
    Slab in = make_slab(nnz, N);
    std::memcpy(in.v.data(), vals, nnz * sizeof(float));
    for (int n = 0; n < N; ++n) std::memcpy(in.ix[n].data(), idx[n], nnz * 4);
    std::vector<uint64_t> order(nnz);
    std::iota(order.begin(), order.end(), 0);
    std::vector<uint32_t> b0(nnz);
    for (uint64_t i = 0; i < nnz; ++i) b0[i] = in.ix[0][i] >> o->shift[0];
    o->cur = make_slab(nnz, N);
    stable_bucket_scatter(in, order, b0, o->sbeg[0], o->cur, N);

    // Greedy LPT per mode.
    o->sched.assign(N, std::vector<std::vector<uint32_t>>(threads));
    for (int n = 0; n < N; ++n) {
        const uint64_t* cn = o->count[n].data();
        std::vector<uint32_t> ord(o->K[n]);
        std::iota(ord.begin(), ord.end(), 0u);
        std::sort(ord.begin(), ord.end(),
                  [&](uint32_t a, uint32_t b) { return cn[a] > cn[b]; });
        using QE = std::pair<uint64_t, int>;
        std::priority_queue<QE, std::vector<QE>, std::greater<QE>> heap;
        for (int t = 0; t < threads; ++t) heap.push({0ull, t});
        for (uint32_t s : ord) {
            if (cn[s] == 0) continue;
            QE top = heap.top(); heap.pop();
            o->sched[n][top.second].push_back(s);
            heap.push({top.first + cn[s], top.second});
        }
    }

    // Cursor table: stride = K_{n+1} rounded up to 8 entries.
    o->cursor.assign(N, {});
    o->stride.assign(N, 0);
    for (int n = 0; n < N; ++n) {
        const int nm = (n + 1) % N;
        const size_t stride = ((size_t)o->K[nm] + 7) & ~(size_t)7;
        o->stride[n] = stride;
        std::vector<int> owner(o->K[n], -1);
        for (int t = 0; t < threads; ++t)
            for (uint32_t s : o->sched[n][t]) owner[s] = t;
        std::vector<uint64_t> hist((size_t)threads * stride, 0);
        for (uint64_t i = 0; i < nnz; ++i) {
            const int t = owner[in.ix[n][i] >> o->shift[n]];
            if (t >= 0) hist[(size_t)t * stride + (in.ix[nm][i] >> o->shift[nm])]++;
        }
        o->cursor[n].assign((size_t)threads * stride, 0);
        for (uint32_t s = 0; s < o->K[nm]; ++s) {
            uint64_t c = o->sbeg[nm][s];
            for (int t = 0; t < threads; ++t) {
                o->cursor[n][(size_t)t * stride + s] = c;
                c += hist[(size_t)t * stride + s];
            }
        }
    }
    return o;
}

void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }

void orc_modes(void* h, int* shift, uint32_t* K, int* kclass) {
    auto* o = static_cast<Oracle*>(h);
    for (int n = 0; n < o->N; ++n) { shift[n] = o->shift[n]; K[n] = o->K[n]; kclass[n] = o->kclass[n]; }
}

void orc_shards(void* h, int n, uint64_t* beg, uint64_t* end) {
    auto* o = static_cast<Oracle*>(h);
    std::memcpy(beg, o->sbeg[n].data(), o->K[n] * 8);
    std::memcpy(end, o->send[n].data(), o->K[n] * 8);
}

int orc_schedule(void* h, int n, uint32_t* counts, uint32_t* flat) {
    auto* o = static_cast<Oracle*>(h);
    int k = 0;
    for (int t = 0; t < o->T; ++t) {
        counts[t] = (uint32_t)o->sched[n][t].size();
        for (uint32_t s : o->sched[n][t]) flat[k++] = s;
    }
    return k;
}

size_t orc_cursors(void* h, int n, uint64_t* out) {
    auto* o = static_cast<Oracle*>(h);
    if (out) std::memcpy(out, o->cursor[n].data(), o->cursor[n].size() * 8);
    return o->cursor[n].size();
}

void orc_get_slab(void* h, float* vals, uint32_t* const* idx) {
    auto* o = static_cast<Oracle*>(h);
    std::memcpy(vals, o->cur.v.data(), o->nnz * 4);
    for (int n = 0; n < o->N; ++n) std::memcpy(idx[n], o->cur.ix[n].data(), o->nnz * 4);
}

void orc_set_slab(void* h, const float* vals, const uint32_t* const* idx) {
    auto* o = static_cast<Oracle*>(h);
    std::memcpy(o->cur.v.data(), vals, o->nnz * 4);
    for (int n = 0; n < o->N; ++n) std::memcpy(o->cur.ix[n].data(), idx[n], o->nnz * 4);
}

// Stable sort of every mode-n shard of the current slab by row.
void orc_fiber_sort(void* h, int n) {
    auto* o = static_cast<Oracle*>(h);
    Slab out = make_slab(o->nnz, o->N);
    for (uint32_t s = 0; s < o->K[n]; ++s) {
        const uint64_t b = o->sbeg[n][s], e = o->send[n][s];
        if (e == b) continue;
        const uint32_t base = s << o->shift[n];
        std::vector<uint64_t> start(o->mn[n] + 1, 0);
        for (uint64_t i = b; i < e; ++i) start[o->cur.ix[n][i] - base + 1]++;
        for (uint32_t k = 0; k < o->mn[n]; ++k) start[k + 1] += start[k];
        for (uint64_t i = b; i < e; ++i) {
            const uint64_t d = b + start[o->cur.ix[n][i] - base]++;
            out.v[d] = o->cur.v[i];
            for (int w = 0; w < o->N; ++w) out.ix[w][d] = o->cur.ix[w][i];
        }
    }
    o->cur.v.swap(out.v);
    o->cur.ix.swap(out.ix);
}

// Processing order of mode n: LPT thread order, shard list order, slab order.
static std::vector<uint64_t> processing_order(const Oracle* o, int n) {
    std::vector<uint64_t> ord;
    ord.reserve(o->nnz);
    for (int t = 0; t < o->T; ++t)
        for (uint32_t s : o->sched[n][t])
            for (uint64_t i = o->sbeg[n][s]; i < o->send[n][s]; ++i) ord.push_back(i);
    return ord;
}

// The mode-n remap: stable counting sort of the processing order by the
// mode-(n+1) shard id.  Replaces the current slab.
void orc_remap(void* h, int n) {
    auto* o = static_cast<Oracle*>(h);
    const int nm = (n + 1) % o->N;
    std::vector<uint64_t> ord = processing_order(o, n);
    std::vector<uint32_t> bk(ord.size());
    for (size_t p = 0; p < ord.size(); ++p) bk[p] = o->cur.ix[nm][ord[p]] >> o->shift[nm];
    Slab out = make_slab(o->nnz, o->N);
    stable_bucket_scatter(o->cur, ord, bk, o->sbeg[nm], out, o->N);
    o->cur.v.swap(out.v);
    o->cur.ix.swap(out.ix);
}

// One PingPong process(n): optional fiber sort, then the remap.
void orc_process_layout(void* h, int n, int fiber_on) {
    auto* o = static_cast<Oracle*>(h);
    if (fiber_on && o->kclass[n] == 2) orc_fiber_sort(h, n);
    orc_remap(h, n);
}

// ---------------------------------------------------------------------------
//  MTTKRP arithmetic.  Y[w] are I_w x Rp row-major FP32 factor matrices.
//  out is I_n x Rp.
// ---------------------------------------------------------------------------

// The reference kernel's own FP32 fold: per nnz, prod = val*Y[w0] (*middle
// factors in increasing w) and out = fmaf(prod, Y[w_last], out), visiting
// the nonzeros in the given slab order (each row's contributions in that
// order).  Matches src/dynasor_kernel.cpp:158-202 bit for bit.
void orc_mttkrp_f32_fold(int N, uint64_t nnz, const float* vals,
                         const uint32_t* const* idx, int n, int Rp,
                         const float* const* Y, float* out, uint32_t I_n)
{
    std::memset(out, 0, (size_t)I_n * Rp * sizeof(float));
    const int w0 = (n == 0) ? 1 : 0;
    int wl = -1;
    for (int w = N - 1; w >= 0; --w) if (w != n && w != w0) { wl = w; break; }
    std::vector<float> prod(Rp);
    for (uint64_t i = 0; i < nnz; ++i) {
        const float v = vals[i];
        const float* y0 = Y[w0] + (size_t)idx[w0][i] * Rp;
        for (int c = 0; c < Rp; ++c) prod[c] = v * y0[c];
        for (int w = 0; w < N; ++w) {
            if (w == n || w == w0 || w == wl) continue;
            const float* yw = Y[w] + (size_t)idx[w][i] * Rp;
            for (int c = 0; c < Rp; ++c) prod[c] = prod[c] * yw[c];
        }
        float* o = out + (size_t)idx[n][i] * Rp;
        if (wl >= 0) {
            const float* yl = Y[wl] + (size_t)idx[wl][i] * Rp;
            for (int c = 0; c < Rp; ++c) o[c] = std::fmaf(prod[c], yl[c], o[c]);
        } else {
            for (int c = 0; c < Rp; ++c) o[c] = o[c] + prod[c];
        }
    }
}

// Exact-as-possible MTTKRP: products and sums in FP64 from FP32 inputs.
// Ranks >= R are skipped (padding).  Follows src/dynasor_reference.cpp:29-49.
void orc_mttkrp_f64(int N, uint64_t nnz, const float* vals,
                    const uint32_t* const* idx, int n, int R, int Rp,
                    const float* const* Y, double* out, uint32_t I_n)
{
    // rows in parallel over a stable row grouping of the nonzeros: each row
    // adds its terms in nonzero order, as a serial loop over the nonzeros
    // would, so the result does not depend on the thread count
    std::vector<uint64_t> rp((size_t)I_n + 1, 0);
    for (uint64_t i = 0; i < nnz; ++i) ++rp[(size_t)idx[n][i] + 1];
    for (uint32_t r = 0; r < I_n; ++r) rp[r + 1] += rp[r];
    std::vector<uint64_t> perm(nnz);
    {
        std::vector<uint64_t> cur(rp.begin(), rp.end() - 1);
        for (uint64_t i = 0; i < nnz; ++i) perm[cur[idx[n][i]]++] = i;
    }
#pragma omp parallel
    {
        std::vector<double> t(R);
#pragma omp for schedule(dynamic, 256)
        for (int64_t row = 0; row < (int64_t)I_n; ++row) {
            double* o = out + (size_t)row * Rp;
            for (int r = 0; r < Rp; ++r) o[r] = 0.0;
            for (uint64_t k = rp[row]; k < rp[row + 1]; ++k) {
                const uint64_t i = perm[k];
                const double v = vals[i];
                for (int r = 0; r < R; ++r) t[r] = v;
                for (int w = 0; w < N; ++w) {
                    if (w == n) continue;
                    const float* yw = Y[w] + (size_t)idx[w][i] * Rp;
                    for (int r = 0; r < R; ++r) t[r] *= (double)yw[r];
                }
                for (int r = 0; r < R; ++r) o[r] += t[r];
            }
        }
    }
}

// Model values at the nonzeros: sum_r lambda_r prod_w Y[w][i_w, r]  (FP64).
void orc_model_values(int N, uint64_t nnz, const uint32_t* const* idx, int R,
                      int Rp, const float* const* Y, const float* lambda,
                      double* out)
{
    for (uint64_t i = 0; i < nnz; ++i) {
        double s = 0;
        for (int r = 0; r < R; ++r) {
            double p = lambda ? (double)lambda[r] : 1.0;
            for (int w = 0; w < N; ++w) p *= (double)Y[w][(size_t)idx[w][i] * Rp + r];
            s += p;
        }
        out[i] = s;
    }
}

// ---------------------------------------------------------------------------
//  CP-ALS initialisation, restated: splitmix64 step of (seed, n) seeds a
//  std::mt19937_64, rows drawn with std::normal_distribution<float>(0,1);
//  padding columns zero.  [src/dynasor_cpals.cpp:42-69]
// ---------------------------------------------------------------------------
void orc_init_factor(uint64_t seed, int n, uint32_t rows, int R, int Rp, float* Y)
{
    uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (uint64_t)(n + 1);
    z ^= z >> 30; z *= 0xBF58476D1CE4E5B9ULL;
    z ^= z >> 27; z *= 0x94D049BB133111EBULL;
    z ^= z >> 31;
    std::mt19937_64 rng(z);
    std::normal_distribution<float> g(0.0f, 1.0f);
    for (uint32_t i = 0; i < rows; ++i) {
        float* y = Y + (size_t)i * Rp;
        for (int r = 0; r < R; ++r) y[r] = g(rng);
        for (int r = R; r < Rp; ++r) y[r] = 0.f;
    }
}

// U(0,1) inputs of the --verify benchmark: one std::mt19937_64(seed) shared
// across modes in order.  [src/main.cpp:326-337, 903-907]
void orc_uniform_factors(uint64_t seed, int N, const uint32_t* dims, int R,
                         int Rp, float* const* Y)
{
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> U(0.0f, 1.0f);
    for (int n = 0; n < N; ++n)
        for (uint32_t i = 0; i < dims[n]; ++i) {
            for (int r = 0; r < R; ++r) Y[n][(size_t)i * Rp + r] = U(rng);
            for (int r = R; r < Rp; ++r) Y[n][(size_t)i * Rp + r] = 0.f;
        }
}

// ---------------------------------------------------------------------------
//  FP64 Gauss-Seidel CP-ALS on the COO tensor (order-independent), from the
//  same initial factors as the reference.  fit_hist receives one fit per
//  iteration; returns the number of iterations run.  Y (in/out) are the
//  FP32 factor buffers (I_n x Rp); they receive the final factors.
// ---------------------------------------------------------------------------
int orc_cpals_f64(int N, uint64_t nnz, const uint32_t* dims, const float* vals,
                  const uint32_t* const* idx, int R, int Rp, int max_iters,
                  double tol, double ridge, float* const* Yio,
                  double* fit_hist, double* lambda_out, int flags)
{
    // flags bit 0: Jacobi; bit 1: the MTTKRP gathers factor entries rounded
    // to BF16 (round to nearest even, as a BF16 copy of FP32 factors holds
    // them), everything else FP64 -- the arithmetic of BF16-gather CP-ALS
    // without FP32 rounding
    const int jacobi = flags & 1;
    const bool bf16_any = (flags & 2) != 0;
    const bool bf16_last_fp32 = (flags & 4) != 0;   // the last mode gathers FP32
    std::vector<std::vector<double>> Y(N), Yh(N), G(N);
    for (int n = 0; n < N; ++n) {
        Y[n].assign((size_t)dims[n] * R, 0);
        for (uint32_t i = 0; i < dims[n]; ++i)
            for (int r = 0; r < R; ++r) Y[n][(size_t)i * R + r] = Yio[n][(size_t)i * Rp + r];
        Yh[n].assign((size_t)dims[n] * R, 0);
        G[n].assign((size_t)R * R, 0);
    }
    // Gram: partial sums over fixed 4096-row blocks, added in block order,
    // so the result does not depend on the OpenMP thread count
    auto gram = [&](int n) {
        const uint32_t I = dims[n];
        const uint32_t nb = (I + 4095) / 4096;
        std::vector<double> part((size_t)nb * R * R, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t blk = 0; blk < (int64_t)nb; ++blk) {
            double* g = &part[(size_t)blk * R * R];
            const uint32_t i1 = std::min<uint32_t>(I, (uint32_t)(blk + 1) * 4096);
            for (uint32_t i = (uint32_t)blk * 4096; i < i1; ++i) {
                const double* y = &Y[n][(size_t)i * R];
                for (int a = 0; a < R; ++a)
                    for (int b = 0; b < R; ++b) g[a * R + b] += y[a] * y[b];
            }
        }
        std::fill(G[n].begin(), G[n].end(), 0.0);
        for (uint32_t blk = 0; blk < nb; ++blk)
            for (int a = 0; a < R * R; ++a) G[n][a] += part[(size_t)blk * R * R + a];
    };
    for (int n = 0; n < N; ++n) gram(n);
    double tn2 = 0;
    for (uint64_t i = 0; i < nnz; ++i) tn2 += (double)vals[i] * vals[i];
    const double tn = std::sqrt(tn2);
    std::vector<double> lam(R, 1.0), V((size_t)R * R);
    double fit_prev = 0;
    int it = 0;
    // Row-grouped nonzero lists per mode (a stable counting sort by the
    // mode's index), so rows are summed in parallel without races and each
    // row's terms are added in the input's nonzero order whatever the
    // thread count.
    std::vector<std::vector<uint64_t>> rp(N);
    std::vector<std::vector<uint32_t>> perm(N);
    for (int n = 0; n < N; ++n) {
        rp[n].assign((size_t)dims[n] + 1, 0);
        for (uint64_t i = 0; i < nnz; ++i) ++rp[n][(size_t)idx[n][i] + 1];
        for (uint32_t r = 0; r < dims[n]; ++r) rp[n][r + 1] += rp[n][r];
        perm[n].resize(nnz);
        std::vector<uint64_t> cur(rp[n].begin(), rp[n].end() - 1);
        for (uint64_t i = 0; i < nnz; ++i) perm[n][cur[idx[n][i]]++] = (uint32_t)i;
    }
    std::vector<std::vector<double>> Yg(N);    // gathered copies (BF16-rounded)
    auto to_bf16 = [](double x) -> double {
        float f = (float)x;
        uint32_t u;
        std::memcpy(&u, &f, 4);
        if ((u & 0x7f800000u) != 0x7f800000u) u += 0x7fffu + ((u >> 16) & 1u);
        u &= 0xffff0000u;
        std::memcpy(&f, &u, 4);
        return (double)f;
    };
    auto mttkrp = [&](int n) {
        const bool bf16 = bf16_any && !(bf16_last_fp32 && n == N - 1);
        if (bf16)
            for (int w = 0; w < N; ++w) {
                if (w == n) continue;
                Yg[w].resize(Y[w].size());
                // the FP32 master copy is what the device rounds to BF16
                for (size_t k = 0; k < Y[w].size(); ++k) Yg[w][k] = to_bf16((float)Y[w][k]);
            }
        const std::vector<std::vector<double>>& Ys = bf16 ? Yg : Y;
#pragma omp parallel
        {
            std::vector<double> t(R);
#pragma omp for schedule(dynamic, 256)
            for (int64_t row = 0; row < (int64_t)dims[n]; ++row) {
                double* o = &Yh[n][(size_t)row * R];
                for (int r = 0; r < R; ++r) o[r] = 0.0;
                for (uint64_t k = rp[n][row]; k < rp[n][row + 1]; ++k) {
                    const uint32_t i = perm[n][k];
                    for (int r = 0; r < R; ++r) t[r] = vals[i];
                    for (int w = 0; w < N; ++w) {
                        if (w == n) continue;
                        const double* y = &Ys[w][(size_t)idx[w][i] * R];
                        for (int r = 0; r < R; ++r) t[r] *= y[r];
                    }
                    for (int r = 0; r < R; ++r) o[r] += t[r];
                }
            }
        }
    };
    for (; it < max_iters; ++it) {
        // Jacobi: every MTTKRP from the factors at the start of the
        // iteration (src/dynasor_cpals.cpp:270-278); the per-mode solves
        // below still use the freshest Grams.
        if (jacobi)
            for (int n = 0; n < N; ++n) mttkrp(n);
        for (int n = 0; n < N; ++n) {
            if (!jacobi) mttkrp(n);
            for (int a = 0; a < R * R; ++a) V[a] = 1.0;
            for (int m = 0; m < N; ++m)
                if (m != n) for (int a = 0; a < R * R; ++a) V[a] *= G[m][a];
            double dmax = 0;
            for (int a = 0; a < R; ++a) dmax = std::max(dmax, V[a * R + a]);
            const double eps = std::max(ridge * dmax, 0.0);
            for (int a = 0; a < R; ++a) V[a * R + a] += eps;
            for (int j = 0; j < R; ++j) {           // Cholesky, lower
                double s = V[j * R + j];
                for (int k = 0; k < j; ++k) s -= V[j * R + k] * V[j * R + k];
                if (s < 0) s = 0;
                const double d = std::sqrt(s);
                V[j * R + j] = d;
                const double inv = d > 0 ? 1.0 / d : 0.0;
                for (int i = j + 1; i < R; ++i) {
                    double q = V[i * R + j];
                    for (int k = 0; k < j; ++k) q -= V[i * R + k] * V[j * R + k];
                    V[i * R + j] = q * inv;
                }
            }
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < (int64_t)dims[n]; ++i) {   // row solves
                double* x = &Y[n][(size_t)i * R];
                const double* b = &Yh[n][(size_t)i * R];
                for (int r = 0; r < R; ++r) x[r] = b[r];
                for (int r = 0; r < R; ++r) {
                    double s = x[r];
                    for (int k = 0; k < r; ++k) s -= V[r * R + k] * x[k];
                    const double d = V[r * R + r];
                    x[r] = d > 0 ? s / d : 0.0;
                }
                for (int r = R - 1; r >= 0; --r) {
                    double s = x[r];
                    for (int k = r + 1; k < R; ++k) s -= V[k * R + r] * x[k];
                    const double d = V[r * R + r];
                    x[r] = d > 0 ? s / d : 0.0;
                }
            }
            for (int r = 0; r < R; ++r) {              // normalise
                double s = 0;
                for (uint32_t i = 0; i < dims[n]; ++i) s += Y[n][(size_t)i * R + r] * Y[n][(size_t)i * R + r];
                lam[r] = std::sqrt(s);
            }
            for (int r = 0; r < R; ++r) {
                const double inv = lam[r] > 1e-20 ? 1.0 / lam[r] : 0.0;
                for (uint32_t i = 0; i < dims[n]; ++i) Y[n][(size_t)i * R + r] *= inv;
            }
            gram(n);
        }
        double inner = 0;                              // fit
        for (int r = 0; r < R; ++r) {
            double s = 0;
            for (uint32_t i = 0; i < dims[N - 1]; ++i)
                s += Y[N - 1][(size_t)i * R + r] * Yh[N - 1][(size_t)i * R + r];
            inner += lam[r] * s;
        }
        double m2 = 0;
        for (int a = 0; a < R; ++a)
            for (int b = 0; b < R; ++b) {
                double hp = 1;
                for (int n = 0; n < N; ++n) hp *= G[n][a * R + b];
                m2 += lam[a] * lam[b] * hp;
            }
        double res2 = tn2 - 2 * inner + std::max(0.0, m2);
        if (res2 < 0) res2 = 0;
        const double fit = 1.0 - std::sqrt(res2) / std::max(tn, 1e-30);
        fit_hist[it] = fit;
        if (it > 0 && std::fabs(fit - fit_prev) < tol) { ++it; break; }
        fit_prev = fit;
    }
    for (int n = 0; n < N; ++n)
        for (uint32_t i = 0; i < dims[n]; ++i) {
            for (int r = 0; r < R; ++r) Yio[n][(size_t)i * Rp + r] = (float)Y[n][(size_t)i * R + r];
            for (int r = R; r < Rp; ++r) Yio[n][(size_t)i * Rp + r] = 0.f;
        }
    for (int r = 0; r < R; ++r) lambda_out[r] = lam[r];
    return it;
}

// NCopy copy population: copy k = remap of copy k-1 (no fiber sort in
// between), then a fiber sort of copy k when it is DenseFiber and fiber_on.
// The copy is written to (vals, idx); the current slab is left unchanged.
void orc_ncopy(void* h, int k, int fiber_on, float* vals, uint32_t* const* idx) {
    auto* o = static_cast<Oracle*>(h);
    Slab saved = o->cur;
    for (int c = 0; c < k; ++c) orc_remap(h, c);
    if (fiber_on && o->kclass[k] == 2) orc_fiber_sort(h, k);
    orc_get_slab(h, vals, idx);
    o->cur = std::move(saved);
}

// Morton layout: per-mode bit counts b_n = ceil(log2 I_n) (at least 1),
// bit positions handed out LSB-first round-robin over the modes that still
// need bits; key = OR over modes of the index bits placed at the mode's
// positions; (key, value) pairs stably sorted by key.  -1 when sum b_n > 64.
int orc_morton(int N, uint64_t nnz, const uint32_t* dims, const float* vals,
               const uint32_t* const* idx, uint64_t* mask, uint8_t* bits,
               uint64_t* keys_out, float* vals_out)
{
    int need[8] = {0};
    int total = 0;
    for (int n = 0; n < N; ++n) {
        int b = 1;
        if (dims[n] > 1) { b = 0; for (uint32_t m = dims[n] - 1; m; m >>= 1) ++b; }
        need[n] = b;
        bits[n] = (uint8_t)b;
        total += b;
        mask[n] = 0;
    }
    if (total > 64) return -1;
    std::vector<std::vector<int>> pos(N);
    int at = 0;
    while (at < total)
        for (int n = 0; n < N && at < total; ++n)
            if ((int)pos[n].size() < need[n]) { pos[n].push_back(at); mask[n] |= 1ull << at; ++at; }
    std::vector<std::pair<uint64_t, float>> kv(nnz);
    for (uint64_t i = 0; i < nnz; ++i) {
        uint64_t k = 0;
        for (int n = 0; n < N; ++n)
            for (int j = 0; j < need[n]; ++j)
                if ((idx[n][i] >> j) & 1u) k |= 1ull << pos[n][j];
        kv[i] = {k, vals[i]};
    }
    std::stable_sort(kv.begin(), kv.end(),
                     [](const std::pair<uint64_t, float>& a, const std::pair<uint64_t, float>& b) {
                         return a.first < b.first;
                     });
    for (uint64_t i = 0; i < nnz; ++i) { keys_out[i] = kv[i].first; vals_out[i] = kv[i].second; }
    return 0;
}

} // extern "C"
