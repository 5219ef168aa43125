// ============================================================================
//  morton.cu -- the Morton (Z-curve) layout: one 64-bit key per nonzero
//  interleaving its mode indices, plus the value, sorted by key.
//
//  Replaces build_morton_layout (src/dynasor_morton.cpp:143-352).  The bit
//  plan is the reference's (the key format has to match for .dnp files and
//  for bit-exact keys): mode n gets b_n = ceil(log2 I_n) bits (at least 1),
//  handed out LSB-first round-robin over the modes that still need bits.
//
//  Build on the device: the COO sits in a slab; k_morton_encode writes each
//  key's low and high words into index columns 0 and 1 of the other slab
//  (pdep of every mode index by its mask); stable LSD partition passes
//  (8-bit digits, the remap's machinery) sort by the used key bits, low word
//  first; k_morton_pack writes keys and values to their own 12 B/nnz arrays
//  and the slabs are freed.  With distinct keys (distinct coordinates) the
//  order is the reference's std::sort order; equal keys keep input order.
// ============================================================================
#include "dgpu_internal.h"

#include <algorithm>
#include <utility>

namespace dgpu {

namespace {

int ceil_log2_idx(uint32_t v) {
    if (v <= 1) return 1;
    int b = 0;
    for (uint32_t m = v - 1; m; m >>= 1) ++b;
    return b;
}

struct Dims8 {
    uint32_t d[kMaxModes];
};

__device__ __forceinline__ uint64_t morton_encode(const MortonDec& d, int w, uint32_t x) {
    uint64_t k = 0;
    for (int j = 0; j < d.bits[w]; ++j) k |= (uint64_t)((x >> j) & 1u) << d.pos[w][j];
    return k;
}
__device__ __forceinline__ uint32_t morton_decode(const MortonDec& d, int w, uint64_t key) {
    uint32_t x = 0;
    for (int j = 0; j < d.bits[w]; ++j) x |= (uint32_t)((key >> d.pos[w][j]) & 1u) << j;
    return x;
}

__global__ void k_morton_encode(const __grid_constant__ SlabPtrs in, int N, uint64_t nnz,
                                const __grid_constant__ MortonDec d, const __grid_constant__ SlabOut out)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t key = 0;
        for (int w = 0; w < N; ++w) key |= morton_encode(d, w, in.idx[w][i]);
        out.vals[i] = in.vals[i];
        out.idx[0][i] = (uint32_t)key;
        out.idx[1][i] = (uint32_t)(key >> 32);
        for (int w = 2; w < N; ++w) out.idx[w][i] = 0u;
    }
}

__global__ void k_morton_pack(const __grid_constant__ SlabPtrs s, uint64_t nnz,
                              uint64_t* __restrict__ keys, float* __restrict__ vals)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        keys[i] = (uint64_t)s.idx[0][i] | ((uint64_t)s.idx[1][i] << 32);
        vals[i] = s.vals[i];
    }
}

// err bits: 1 an index outside its mode, 2 a key bit outside every mask,
// 4 keys not ascending
__global__ void k_morton_decode(const uint64_t* __restrict__ keys, const float* __restrict__ vals,
                                uint64_t nnz, int N, const __grid_constant__ MortonDec d,
                                const __grid_constant__ Dims8 dims,
                                const __grid_constant__ SlabOut out, int* __restrict__ err)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t key = keys[i];
        uint64_t back = 0;
        int e = 0;
        for (int w = 0; w < N; ++w) {
            uint32_t x = morton_decode(d, w, key);
            back |= morton_encode(d, w, x);
            if (x >= dims.d[w]) { e |= 1; x = 0; }
            out.idx[w][i] = x;
        }
        if (back != key) e |= 2;
        if (i > 0 && keys[i - 1] > key) e |= 4;
        out.vals[i] = vals[i];
        if (e) atomicOr(err, e);
    }
}

unsigned grid_for_nnz(uint64_t nnz) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((nnz + 255) / 256, 148ull * 8));
}

}  // namespace

void free_slabs(Plan& p) {
    for (auto& s : p.slab) {
        if (!s.raw) continue;
        dev_free(s.raw);
        p.device_bytes -= s.bytes;
        s = Slab{};
    }
}

bool morton_plan(int N, const uint32_t* dims, uint64_t* mask, uint8_t* bits) {
    int left[kMaxModes] = {};
    int total = 0;
    for (int n = 0; n < N; ++n) {
        left[n] = ceil_log2_idx(dims[n]);
        bits[n] = (uint8_t)left[n];
        total += left[n];
        mask[n] = 0;
    }
    if (total > 64) return false;
    int pos = 0;
    for (bool moved = true; pos < 64 && moved;) {
        moved = false;
        for (int n = 0; n < N && pos < 64; ++n) {
            if (left[n] == 0) continue;
            mask[n] |= 1ull << pos++;
            --left[n];
            moved = true;
        }
    }
    return true;
}

MortonDec morton_decoder(const Plan& p) {
    MortonDec d{};
    for (int w = 0; w < p.N; ++w) {
        int j = 0;
        for (int b = 0; b < 64 && j < 32; ++b)
            if ((p.mmask[w] >> b) & 1ull) d.pos[w][j++] = (uint8_t)b;
        d.bits[w] = (uint8_t)j;
    }
    return d;
}

int morton_build(Plan& p, int src) {
    if (!morton_plan(p.N, p.dims, p.mmask, p.mbits)) {
        set_error("morton: the mode sizes need more than 64 key bits (sum of ceil(log2 I_n))");
        return DGPU_ERR_ARG;
    }
    const MortonDec d = morton_decoder(p);
    int a = 1 - src;
    k_morton_encode<<<grid_for_nnz(p.nnz), 256, 0, p.stream>>>(
        slab_in(p.slab[src], p.N), p.N, p.nnz, d, slab_out(p.slab[a], p.N));
    DGPU_CUDA(cudaGetLastError());
    // stable LSD passes over the used key bits: low word, then high word
    int total = 0;
    for (int n = 0; n < p.N; ++n) total += p.mbits[n];
    int b = src;
    for (int word = 0; word < 2; ++word) {
        const int wbits = std::min(32, std::max(0, total - 32 * word));
        if (wbits == 0) break;
        const int passes = (wbits + kDefaultDigitBits - 1) / kDefaultDigitBits;
        const int dbits = (wbits + passes - 1) / passes;
        for (int k = 0; k < passes; ++k) {
            const int sh = k * dbits;
            const int nbits = std::min(dbits, wbits - sh);
            const uint32_t mask = (nbits >= 32) ? 0xffffffffu : ((1u << nbits) - 1u);
            DGPU_TRY(stable_partition(p, p.slab[a], p.ident, word, sh, mask, mask + 1u, p.slab[b]));
            std::swap(a, b);
        }
    }
    DGPU_TRY(dev_alloc(p, (void**)&p.mkeys, p.nnz * sizeof(uint64_t)));
    DGPU_TRY(dev_alloc(p, (void**)&p.mvals, p.nnz * sizeof(float)));
    k_morton_pack<<<grid_for_nnz(p.nnz), 256, 0, p.stream>>>(slab_in(p.slab[a], p.N), p.nnz,
                                                              p.mkeys, p.mvals);
    DGPU_CUDA(cudaGetLastError());
    DGPU_TRY(sync_checked(p));
    free_slabs(p);
    return DGPU_OK;
}

int morton_check_decode(Plan& p, int dst) {
    const MortonDec d = morton_decoder(p);
    Dims8 dims{};
    for (int n = 0; n < p.N; ++n) dims.d[n] = p.dims[n];
    DGPU_CUDA(cudaMemsetAsync(p.err_flag, 0, sizeof(int), p.stream));
    k_morton_decode<<<grid_for_nnz(p.nnz), 256, 0, p.stream>>>(
        p.mkeys, p.mvals, p.nnz, p.N, d, dims, slab_out(p.slab[dst], p.N), p.err_flag);
    DGPU_CUDA(cudaGetLastError());
    int err_h = 0;
    DGPU_CUDA(cudaMemcpyAsync(&err_h, p.err_flag, sizeof(int), cudaMemcpyDeviceToHost, p.stream));
    DGPU_CUDA(cudaStreamSynchronize(p.stream));
    DGPU_CUDA(cudaMemsetAsync(p.err_flag, 0, sizeof(int), p.stream));
    if (err_h & 1) { set_error("morton: a key decodes to an index outside its mode"); return DGPU_ERR_INDEX; }
    if (err_h & 2) { set_error("morton: a key has bits outside the mode masks"); return DGPU_ERR_IO; }
    if (err_h & 4) { set_error("morton: keys are not in ascending order"); return DGPU_ERR_IO; }
    return DGPU_OK;
}

}  // namespace dgpu
