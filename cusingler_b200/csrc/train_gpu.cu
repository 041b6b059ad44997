// Marker training on the device: per-label medians and the per-label-pair marker lists of the
// reference's DataParser::trainData (src/io.cpp:141-262 of STOmics/cusingler), with the same results
// as the host restatement in train.cpp.
//
// 1. Per-label medians of every gene, implicit zeros included (src/io.cpp:143-164).  The stored
//    entries of the label-grouped reference CSR are counted and scattered into one segment per
//    (label, gene); one warp per segment then takes the order statistics len/2 (and len/2 - 1 for an
//    even label size) of the segment's values with the implicit zeros placed where the reference's
//    sorted column has them (after the negative values, before the stored zeros and positives), by
//    radix selection on ordered float keys.
// 2. Per ordered label pair (a, b), the difference d_g = int(round((med_a[g] - med_b[g]) * 1e6))
//    (FP32 subtraction, FP64 scaling and rounding, as the reference writes it) of every gene.  The
//    reference's order for a pair is: difference descending, ties to the smaller gene -- one sort key
//    ((0x7fffffff - d) << 32 | g).  Its positive-difference prefix is the pair's marker list (the
//    concatenated lists `pair_genes`), the first n_common of the whole order feed the score-step
//    gene set and the first n_thre of the positive list the fine-tune gene pool.  One CTA per pair
//    sorts the pair's positive keys in shared memory (global scratch when they do not fit); when a
//    pair has fewer than n_common positive genes, its zero-difference genes follow in gene order and
//    then its negative ones, closest to zero first.

#include <algorithm>
#include <vector>

#include "device_util.cuh"
#include "kernels.cuh"
#include "sgr_internal.h"

namespace sgr {
namespace {

constexpr int PAIR_THREADS = 256;
constexpr int SMEM_KEYS = 8192;  // keys a pair sorts in shared memory (64 KB)

// (label, gene) counts of the stored entries of a label-grouped CSR; one warp per row
__global__ void label_gene_count_kernel(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                                        uint32_t R, const int32_t* __restrict__ colmap,
                                        const int32_t* __restrict__ row_label, uint32_t W,
                                        uint32_t* __restrict__ counts) {
    const int lane = threadIdx.x & 31;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < R; r += (gridDim.x * blockDim.x) >> 5) {
        const uint64_t base = (uint64_t)row_label[r] * W;
        for (int i = indptr[r] + lane; i < indptr[r + 1]; i += 32) {
            const int g = colmap[indices[i]];
            if (g >= 0) atomicAdd(counts + base + g, 1u);
        }
    }
}

// values scattered into their (label, gene) segment (order inside a segment is arbitrary)
__global__ void label_gene_fill_kernel(const float* __restrict__ data, const int32_t* __restrict__ indptr,
                                       const int32_t* __restrict__ indices, uint32_t R,
                                       const int32_t* __restrict__ colmap, const int32_t* __restrict__ row_label,
                                       uint32_t W, uint32_t* __restrict__ cursor, float* __restrict__ vals) {
    const int lane = threadIdx.x & 31;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < R; r += (gridDim.x * blockDim.x) >> 5) {
        const uint64_t base = (uint64_t)row_label[r] * W;
        for (int i = indptr[r] + lane; i < indptr[r + 1]; i += 32) {
            const int g = colmap[indices[i]];
            if (g >= 0) vals[atomicAdd(cursor + base + g, 1u)] = data[i];
        }
    }
}

// Median of one (label, gene) segment with the label's implicit zeros; one warp per segment.
__global__ void __launch_bounds__(256) median_kernel(const float* __restrict__ vals, const uint32_t* __restrict__ off,
                                                     const uint32_t* __restrict__ cnt,
                                                     const uint32_t* __restrict__ label_len, uint32_t L, uint32_t W,
                                                     float* __restrict__ med) {
    __shared__ int hist[8][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t n_seg = (uint64_t)L * W;
    for (uint64_t seg = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; seg < n_seg;
         seg += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const int n = (int)cnt[seg];
        const int len = (int)label_len[seg / W];
        float m = 0.f;
        if (n > 0) {
            const float* v = vals + off[seg];
            int neg = 0;
            for (int i = lane; i < n; i += 32) neg += v[i] < 0.f ? 1 : 0;
            const int p0 = __reduce_add_sync(FULL, neg), nz = len - n;
            // t-th value of the label's sorted column: negatives, the implicit zeros, then the rest
            auto at = [&](int t) -> float {
                if (t < p0) return key_float(warp_select(v, n, t, hist[warp], lane));
                if (t < p0 + nz) return 0.f;
                return key_float(warp_select(v, n, t - nz, hist[warp], lane));
            };
            if (len % 2 == 0) m = __fdiv_rn(__fadd_rn(at(len / 2), at(len / 2 - 1)), 2.0f);
            else m = at(len / 2);
        }
        if (lane == 0) med[seg] = m;
    }
}

__device__ __forceinline__ int scaled_diff(float a, float b) {
    return (int)round(__dmul_rn((double)__fsub_rn(a, b), 1e6));
}

// (0x7fffffff - d) in unsigned arithmetic: negative d would overflow a signed subtraction
__device__ __forceinline__ uint64_t desc_key(int d, uint32_t g) {
    return ((uint64_t)(0x7fffffffu - (uint32_t)d) << 32) | g;
}

// block-wide sum of per-thread values
__device__ int block_sum(int x, int* red) {
    x = __reduce_add_sync(FULL, x);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    __syncthreads();
    return t;
}

// Positive and zero difference counts of every ordered pair; one CTA per pair.
__global__ void __launch_bounds__(PAIR_THREADS) pair_count_kernel(const float* __restrict__ med, uint32_t L,
                                                                  uint32_t W, uint32_t* __restrict__ n_pos,
                                                                  uint32_t* __restrict__ n_zero) {
    __shared__ int red[PAIR_THREADS / 32];
    for (uint32_t p = blockIdx.x; p < L * L; p += gridDim.x) {
        const uint32_t a = p / L, b = p % L;
        int pos = 0, zero = 0;
        if (a != b)
            for (uint32_t g = threadIdx.x; g < W; g += blockDim.x) {
                const int d = scaled_diff(med[(size_t)a * W + g], med[(size_t)b * W + g]);
                pos += d > 0;
                zero += d == 0;
            }
        pos = block_sum(pos, red);
        zero = block_sum(zero, red);
        if (threadIdx.x == 0) {
            n_pos[p] = (uint32_t)pos;
            n_zero[p] = (uint32_t)zero;
        }
    }
}

// Ascending bitonic sort of n (a power of two) keys by the whole block; keys in shared or global memory.
__device__ void block_bitonic(uint64_t* keys, int n) {
    for (int size = 2; size <= n; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < (n >> 1); t += blockDim.x) {
                const int i = 2 * t - (t & (stride - 1)), j = i + stride;
                const uint64_t x = keys[i], y = keys[j];
                if ((x > y) == ((i & size) == 0)) {
                    keys[i] = y;
                    keys[j] = x;
                }
            }
            __syncthreads();
        }
}

__device__ __forceinline__ int pow2_ceil(int v) {
    int n = 1;
    while (n < v) n <<= 1;
    return n;
}

struct PairArgs {
    const float* med;
    uint32_t L, W;
    int n_common, n_thre;
    const uint32_t* n_pos;
    const uint32_t* n_zero;
    const uint32_t* pos_off;  // first entry of each pair's list in genes
    uint32_t* genes;          // concatenated positive lists
    uint8_t* in_common;       // W flags
    uint8_t* in_thre;         // W flags
    uint64_t* tmp;            // per CTA: pow2(W) keys for lists above SMEM_KEYS (nullptr: none needed)
    int tmp_keys;
};

// Marker lists of every ordered pair; one CTA per pair.
__global__ void __launch_bounds__(PAIR_THREADS) pair_rank_kernel(PairArgs a) {
    extern __shared__ uint64_t skeys[];  // SMEM_KEYS keys
    __shared__ int red[PAIR_THREADS / 32];
    __shared__ int s_n;
    const uint32_t L = a.L, W = a.W;
    for (uint32_t p = blockIdx.x; p < L * L; p += gridDim.x) {
        const uint32_t pa = p / L, pb = p % L;
        if (pa == pb) continue;  // block-uniform
        const float* m1 = a.med + (size_t)pa * W;
        const float* m2 = a.med + (size_t)pb * W;
        const int P = (int)a.n_pos[p], Z = (int)a.n_zero[p];
        // positive genes, sorted by (difference descending, gene ascending)
        {
            const int n2 = pow2_ceil(max(P, 1));
            uint64_t* keys = n2 <= SMEM_KEYS ? skeys : a.tmp + (size_t)blockIdx.x * a.tmp_keys;
            if (threadIdx.x == 0) s_n = 0;
            __syncthreads();
            for (uint32_t g = threadIdx.x; g < W; g += blockDim.x) {
                const int d = scaled_diff(m1[g], m2[g]);
                if (d > 0) keys[atomicAdd(&s_n, 1)] = desc_key(d, g);
            }
            __syncthreads();
            for (int i = P + threadIdx.x; i < n2; i += blockDim.x) keys[i] = ~0ull;
            __syncthreads();
            block_bitonic(keys, n2);
            uint32_t* out = a.genes + a.pos_off[p];
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                const uint32_t g = (uint32_t)keys[i];
                out[i] = g;
                if (i < a.n_thre) a.in_thre[g] = 1;
                if (i < a.n_common) a.in_common[g] = 1;
            }
            __syncthreads();
        }
        if (P >= a.n_common) continue;
        // then the zero-difference genes in gene order
        int need = a.n_common - P;
        int seen = 0;  // zero genes before this chunk
        for (uint32_t g0 = 0; g0 < W && seen < need; g0 += blockDim.x) {
            const uint32_t g = g0 + threadIdx.x;
            const bool z = g < W && scaled_diff(m1[g], m2[g]) == 0;
            const unsigned bal = __ballot_sync(FULL, z);
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            if (lane == 0) red[warp] = __popc(bal);
            __syncthreads();
            int before = seen;
            for (int w = 0; w < warp; ++w) before += red[w];
            int total = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) total += red[w];
            const int idx = before + __popc(bal & ((1u << lane) - 1u));
            if (z && idx < need) a.in_common[g] = 1;
            __syncthreads();
            seen += total;
        }
        if (P + Z >= a.n_common) continue;
        // then the negative ones, closest to zero first (difference descending, gene ascending)
        need = a.n_common - P - Z;
        const int N = (int)W - P - Z;
        const int n2 = pow2_ceil(max(N, 1));
        uint64_t* keys = n2 <= SMEM_KEYS ? skeys : a.tmp + (size_t)blockIdx.x * a.tmp_keys;
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        for (uint32_t g = threadIdx.x; g < W; g += blockDim.x) {
            const int d = scaled_diff(m1[g], m2[g]);
            if (d < 0) keys[atomicAdd(&s_n, 1)] = desc_key(d, g);
        }
        __syncthreads();
        for (int i = N + threadIdx.x; i < n2; i += blockDim.x) keys[i] = ~0ull;
        __syncthreads();
        block_bitonic(keys, n2);
        for (int i = threadIdx.x; i < need && i < N; i += blockDim.x) a.in_common[(uint32_t)keys[i]] = 1;
        __syncthreads();
    }
}

int grid_for(size_t items_per_block_unit, int per_sm) {
    return (int)std::max<size_t>(1, std::min<size_t>(items_per_block_unit, (size_t)device_sm_count() * per_sm));
}

}  // namespace

void rank_markers_device(const float* data, const int32_t* indices, const int32_t* indptr, uint32_t R,
                         uint32_t ref_cols, int64_t nnz, Markers& m, cudaStream_t s) {
    const uint32_t L = m.n_labels, W = m.W;
    const size_t LW = (size_t)L * W;
    if (LW >= (size_t)1 << 32) fail(SGR_ERR_UNSUPPORTED, "labels x genes above 2^32");
    if (nnz >= ((int64_t)1 << 32)) fail(SGR_ERR_UNSUPPORTED, "reference entries above 2^32");
    const int n_common = marker_count(L), n_thre = marker_count(2);
    if ((uint32_t)n_common > W) fail(SGR_ERR_UNSUPPORTED, "more marker genes per label pair than genes");

    std::vector<int32_t> row_label(std::max<uint32_t>(R, 1), 0);
    std::vector<uint32_t> label_len(L);
    for (uint32_t l = 0; l < L; ++l) {
        label_len[l] = m.ctidx[2 * l + 1];
        for (uint32_t r = m.ctidx[2 * l]; r < m.ctidx[2 * l] + m.ctidx[2 * l + 1]; ++r) row_label[r] = (int32_t)l;
    }
    DevBuf<int32_t> d_row_label, d_colmap;
    DevBuf<uint32_t> d_label_len, cnt, off, cursor;
    DevBuf<int32_t> scan_tmp;
    DevBuf<float> vals, med;
    d_row_label.upload(row_label, s);
    d_colmap.upload(m.ref_colmap, s);
    d_label_len.upload(label_len, s);
    cnt.ensure(LW + 1);
    off.ensure(LW + 1);
    cursor.ensure(LW + 1);
    SGR_CUDA(cudaMemsetAsync(cnt.p, 0, (LW + 1) * sizeof(uint32_t), s));
    const int row_grid = grid_for(((size_t)R + 7) / 8, 8);
    label_gene_count_kernel<<<row_grid, 256, 0, s>>>(indptr, indices, R, d_colmap.p, d_row_label.p, W, cnt.p);
    SGR_LAUNCH_CHECK();
    launch_exclusive_scan(reinterpret_cast<const int32_t*>(cnt.p), reinterpret_cast<int32_t*>(off.p), (uint32_t)LW,
                          scan_tmp.ensure(2 * ((LW + 4095) / 4096) + 1), s);
    SGR_CUDA(cudaMemcpyAsync(cursor.p, off.p, (LW + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    vals.ensure((size_t)std::max<int64_t>(nnz, 1));
    label_gene_fill_kernel<<<row_grid, 256, 0, s>>>(data, indptr, indices, R, d_colmap.p, d_row_label.p, W,
                                                    cursor.p, vals.p);
    SGR_LAUNCH_CHECK();
    med.ensure(LW);
    median_kernel<<<grid_for((LW + 7) / 8, 8), 256, 0, s>>>(vals.p, off.p, cnt.p, d_label_len.p, L, W, med.p);
    SGR_LAUNCH_CHECK();
    vals.release();

    const size_t LL = (size_t)L * L;
    DevBuf<uint32_t> n_pos, n_zero, pos_off, genes;
    n_pos.ensure(LL);
    n_zero.ensure(LL);
    const int pair_grid = grid_for(LL, 4);
    pair_count_kernel<<<pair_grid, PAIR_THREADS, 0, s>>>(med.p, L, W, n_pos.p, n_zero.p);
    SGR_LAUNCH_CHECK();
    std::vector<uint32_t> hp(LL), hz(LL);
    SGR_CUDA(cudaMemcpyAsync(hp.data(), n_pos.p, LL * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SGR_CUDA(cudaMemcpyAsync(hz.data(), n_zero.p, LL * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SGR_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> hoff(LL);
    uint64_t total = 0;
    bool big = false;
    for (size_t p = 0; p < LL; ++p) {
        hoff[p] = (uint32_t)total;
        total += hp[p];
        const int P = (int)hp[p], Z = (int)hz[p], N = (int)W - P - Z;
        if (P > SMEM_KEYS || (P + Z < n_common && N > SMEM_KEYS)) big = true;
    }
    if (total >= ((uint64_t)1 << 32)) fail(SGR_ERR_UNSUPPORTED, "pair marker lists above 2^32 entries");
    pos_off.upload(hoff, s);
    genes.ensure(std::max<uint64_t>(total, 1));
    DevBuf<uint8_t> flags;
    flags.ensure(2 * (size_t)W);
    SGR_CUDA(cudaMemsetAsync(flags.p, 0, 2 * (size_t)W, s));
    DevBuf<uint64_t> tmp;
    int tmp_keys = 0;
    if (big) {  // lists longer than shared memory holds sort in a global region per CTA
        tmp_keys = 1;
        while (tmp_keys < (int)W) tmp_keys <<= 1;
        tmp.ensure((size_t)pair_grid * tmp_keys);
    }
    PairArgs pa{med.p, L, W, n_common, n_thre, n_pos.p, n_zero.p, pos_off.p, genes.p, flags.p, flags.p + W,
                tmp.p, tmp_keys};
    const int smem = SMEM_KEYS * (int)sizeof(uint64_t);
    SGR_CUDA(cudaFuncSetAttribute(pair_rank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    pair_rank_kernel<<<pair_grid, PAIR_THREADS, smem, s>>>(pa);
    SGR_LAUNCH_CHECK();
    count_launch(5);

    m.pair_genes.resize(total);
    std::vector<uint8_t> hflags(2 * (size_t)W);
    if (total)
        SGR_CUDA(cudaMemcpyAsync(m.pair_genes.data(), genes.p, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SGR_CUDA(cudaMemcpyAsync(hflags.data(), flags.p, hflags.size(), cudaMemcpyDeviceToHost, s));
    SGR_CUDA(cudaStreamSynchronize(s));
    m.pair_idx.clear();
    for (size_t p = 0; p < LL; ++p) {
        if (p / L == p % L) {
            m.pair_idx.push_back(0);
            m.pair_idx.push_back(0);
        } else {
            m.pair_idx.push_back(hoff[p]);
            m.pair_idx.push_back(hp[p]);
        }
    }
    finish_markers(m, hflags.data(), hflags.data() + W);
}

}  // namespace sgr
