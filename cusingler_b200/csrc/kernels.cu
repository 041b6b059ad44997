// Device kernels of the SingleR path (gather + rank, CSR compaction, SIMT correlation, per-label
// quantile selection, fine-tune correlation and selection) for sm_100a.
//
// Reference kernels restated here (STOmics/cusingler src/cusingler.cu):
//   csr2dense (204-281) + get_device_ref_lines (566-577) + csrFilter codes (src/io.cpp:470-523)
//       -> rank_kernel: one warp per cell row gathers the row's marker entries straight from the
//          CSR, counts each entry's #less / #equal through 256 value buckets in shared memory and
//          writes tie-averaged doubled centred ranks.
//   rankdata_bin3 / rankdata_batch / rankdata (745-801, 601-625, 158-179)
//       -> the same half-integer ranks 1 + #less + (#equal - 1)/2, as d = 2*rank - (G+1).
//   spearman (918-945)        -> corr_simt_kernel (fp32ref: fma chain over genes in order).
//   spearman_reduce (803-856) -> ft_corr_kernel (fp32ref: 128 contiguous chunks + pairwise tree).
//   percentile + get_label's argmax and flags (947-978, 1080-1133)
//       -> select_first_kernel (radix selection of the two order statistics per label, libstdc++
//          std::sort restated for NaN-bearing lists, std::minmax_element order for the argmax).

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <type_traits>

#include <cuda_fp16.h>

#include "kernels.cuh"
#include "sgr_internal.h"
#include "stl_order.h"
#include "device_util.cuh"

namespace sgr {
namespace {

// d at position p of a rank row already written to global memory by the warp's lanes (read through
// L2: other lanes wrote it).
__device__ __forceinline__ int stage_d(const unsigned char* row, int mode, int Kp, int p, int w) {
    if (mode == RANK_LIMBS) {
        const signed char* s = reinterpret_cast<const signed char*>(row);
        return limb_mult(w) * (int)__ldcg(s + p) + (int)__ldcg(s + 2 * Kp + p);
    }
    if (mode == RANK_F16)
        return __half2int_rn(__ushort_as_half(__ldcg(reinterpret_cast<const unsigned short*>(row) + p)));
    return __ldcg(reinterpret_cast<const short*>(row) + p);
}

__device__ __forceinline__ void stage_put(unsigned char* stage, int mode, int Kp, int p, int d, int w) {
    if (mode == RANK_LIMBS) {
        int h, l, s;
        split_limbs(d, w, h, l, s);
        int8_t* st = reinterpret_cast<int8_t*>(stage);
        st[p] = (int8_t)h;
        st[Kp + p] = (int8_t)l;
        st[2 * Kp + p] = (int8_t)s;
    } else if (mode == RANK_F16) {
        reinterpret_cast<__half*>(stage)[p] = __int2half_rn(d);
    } else {
        reinterpret_cast<int16_t*>(stage)[p] = (int16_t)d;
    }
}

// Bucket of a rank key's value on the map (x - fmin) * scale (0 for NaN and a zero scale).
__device__ __forceinline__ int rank_bucket(uint64_t key, float fmin, float scale) {
    const float t = (key_float((uint32_t)(key >> 32)) - fmin) * scale;
    return t >= 0.f ? min(255, (int)t) : 0;
}

constexpr int GATHER_CHUNKS = 8;  // 32-entry chunks of a row whose loads are in flight together

__global__ void __launch_bounds__(256) rank_kernel(RankLaunch a, int warp_bytes) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    // with a compact column map: its bits and per-word prefixes first, then the warps' buffers
    const int n_words = (int)((a.n_cols + 31) / 32);
    const int map_bytes = a.map_bits ? ((n_words * 6 + 15) & ~15) : 0;
    uint32_t* sbits = reinterpret_cast<uint32_t*>(smem);
    uint16_t* spre = reinterpret_cast<uint16_t*>(smem + 4 * n_words);
    if (a.map_bits) {
        for (int w = threadIdx.x; w < n_words; w += blockDim.x) {
            sbits[w] = a.map_bits[w];
            spre[w] = a.map_prefix[w];
        }
        __syncthreads();
    }
    // per warp: keys (cap x 8 B) | values by bucket (cap x 4 B) | 256 bucket counts / ends; the
    // output row is written in place in global memory (zeros first, then the stored entries)
    uint64_t* keys = reinterpret_cast<uint64_t*>(smem + map_bytes + (size_t)warp * warp_bytes);
    uint32_t* vals = reinterpret_cast<uint32_t*>(keys + a.cap);
    int* hist = reinterpret_cast<int*>(vals + a.cap);
    const uint32_t n_items = a.n_items_dev ? (uint32_t)*a.n_items_dev : a.n_items;
    for (uint32_t item = blockIdx.x * wpb + warp; item < n_items; item += gridDim.x * wpb) {
        RankItem it;
        if (a.items) {
            it = a.items[item];
        } else {
            it.row = a.row0 + item;
            it.group = 0;
            it.slot = item;
        }
        const RankGroup g = a.groups[it.group];
        const int G = g.G, Kp = g.Kp;
        const int beg = a.indptr[it.row], end = a.indptr[it.row + 1];

        // 1) compact the row's entries in the gene subset into (value key, position) sort keys;
        //    several chunks of 32 entries per step, their loads issued before any is used
        int k = 0, bad = 0;
        if (a.map_bits) {
            // compact map in shared memory: index and value loads are independent, one memory
            // latency per step of GATHER_CHUNKS chunks
            for (int base = beg; base < end; base += 32 * GATHER_CHUNKS) {
                int c[GATHER_CHUNKS];
                float v[GATHER_CHUNKS];
#pragma unroll
                for (int t = 0; t < GATHER_CHUNKS; ++t) {
                    const int i = base + 32 * t + lane;
                    c[t] = i < end ? __ldcs(a.indices + i) : -1;
                    v[t] = i < end ? __ldcs(a.data + i) : 0.f;
                }
#pragma unroll
                for (int t = 0; t < GATHER_CHUNKS; ++t) {
                    const int i = base + 32 * t + lane;
                    bad |= (i < end && (unsigned)c[t] >= a.n_cols) ? 1 : 0;
                    int pos = -1;
                    if ((unsigned)c[t] < a.n_cols) {
                        const uint32_t wv = sbits[c[t] >> 5], bit = 1u << (c[t] & 31);
                        if (wv & bit) pos = (int)spre[c[t] >> 5] + __popc(wv & (bit - 1u));
                    }
                    const bool hit = pos >= 0;
                    if (hit && v[t] != v[t]) bad |= 2;
                    const unsigned m = __ballot_sync(FULL, hit);
                    if (hit) {
                        const int idx = k + __popc(m & ((1u << lane) - 1u));
                        if (idx < a.cap) keys[idx] = ((uint64_t)ord_key(canon_zero(v[t])) << 32) | (uint32_t)pos;
                    }
                    k += __popc(m);
                }
            }
        } else {
            for (int base = beg; base < end; base += 128) {
                int c[4], pos[4];
                float v[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int i = base + 32 * t + lane;
                    c[t] = i < end ? __ldg(a.indices + i) : -1;
                    bad |= (i < end && (unsigned)c[t] >= a.n_cols) ? 1 : 0;
                }
#pragma unroll
                for (int t = 0; t < 4; ++t) pos[t] = (unsigned)c[t] < a.n_cols ? __ldg(g.colmap + c[t]) : -1;
#pragma unroll
                for (int t = 0; t < 4; ++t) v[t] = pos[t] >= 0 ? __ldg(a.data + base + 32 * t + lane) : 0.f;
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const bool hit = pos[t] >= 0;
                    if (hit && v[t] != v[t]) bad |= 2;
                    const unsigned m = __ballot_sync(FULL, hit);
                    if (hit) {
                        const int idx = k + __popc(m & ((1u << lane) - 1u));
                        if (idx < a.cap) keys[idx] = ((uint64_t)ord_key(canon_zero(v[t])) << 32) | (uint32_t)pos[t];
                    }
                    k += __popc(m);
                }
            }
        }
        bad = __reduce_or_sync(FULL, bad);
        if (bad && lane == 0) atomicOr(a.status, bad);
        __syncwarp();
        const bool fits = k <= a.cap;
        if (!fits && a.overflow) {  // ranked by the second, large-buffer launch
            if (lane == 0) a.overflow[atomicAdd(a.n_overflow, 1)] = it;
            continue;
        }
        // bucket counting instead of a sort: 256 buckets over a linear map of [min, max] of the
        // entries' value keys (monotone, so equal values share a bucket); every entry of a lower
        // bucket is smaller, and the rest of #less / #equal is counted inside the entry's bucket
        float fmin = 0.f, scale = 0.f;
        if (fits && k > 0) {
            uint32_t kmin = 0xffffffffu, kmax = 0u;
            for (int j = lane; j < k; j += 32) {
                const uint32_t u = (uint32_t)(keys[j] >> 32);
                kmin = min(kmin, u);
                kmax = max(kmax, u);
            }
            kmin = __reduce_min_sync(FULL, kmin);
            kmax = __reduce_max_sync(FULL, kmax);
            fmin = key_float(kmin);
            const float span = key_float(kmax) - fmin;
            scale = (span > 0.f && span < 1e30f) ? 256.0f / span : 0.f;
            for (int b = lane; b < 256; b += 32) hist[b] = 0;
            __syncwarp();
            for (int j = lane; j < k; j += 32) atomicAdd(&hist[rank_bucket(keys[j], fmin, scale)], 1);
            __syncwarp();
            int c[8], sum = 0;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                c[t] = hist[8 * lane + t];
                sum += c[t];
            }
            int acc = warp_incl_scan(sum, lane) - sum;
#pragma unroll
            for (int t = 0; t < 8; ++t) {  // each lane rewrites only the counts it read
                hist[8 * lane + t] = acc;
                acc += c[t];
            }
            __syncwarp();
            for (int j = lane; j < k; j += 32) {
                const uint64_t key = keys[j];
                vals[atomicAdd(&hist[rank_bucket(key, fmin, scale)], 1)] = (uint32_t)(key >> 32);
            }
            __syncwarp();  // hist[b] is now the end of bucket b, and bucket b starts where b - 1 ends
        }

        // 2) every position of the subset starts as an implicit zero: rank (G-k+1)/2, d = -k;
        //    the padding [G, Kp) is 0 so that it adds nothing to a dot product.  Written straight
        //    into the output row (coalesced words); the stored entries are written over it below.
        const int row_bytes = a.out_mode == RANK_LIMBS ? 3 * Kp : 2 * Kp;
        unsigned char* stage = reinterpret_cast<unsigned char*>(g.out) + (size_t)it.slot * row_bytes;
        const int d0 = -k;
        if (a.out_mode == RANK_LIMBS) {
            int h0, l0, s0;
            split_limbs(d0, g.limb_w, h0, l0, s0);
            uint32_t* st = reinterpret_cast<uint32_t*>(stage);
            const int wpp = Kp / 4;  // words per plane (Kp is a multiple of 16)
#pragma unroll
            for (int plane = 0; plane < 3; ++plane) {
                const uint32_t full = (uint32_t)(uint8_t)(int8_t)(plane == 0 ? h0 : plane == 1 ? l0 : s0) * 0x01010101u;
                for (int w = lane; w < wpp; w += 32) {
                    const int left = G - 4 * w;  // subset positions in this word
                    st[plane * wpp + w] = left >= 4 ? full : left <= 0 ? 0u : full & ((1u << (8 * left)) - 1u);
                }
            }
        } else if (a.out_mode == RANK_F16) {
            __half* st = reinterpret_cast<__half*>(stage);
            const __half h0 = __int2half_rn(d0), z = __int2half_rn(0);
            for (int p = lane; p < Kp; p += 32) st[p] = p < G ? h0 : z;
        } else {
            int16_t* st = reinterpret_cast<int16_t*>(stage);
            for (int p = lane; p < Kp; p += 32) st[p] = p < G ? (int16_t)d0 : (int16_t)0;
        }
        __syncwarp();

        // the zeros are in place before any lane writes a stored entry over them (__syncwarp above)
        // 3) stored entries: d = 2 * (G - k + #less + (#equal + 1)/2) - (G + 1)
        int64_t sq = 0;
        if (fits) {
            for (int j = lane; j < k; j += 32) {
                const uint64_t key = keys[j];
                const uint32_t hv = (uint32_t)(key >> 32);
                const int b = rank_bucket(key, fmin, scale);
                const int e = hist[b], st = b > 0 ? hist[b - 1] : 0;
                int less = st, eq = 0;  // entries of lower buckets, then this bucket's
                for (int t = st; t < e; ++t) {
                    const uint32_t u = vals[t];
                    less += u < hv;
                    eq += u == hv;
                }
                const int d = G - 2 * k + 2 * less + eq;
                stage_put(stage, a.out_mode, Kp, (int)(uint32_t)key, d, g.limb_w);
                sq += (int64_t)d * d;
            }
        } else {
            // more entries than the sort buffer holds: count directly over the row
            for (int i = beg + lane; i < end; i += 32) {
                const int c = a.indices[i];
                if ((unsigned)c >= a.n_cols) continue;
                const int pos = g.colmap[c];
                if (pos < 0) continue;
                const float v = canon_zero(a.data[i]);
                int less = 0, eq = 0;
                for (int j = beg; j < end; ++j) {
                    const int c2 = a.indices[j];
                    if ((unsigned)c2 >= a.n_cols || g.colmap[c2] < 0) continue;
                    const float w = canon_zero(a.data[j]);
                    less += w < v;
                    eq += w == v;
                }
                const int d = G - 2 * k + 2 * less + eq;
                stage_put(stage, a.out_mode, Kp, pos, d, g.limb_w);
                sq += (int64_t)d * d;
            }
        }
        sq = warp_sum_i64(sq);
        __syncwarp();
        const int64_t n2 = sq + (int64_t)(G - k) * k * k;
        if (lane == 0) {
            g.n2[it.slot] = n2;
            g.rinv[it.slot] = n2 > 0 ? 1.0 / sqrt((double)n2) : __longlong_as_double(0x7ff8000000000000ll);
        }

        // 4) FP32 self-norm in the reference's order (fp32ref mode only)
        if (a.norm_mode == NORM_SEQ) {
            if (lane == 0) {
                float acc = 0.f;
                for (int p = 0; p < G; ++p) {
                    const float x = stage_d(stage, a.out_mode, Kp, p, g.limb_w) * 0.5f;
                    acc = fmaf(x, x, acc);
                }
                g.f32norm[it.slot] = acc;
            }
        } else if (a.norm_mode == NORM_TREE128) {
            const int step = (G + 127) / 128;
            float c[4];
            for (int t = 0; t < 4; ++t) {
                const int ch = 4 * lane + t;
                float acc = 0.f;
                for (int p = ch * step; p < (ch + 1) * step && p < G; ++p) {
                    const float x = stage_d(stage, a.out_mode, Kp, p, g.limb_w) * 0.5f;
                    acc = fmaf(x, x, acc);
                }
                c[t] = acc;
            }
            float v = __fadd_rn(__fadd_rn(c[0], c[1]), __fadd_rn(c[2], c[3]));
            for (int o = 1; o < 32; o <<= 1) {
                const float w = __shfl_down_sync(FULL, v, o);
                if ((lane & (2 * o - 1)) == 0) v = __fadd_rn(v, w);
            }
            if (lane == 0) g.f32norm[it.slot] = v;
        }

        __syncwarp();
    }
}

// ---- CSR compaction --------------------------------------------------------------------------

// row_mask (optional): rows with mask 0 are left empty.
__global__ void filter_count_kernel(const int32_t* indptr, const int32_t* indices, uint32_t n_rows, uint32_t n_cols,
                                    const int32_t* map, int32_t* counts, const uint8_t* row_mask, int* row_max) {
    const int lane = threadIdx.x & 31;
    int mx = 0;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n_rows;
         row += (gridDim.x * blockDim.x) >> 5) {
        if (row_mask && !row_mask[row]) {
            if (lane == 0) counts[row] = 0;
            continue;
        }
        int cnt = 0;
        for (int i = indptr[row] + lane; i < indptr[row + 1]; i += 32) {
            const int c = indices[i];
            cnt += ((unsigned)c < n_cols && map[c] >= 0);
        }
        cnt = __reduce_add_sync(FULL, cnt);
        if (lane == 0) counts[row] = cnt;
        mx = max(mx, cnt);
    }
    if (row_max && lane == 0 && mx > 0) atomicMax(row_max, mx);
}

__global__ void filter_fill_kernel(const float* data, const int32_t* indptr, const int32_t* indices, uint32_t n_rows,
                                   uint32_t n_cols, const int32_t* map, const int32_t* out_ptr, float* out_data,
                                   int32_t* out_indices, const uint8_t* row_mask) {
    const int lane = threadIdx.x & 31;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n_rows;
         row += (gridDim.x * blockDim.x) >> 5) {
        if (row_mask && !row_mask[row]) continue;
        int base = out_ptr[row];
        const int beg = indptr[row], end = indptr[row + 1];
        for (int i0 = beg; i0 < end; i0 += 32) {
            const int i = i0 + lane;
            int nc = -1;
            if (i < end) {
                const int c = indices[i];
                if ((unsigned)c < n_cols) nc = map[c];
            }
            const unsigned m = __ballot_sync(FULL, nc >= 0);
            if (nc >= 0) {
                const int o = base + __popc(m & ((1u << lane) - 1u));
                out_data[o] = data[i];
                out_indices[o] = nc;
            }
            base += __popc(m);
        }
    }
}

// Exclusive scan of n values into out[0..n] (out[n] = total) by one block of 1024 threads.
__global__ void __launch_bounds__(1024) scan_kernel(const int32_t* in, int32_t* out, uint32_t n) {
    __shared__ int32_t warp_tot[32];
    __shared__ int32_t carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const int32_t v = i < n ? in[i] : 0;
        int32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(FULL, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int32_t t = warp_tot[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t y = __shfl_up_sync(FULL, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;
        }
        __syncthreads();
        const int32_t excl = carry + (warp ? warp_tot[warp - 1] : 0) + x - v;
        if (i < n) out[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

// ---- score-step correlation on CUDA cores -----------------------------------------------------
//
// 128 x 128 output tile per block, 8 x 8 per thread, genes in ascending order (BK = 8), so each
// output is one fused multiply-add chain over genes 0..G-1 exactly as the reference's spearman
// kernel accumulates it.  Padding genes hold d = 0 and leave the chain unchanged.
template <bool FP32>
__global__ void __launch_bounds__(256) corr_simt_kernel(const int8_t* A, const int8_t* B, int nq, int R, int G,
                                                        int Kp, const float* fa, const float* fb, const double* ra,
                                                        const double* rb, const int64_t* na, const int64_t* nb,
                                                        float* out, int64_t ld, int m) {
    using T = typename std::conditional<FP32, float, double>::type;
    __shared__ T As[8][132];
    __shared__ T Bs[8][132];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * 128, n0 = blockIdx.x * 128;
    const int lr = threadIdx.x >> 1, lk = (threadIdx.x & 1) * 4;
    T acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = T(0);
    const int Kend = (G + 7) & ~7;
    for (int k0 = 0; k0 < Kend; k0 += 8) {
        {
            const int q = m0 + lr;
            uint32_t h4 = 0, l4 = 0;
            if (q < nq) {
                const int8_t* row = A + (size_t)q * 3 * Kp;
                h4 = *reinterpret_cast<const uint32_t*>(row + k0 + lk);
                l4 = *reinterpret_cast<const uint32_t*>(row + 2 * Kp + k0 + lk);  // the S plane
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int d = m * (int)(int8_t)(h4 >> (8 * b)) + (int)(int8_t)(l4 >> (8 * b));
                As[lk + b][lr] = FP32 ? T(d * 0.5f) : T(d);
            }
        }
        {
            const int r = n0 + lr;
            uint32_t h4 = 0, l4 = 0;
            if (r < R) {
                const int8_t* row = B + (size_t)r * 3 * Kp;
                h4 = *reinterpret_cast<const uint32_t*>(row + k0 + lk);
                l4 = *reinterpret_cast<const uint32_t*>(row + 2 * Kp + k0 + lk);  // the S plane
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int d = m * (int)(int8_t)(h4 >> (8 * b)) + (int)(int8_t)(l4 >> (8 * b));
                Bs[lk + b][lr] = FP32 ? T(d * 0.5f) : T(d);
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            T av[8], bv[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) av[i] = As[kk][ty * 8 + i];
#pragma unroll
            for (int j = 0; j < 8; ++j) bv[j] = Bs[kk][tx * 8 + j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int q = m0 + ty * 8 + i;
        if (q >= nq) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int r = n0 + tx * 8 + j;
            if (r >= R) continue;
            float s;
            if (FP32) {
                const float div = sqrtf(fa[q] * fb[r]);
                s = div != 0.f ? (float)acc[i][j] / div : __int_as_float(0x7fffffff);
            } else {
                s = (na[q] == 0 || nb[r] == 0) ? __int_as_float(0x7fffffff)
                                               : (float)(((double)acc[i][j] * ra[q]) * rb[r]);
            }
            out[(size_t)q * ld + r] = s;
        }
    }
}

// ---- per-label quantile ------------------------------------------------------------------------

// STAGE: the block first copies the query's score row (row_len floats) into shared memory with
// 16-byte loads, and warps take labels from `lorder` (longest first) through a shared counter; every
// selection pass then reads shared memory instead of global memory.
template <bool STAGE, int NW = STAGE ? 16 : 8>
__global__ void __launch_bounds__(NW * 32) select_first_kernel(const float* scores, int64_t ld, int nq, int L,
                                                           const LabelQ* lq, float p, float thre, const int64_t* qn2,
                                                           float* label_scores, int32_t* first, uint8_t* flags,
                                                           float* scratch, int64_t spw, int* status, int row_len,
                                                           const int32_t* lorder, const uint32_t* ext_min,
                                                           const uint32_t* ext_max) {
    extern __shared__ __align__(16) float srow[];
    __shared__ float ls[256];
    __shared__ int hist[NW][256];
    __shared__ int s_mx, s_next;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* my_scratch = scratch ? scratch + (size_t)(blockIdx.x * NW + warp) * spw : nullptr;
    const bool vec = STAGE && (ld % 4) == 0 && (reinterpret_cast<uintptr_t>(scores) & 15) == 0;
    for (int q = blockIdx.x; q < nq; q += gridDim.x) {
        const float* row = scores + (size_t)q * ld;
        const bool qnan = qn2[q] == 0;
        if (STAGE) {
            if (!qnan) {
                if (vec) {
                    const float4* src = reinterpret_cast<const float4*>(row);
                    float4* dst = reinterpret_cast<float4*>(srow);
                    for (int i = threadIdx.x; i < row_len / 4; i += NW * 32) dst[i] = __ldcs(src + i);
                    for (int i = (row_len & ~3) + threadIdx.x; i < row_len; i += NW * 32) srow[i] = __ldcs(row + i);
                } else {
                    for (int i = threadIdx.x; i < row_len; i += NW * 32) srow[i] = __ldcs(row + i);
                }
            }
            // the block's next row is brought into L2 while this one is selected, so that its staging
            // loads hit L2 (16-byte aligned rows, ld % 4 == 0: the rounded-up size stays in the row)
            if (vec && threadIdx.x == 0 && q + (int)gridDim.x < nq && qn2[q + gridDim.x] != 0) {
                const float* nxt = scores + (size_t)(q + gridDim.x) * ld;
                const uint32_t bytes = (uint32_t)(row_len * 4 + 15) & ~15u;
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(nxt), "r"(bytes) : "memory");
            }
            if (threadIdx.x == 0) s_next = 0;
            __syncthreads();
            row = srow;
            for (;;) {
                int i = 0;
                if (lane == 0) i = atomicAdd(&s_next, 1);
                i = __shfl_sync(FULL, i, 0);
                if (i >= L) break;
                const int l = lorder[i];
                const LabelQ d = lq[l];
                float r;
                if (qnan) r = __int_as_float(0x7fffffff);
                else if (ext_min && !d.has_nan && d.kind != 0)  // extremes from the correlation epilogue
                    r = quantile_warp_core(row + d.start, d, p, hist[warp], my_scratch, lane, status,
                                           ext_min[(size_t)q * L + l], ext_max[(size_t)q * L + l], false);
                else r = quantile_warp(row + d.start, d, p, hist[warp], my_scratch, lane, status);
                if (lane == 0) ls[l] = r;
            }
        } else {
            for (int l = warp; l < L; l += NW) {
                const LabelQ d = lq[l];
                float r;
                if (qnan) r = __int_as_float(0x7fffffff);
                else r = quantile_warp(row + d.start, d, p, hist[warp], my_scratch, lane, status);
                if (lane == 0) ls[l] = r;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int mn, mx;
            stl::minmax(ls, L, &mn, &mx);
            s_mx = mx;
            first[q] = mx;
        }
        __syncthreads();
        const float t = __fsub_rn(ls[s_mx], thre);
        for (int l = threadIdx.x; l < L; l += blockDim.x) {
            label_scores[(size_t)q * L + l] = ls[l];
            if (flags) flags[(size_t)q * L + l] = ls[l] >= t ? 1 : 0;
        }
        __syncthreads();
    }
}

// Warp-per-row form: each warp selects every label of its query rows straight from the score rows
// (global memory; a label's second pass hits L1 / L2), so no block barrier waits for a row's longest
// label, and a CTA needs only a histogram per warp (up to 64 warps per SM).  Every row has the same
// labels, so the warps' work is balanced by construction.  Each warp prefetches into L2 the list of the
// label two ahead in its row.
// MINB: CTAs per SM the register allocation is sized for (2: 64 registers and 32 warps per SM,
// 3: 40 registers and 48 warps per SM).
template <int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) select_rows_kernel(const float* scores, int64_t ld, int nq, int L,
                                                           const LabelQ* lq, float p, float thre,
                                                           const int64_t* qn2, float* label_scores, int32_t* first,
                                                           uint8_t* flags, float* scratch, int64_t spw, int* status,
                                                           int row_len, const int32_t* lorder,
                                                           const uint32_t* ext_min, const uint32_t* ext_max) {
    __shared__ int hist[NW][256];
    __shared__ float ls_all[NW][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * NW + warp, n_warps = gridDim.x * NW;
    float* my_scratch = scratch ? scratch + (size_t)gw * spw : nullptr;
    float* ls = ls_all[warp];
    // rows start on 16 bytes when ld is a multiple of 4, so a label's list widened to 16-byte bounds
    // stays inside its row
    const bool pf = (ld % 4) == 0 && (reinterpret_cast<uintptr_t>(scores) & 15) == 0;
    for (int q = gw; q < nq; q += n_warps) {
        const float* row = scores + (size_t)q * ld;
        const bool qnan = qn2[q] == 0;
        // L2 prefetch of the list of the label two ahead (a whole row fetched a row ahead is evicted
        // before use: every warp of the GPU streams its own rows meanwhile)
        auto prefetch_label = [&](int idx) {
            if (pf && !qnan && lane == 0 && idx < L) {
                const LabelQ dn = lq[lorder[idx]];
                const uintptr_t a0 = reinterpret_cast<uintptr_t>(row + dn.start) & ~uintptr_t(15);
                const uintptr_t a1 = (reinterpret_cast<uintptr_t>(row + dn.start + dn.len) + 15) & ~uintptr_t(15);
                if (a1 > a0)
                    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"((uint32_t)(a1 - a0))
                                 : "memory");
            }
        };
        prefetch_label(0);
        prefetch_label(1);
        for (int i = 0; i < L; ++i) {
            prefetch_label(i + 2);
            const int l = lorder[i];
            const LabelQ d = lq[l];
            float r;
            if (qnan) r = __int_as_float(0x7fffffff);
            else if (ext_min && !d.has_nan && d.kind != 0)  // extremes from the correlation epilogue
                r = quantile_warp_core(row + d.start, d, p, hist[warp], my_scratch, lane, status,
                                       ext_min[(size_t)q * L + l], ext_max[(size_t)q * L + l], false);
            else r = quantile_warp(row + d.start, d, p, hist[warp], my_scratch, lane, status);
            if (lane == 0) ls[l] = r;
        }
        __syncwarp();
        int mn = 0, mx = 0;
        if (lane == 0) {
            stl::minmax(ls, L, &mn, &mx);
            first[q] = mx;
        }
        mx = __shfl_sync(FULL, mx, 0);
        const float t = __fsub_rn(ls[mx], thre);
        for (int l = lane; l < L; l += 32) {
            label_scores[(size_t)q * L + l] = ls[l];
            if (flags) flags[(size_t)q * L + l] = ls[l] >= t ? 1 : 0;
        }
        __syncwarp();
    }
}

// ---- fine-tune correlation and selection ------------------------------------------------------

template <bool FP32>
__global__ void __launch_bounds__(256) ft_corr_kernel(const FtGroup* groups, const FtCorrItem* items, uint32_t n_items,
                                                      const int16_t* qd, const int16_t* rd, const float* qf,
                                                      const float* rf, const double* qr, const double* rr,
                                                      const int64_t* qn, const int64_t* rn, float* scores) {
    const int lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    for (uint32_t w = blockIdx.x * wpb + (threadIdx.x >> 5); w < n_items; w += gridDim.x * wpb) {
        const FtCorrItem it = items[w];
        const FtGroup g = groups[it.group];
        const int G = g.G, Kp = g.Kp;
        const int step = (G + 127) / 128;
        const int64_t rrow = g.r_row + it.ref;
        const int16_t* y = rd + g.r_el + (int64_t)it.ref * Kp;
        for (uint32_t q = it.q_begin; q < it.q_end; ++q) {
            const int64_t qrow = g.q_row + q;
            const int16_t* x = qd + g.q_el + (int64_t)q * Kp;
            float s;
            if (FP32) {
                float c[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int ch = 4 * lane + t;
                    float acc = 0.f;
                    for (int i = ch * step; i < (ch + 1) * step && i < G; ++i)
                        acc = fmaf(x[i] * 0.5f, y[i] * 0.5f, acc);
                    c[t] = acc;
                }
                float v = __fadd_rn(__fadd_rn(c[0], c[1]), __fadd_rn(c[2], c[3]));
                for (int o = 1; o < 32; o <<= 1) {
                    const float u = __shfl_down_sync(FULL, v, o);
                    if ((lane & (2 * o - 1)) == 0) v = __fadd_rn(v, u);
                }
                const float div = sqrtf(qf[qrow] * rf[rrow]);
                s = div != 0.f ? v / div : __int_as_float(0x7fffffff);
            } else {
                int64_t acc = 0;
                for (int i = lane; i < G; i += 32) acc += (int32_t)x[i] * (int32_t)y[i];
                acc = warp_sum_i64(acc);
                s = (qn[qrow] == 0 || rn[rrow] == 0) ? __int_as_float(0x7fffffff)
                                                     : (float)(((double)acc * qr[qrow]) * rr[rrow]);
            }
            if (lane == 0) scores[g.s_off + (int64_t)q * g.n_ref + it.ref] = s;
        }
    }
}

__global__ void __launch_bounds__(256) ft_select_kernel(const FtGroup* groups, const FtSelItem* items, uint32_t n_items,
                                                        const LabelQ* lq, float p, const float* scores,
                                                        float* label_scores, float* scratch, int64_t spw,
                                                        int* status) {
    __shared__ int hist[8][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* my_scratch = scratch ? scratch + (size_t)(blockIdx.x * 8 + warp) * spw : nullptr;
    for (uint32_t w = blockIdx.x * 8 + warp; w < n_items; w += gridDim.x * 8) {
        const FtSelItem it = items[w];
        const FtGroup g = groups[it.group];
        const float* row = scores + g.s_off + (int64_t)it.cell * g.n_ref;
        for (int j = 0; j < g.n_labels; ++j) {
            const LabelQ d = lq[g.lq_off + j];
            const float r = quantile_warp(row + d.start, d, p, hist[warp], my_scratch, lane, status);
            if (lane == 0) label_scores[g.out_off + (int64_t)it.cell * g.n_labels + j] = r;
        }
    }
}

std::atomic<uint64_t> g_launches{0};

}  // namespace

uint64_t launch_count() { return g_launches.load(); }
void count_launch(uint64_t n) { g_launches += n; }

int device_sm_count() {
    // cached per device: launch shapes use the SM count of whichever device is current
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cached[kMaxDevices];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDevices) dev = 0;
    int n = cached[dev].load(std::memory_order_relaxed);
    if (n <= 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
            cudaGetLastError();
            n = 148;
        }
        cached[dev].store(n, std::memory_order_relaxed);  // every thread stores the same value
    }
    return n;
}

namespace {
int sm_count() { return device_sm_count(); }
}  // namespace

namespace {
void launch_rank_tier(const RankLaunch& a, long max_blocks, cudaStream_t s) {
    const int warp_bytes = ((a.cap * 12 + 256 * 4) + 15) & ~15;
    const int map_bytes = a.map_bits ? (int)(((a.n_cols + 31) / 32 * 6 + 15) & ~15u) : 0;
    // warps per CTA: the most resident warps per SM, then the widest CTA
    int wpb = 0, best = 0;
    for (int w = 8; w >= 1; --w) {
        const int sm_bytes = map_bytes + w * warp_bytes;
        if (sm_bytes > 200 * 1024) continue;
        const int resident = w * std::min(8, (228 * 1024) / (sm_bytes + 1024));
        if (resident > best) {
            best = resident;
            wpb = w;
        }
    }
    if (wpb < 1) fail(SGR_ERR_UNSUPPORTED, "gene subset too wide for the rank kernel's shared memory");
    const int smem = map_bytes + wpb * warp_bytes;
    SGR_CUDA(cudaFuncSetAttribute(rank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int per_sm = std::max(1, std::min(8, (228 * 1024) / (smem + 1024)));
    long blocks = (long)sm_count() * per_sm;
    if (max_blocks > 0) blocks = std::min(blocks * 4, (max_blocks + wpb - 1) / wpb);
    rank_kernel<<<(unsigned)std::max(1L, blocks), 32 * wpb, smem, s>>>(a, warp_bytes);
    SGR_LAUNCH_CHECK();
    count_launch();
}
}  // namespace

void column_bits(const int32_t* colmap, uint32_t n_cols, uint32_t* bits, uint16_t* prefix) {
    const uint32_t n_words = (n_cols + 31) / 32;
    uint32_t count = 0;
    for (uint32_t w = 0; w < n_words; ++w) {
        if (count > 0xffffu) fail(SGR_ERR_UNSUPPORTED, "column subset above 65535 positions");
        prefix[w] = (uint16_t)count;
        uint32_t b = 0;
        for (uint32_t i = 0; i < 32 && 32 * w + i < n_cols; ++i)
            if (colmap[32 * w + i] >= 0) {
                if ((uint32_t)colmap[32 * w + i] != count) fail(SGR_ERR_INVALID_ARGUMENT, "column map not increasing");
                b |= 1u << i;
                ++count;
            }
        bits[w] = b;
    }
}

void launch_rank(const RankLaunch& a, cudaStream_t s) {
    if (a.n_items == 0) return;
    constexpr int kSmallCap = 384;  // 3 CTAs of 8 warps per SM with a 1,152-column stage
    if (!a.overflow || a.cap <= kSmallCap) {
        RankLaunch b = a;
        b.overflow = nullptr;
        launch_rank_tier(b, a.n_items, s);
        return;
    }
    SGR_CUDA(cudaMemsetAsync(a.n_overflow, 0, sizeof(int), s));
    RankLaunch small = a;
    small.cap = kSmallCap;
    launch_rank_tier(small, a.n_items, s);
    RankLaunch big = a;
    big.items = a.overflow;
    big.n_items_dev = a.n_overflow;
    big.overflow = nullptr;
    launch_rank_tier(big, 0, s);  // grid sized to the device: the row count is on the device
}

void launch_filter_count(const int32_t* indptr, const int32_t* indices, uint32_t n_rows, uint32_t n_cols,
                         const int32_t* map, int32_t* counts, cudaStream_t s, const uint8_t* row_mask,
                         int* row_max) {
    if (!n_rows) return;
    const unsigned blocks = std::min<unsigned>((n_rows + 7) / 8, sm_count() * 16);
    filter_count_kernel<<<blocks, 256, 0, s>>>(indptr, indices, n_rows, n_cols, map, counts, row_mask, row_max);
    SGR_LAUNCH_CHECK();
    count_launch();
}

namespace {
__global__ void mark_rows_kernel(const int32_t* list, int n, uint8_t* mask) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) mask[list[i]] = 1;
}
}  // namespace

namespace {
__global__ void sum_listed_kernel(const int32_t* list, const int* n, const int32_t* vals, unsigned long long* out) {
    unsigned long long t = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < *n; i += gridDim.x * blockDim.x) t += (unsigned)vals[list[i]];
    t = __reduce_add_sync(0xffffffffu, (unsigned)t);
    if ((threadIdx.x & 31) == 0 && t) atomicAdd(out, t);
}
}  // namespace

void launch_sum_listed(const int32_t* list, const int* n, const int32_t* vals, unsigned long long* out,
                       cudaStream_t s) {
    sum_listed_kernel<<<sm_count(), 256, 0, s>>>(list, n, vals, out);
    SGR_LAUNCH_CHECK();
    count_launch();
}

void launch_mark_rows(const int32_t* list, int n, uint8_t* mask, cudaStream_t s) {
    if (n <= 0) return;
    mark_rows_kernel<<<std::min((n + 255) / 256, sm_count() * 4), 256, 0, s>>>(list, n, mask);
    SGR_LAUNCH_CHECK();
    count_launch();
}

namespace {
constexpr uint32_t kScanTile = 4096;  // values per block of the tiled scan: 1024 threads x 4

// Sum of each 4096-value tile.
__global__ void __launch_bounds__(1024) tile_sum_kernel(const int32_t* in, uint32_t n, int32_t* part) {
    __shared__ int32_t ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * 4;
    int32_t v = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) v += base + j < n ? in[base + j] : 0;
    v = __reduce_add_sync(FULL, v);
    if (lane == 0) ws[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int32_t t = __reduce_add_sync(FULL, ws[lane]);
        if (lane == 0) part[blockIdx.x] = t;
    }
}

// Exclusive scan of each tile (4 consecutive values per thread) plus the tile's offset part_ex[b];
// block 0 also writes the total out[n] = part_ex[nb].
__global__ void __launch_bounds__(1024) tile_scan_kernel(const int32_t* in, int32_t* out, uint32_t n,
                                                         const int32_t* part_ex, uint32_t nb) {
    __shared__ int32_t ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * 4;
    int32_t v[4], sum = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        v[j] = base + j < n ? in[base + j] : 0;
        sum += v[j];
    }
    const int32_t x = warp_incl_scan(sum, lane);
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) ws[lane] = warp_incl_scan(ws[lane], lane);
    __syncthreads();
    int32_t e = part_ex[blockIdx.x] + (warp ? ws[warp - 1] : 0) + x - sum;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (base + j < n) out[base + j] = e;
        e += v[j];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = part_ex[nb];
}
}  // namespace

void launch_exclusive_scan(const int32_t* in, int32_t* out, uint32_t n, int32_t* scratch, cudaStream_t s) {
    const uint32_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb <= 2 || scratch == nullptr) {  // one block walks the values
        scan_kernel<<<1, 1024, 0, s>>>(in, out, n);
        SGR_LAUNCH_CHECK();
        count_launch();
        return;
    }
    // tile sums, their scan (one block), then each tile's scan from its offset
    int32_t* part = scratch;
    int32_t* part_ex = scratch + nb;
    tile_sum_kernel<<<nb, 1024, 0, s>>>(in, n, part);
    SGR_LAUNCH_CHECK();
    scan_kernel<<<1, 1024, 0, s>>>(part, part_ex, nb);
    SGR_LAUNCH_CHECK();
    tile_scan_kernel<<<nb, 1024, 0, s>>>(in, out, n, part_ex, nb);
    SGR_LAUNCH_CHECK();
    count_launch(3);
}

void launch_filter_fill(const float* data, const int32_t* indptr, const int32_t* indices, uint32_t n_rows,
                        uint32_t n_cols, const int32_t* map, const int32_t* out_ptr, float* out_data,
                        int32_t* out_indices, cudaStream_t s, const uint8_t* row_mask) {
    if (!n_rows) return;
    const unsigned blocks = std::min<unsigned>((n_rows + 7) / 8, sm_count() * 16);
    filter_fill_kernel<<<blocks, 256, 0, s>>>(data, indptr, indices, n_rows, n_cols, map, out_ptr, out_data,
                                              out_indices, row_mask);
    SGR_LAUNCH_CHECK();
    count_launch();
}

void launch_corr_simt(bool fp32ref, const int8_t* A, const int8_t* B, int nq, int R, int G, int Kp, const float* fa,
                      const float* fb, const double* ra, const double* rb, const int64_t* na, const int64_t* nb,
                      float* scores, int64_t ld, int limb_w, cudaStream_t s) {
    if (nq <= 0 || R <= 0) return;
    dim3 grid((R + 127) / 128, (nq + 127) / 128);
    const int m = limb_mult(limb_w);
    if (fp32ref)
        corr_simt_kernel<true><<<grid, 256, 0, s>>>(A, B, nq, R, G, Kp, fa, fb, ra, rb, na, nb, scores, ld, m);
    else
        corr_simt_kernel<false><<<grid, 256, 0, s>>>(A, B, nq, R, G, Kp, fa, fb, ra, rb, na, nb, scores, ld, m);
    SGR_LAUNCH_CHECK();
    count_launch();
}

LabelQ make_lq(int start, int len, float p) {
    LabelQ q{};
    q.start = start;
    q.len = len;
    if (len <= 1) {
        q.kind = 0;
        return q;
    }
    const float step = 1.0 / (len - 1);
    q.step = step;
    const float first = 0 * step, last = (len - 1) * step;
    if (p <= first) {
        q.kind = 1;
        return q;
    }
    if (last <= p) {
        q.kind = 2;
        return q;
    }
    int lo = 0, hi = len;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (mid * step < p) lo = mid + 1;
        else hi = mid;
    }
    q.kind = 3;
    q.k = lo;
    q.prev_index = (lo - 1) * step;
    return q;
}

void launch_select_first(const float* scores, int64_t ld, int nq, int L, const LabelQ* lq, float p, float thre,
                         const int64_t* qn2, float* label_scores, int32_t* first, uint8_t* flags, float* scratch,
                         int64_t spw, int* status, int row_len, const int32_t* lorder, cudaStream_t s,
                         const uint32_t* ext_min, const uint32_t* ext_max, int warps) {
    if (nq <= 0) return;
    const size_t stage_bytes = (((size_t)std::max(row_len, 1) * 4 + 15) & ~size_t(15));
    if (lorder && (warps == 0 || warps == 1)) {  // one warp per row, 16 warps per CTA
        auto kern = warps == 1 ? select_rows_kernel<16, 3> : select_rows_kernel<16, 2>;
        int per_sm = 0;
        SGR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 512, 0));
        per_sm = std::max(1, std::min(per_sm, 4));  // scratch is sized for 64 warps per SM
        const unsigned blocks = (unsigned)std::min<long>((nq + 15) / 16, (long)sm_count() * per_sm);
        kern<<<blocks, 512, 0, s>>>(scores, ld, nq, L, lq, p, thre, qn2, label_scores, first, flags, scratch, spw,
                                    status, row_len, lorder, ext_min, ext_max);
    } else if (lorder && stage_bytes <= 200 * 1024) {
        auto kern = warps == 8 ? select_first_kernel<true, 8> : select_first_kernel<true, 16>;
        const int threads = 32 * (warps == 8 ? 8 : 16);
        SGR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_bytes));
        int per_sm = 0;
        SGR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, stage_bytes));
        per_sm = std::max(1, std::min(per_sm, 2));  // at most 32 warps per SM use scratch
        const unsigned blocks = (unsigned)std::min<long>(nq, (long)sm_count() * per_sm);
        kern<<<blocks, threads, stage_bytes, s>>>(scores, ld, nq, L, lq, p, thre, qn2, label_scores, first, flags,
                                                  scratch, spw, status, row_len, lorder, ext_min, ext_max);
    } else {
        const unsigned blocks = scratch ? (unsigned)std::min<long>(nq, sm_count() * 2)
                                        : (unsigned)std::min<long>(nq, sm_count() * 8);
        select_first_kernel<false><<<blocks, 256, 0, s>>>(scores, ld, nq, L, lq, p, thre, qn2, label_scores, first,
                                                          flags, scratch, spw, status, row_len, lorder, nullptr,
                                                          nullptr);
    }
    SGR_LAUNCH_CHECK();
    count_launch();
}

void launch_ft_corr(bool fp32ref, const FtGroup* groups, const FtCorrItem* items, uint32_t n_items, const int16_t* qd,
                    const int16_t* rd, const float* qf, const float* rf, const double* qr, const double* rr,
                    const int64_t* qn, const int64_t* rn, float* scores, cudaStream_t s) {
    if (!n_items) return;
    const unsigned blocks = std::min<unsigned>((n_items + 7) / 8, sm_count() * 16);
    if (fp32ref)
        ft_corr_kernel<true><<<blocks, 256, 0, s>>>(groups, items, n_items, qd, rd, qf, rf, qr, rr, qn, rn, scores);
    else
        ft_corr_kernel<false><<<blocks, 256, 0, s>>>(groups, items, n_items, qd, rd, qf, rf, qr, rr, qn, rn, scores);
    SGR_LAUNCH_CHECK();
    count_launch();
}

void launch_ft_select(const FtGroup* groups, const FtSelItem* items, uint32_t n_items, const LabelQ* lq, float p,
                      const float* scores, float* label_scores, float* scratch, int64_t spw, int* status,
                      cudaStream_t s) {
    if (!n_items) return;
    const unsigned blocks = scratch ? (unsigned)std::min<long>((n_items + 7) / 8, sm_count() * 2)
                                    : (unsigned)std::min<long>((n_items + 7) / 8, sm_count() * 8);
    ft_select_kernel<<<blocks, 256, 0, s>>>(groups, items, n_items, lq, p, scores, label_scores, scratch, spw, status);
    SGR_LAUNCH_CHECK();
    count_launch();
}

}  // namespace sgr
