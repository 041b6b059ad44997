// Persistent fine-tune kernel (exact arithmetic) and the reference pre-sort it reads.
//
// Restates the reference's per-cell fine-tune loop (src/cusingler.cu:1138-1333 of
// STOmics/cusingler: finetune_round + cufinetune) as one persistent kernel.  Each CTA takes the
// next query cell from a device work queue and runs all of that cell's rounds on the device:
//   1. gene set S = union over ordered candidate pairs of the first min(len, gene_thre(n)) genes of
//      the pair's fine-tune list; fewer than 20 genes keeps the first candidate;
//   2. the query's ranks over S (its thre-pool entries, sorted in shared memory);
//   3. for every reference cell of every candidate label, the rank correlation over S;
//   4. per label the quantile of those correlations, then the reference's keep/drop rule.
//
// Step 3 never builds a dense rank row.  With d = 2*rank - (|S|+1) and e = d + k (k = stored
// entries of the row inside S), e is 0 at every implicit zero, so
//     sum_g d_q d_r = sum_{g stored in both} e_q e_r - |S| k_q k_r.
// Each reference row's thre-pool entries are sorted by value once (ref_presort_kernel), the last
// entry of each run of equal values flagged.  For any S, one pass over the row keeping the entries
// inside S yields every kept entry's rank: a run of b kept entries with a kept entries before it
// gives each of them 2 #less + #equal = z = 2a + b.  The pass accumulates per run
// X = sum z s, Y = sum s (s = the query's e summed over the run's genes) and T = sum (b^3 - b);
// the other two sums are closed forms of k_r, the kept count: Z1 = sum b z = k_r^2 (the z of a run
// average the odd numbers 2i + 1 it covers) and Z2 = sum b z^2 = ((4 k_r^3 - k_r) - T) / 3 (sum of
// (2i + 1)^2 minus each run's tie spread).  Then, exactly in int64,
//     N   = X + (|S| - k_r) Y - |S| k_q k_r
//     n_r = Z2 + 2 c Z1 + k_r c^2 + (|S| - k_r) k_r^2,   c = |S| - 2 k_r.
// Layout: the rows of each label form blocks of 32 consecutive rows; a block stores entry j of its
// t-th row at block start + (j / 4) * 128 + t * 4 + j % 4 and is as long as its longest row (rounded
// up to 4), shorter rows padded with entries of gene id Wt, whose e-value is SENT.  One warp scores
// the 32 rows of a block, one lane each, so a warp's 16-byte load of entry vector j / 4 covers 512
// contiguous bytes.
// The score is float((N * (1/sqrt(n_q))) * (1/sqrt(n_r))) in FP64, the same
// formula as the score step's exact mode.

#include <algorithm>
#include <cstdint>

#include "kernels.cuh"
#include "sgr_internal.h"
#include "stl_order.h"
#include "device_util.cuh"

namespace sgr {

namespace {

constexpr int SENT = INT32_MIN;  // "gene not in S"

// Packed e-value of row_score's packed path: (1 << shift) + e at genes of S, 0 elsewhere.
__device__ __forceinline__ int pack_e(int v, int shift) { return v >= 0 ? (int)((1u << shift) + (uint32_t)v) : 0; }

// One warp per reference row: its thre-pool entries sorted by (value, gene), each packed as
// gene | last << 31, where last marks the final entry of a run of equal values.  Entry j of row r is
// written at ell_base[r] + (j / 4) * 128 + j % 4; entries k .. ell_len[r] - 1 are pad_gene | 1 << 31.
__global__ void __launch_bounds__(256) ref_presort_kernel(const float* data, const int32_t* idx, const int32_t* ptr,
                                                          const int32_t* ell_base, const int32_t* ell_len,
                                                          uint32_t n_rows, int cap, uint32_t pad_gene, uint32_t* out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    uint64_t* keys = reinterpret_cast<uint64_t*>(smem) + (size_t)warp * cap;
    constexpr uint32_t LAST = 0x80000000u;
    for (uint32_t row = blockIdx.x * wpb + warp; row < n_rows; row += gridDim.x * wpb) {
        const int beg = ptr[row], k = ptr[row + 1] - beg;
        uint32_t* ob = out + ell_base[row];
        auto o = [ob](int j) -> uint32_t& { return ob[(j >> 2) * 128 + (j & 3)]; };
        for (int j = k + lane; j < ell_len[row]; j += 32) o(j) = pad_gene | LAST;
        if (k <= cap) {
            int n = 1;
            while (n < k) n <<= 1;
            for (int i = lane; i < n; i += 32)
                keys[i] = i < k ? ((uint64_t)ord_key(canon_zero(data[beg + i])) << 32) | (uint32_t)idx[beg + i]
                                : ~0ull;
            __syncwarp();
            if (k > 1) warp_bitonic(keys, n, lane);
            for (int j = lane; j < k; j += 32) {
                const uint64_t key = keys[j];
                const bool last = j + 1 == k || (uint32_t)(keys[j + 1] >> 32) != (uint32_t)(key >> 32);
                o(j) = (uint32_t)(key & 0xffffu) | (last ? LAST : 0u);
            }
            __syncwarp();
        } else {
            // rows longer than the sort buffer: position and run end by counting
            for (int i = lane; i < k; i += 32) {
                const float v = canon_zero(data[beg + i]);
                const int g = idx[beg + i];
                int pos = 0, eq_after = 0;
                for (int j = 0; j < k; ++j) {
                    const float w = canon_zero(data[beg + j]);
                    const int h = idx[beg + j];
                    pos += (w < v) || (w == v && h < g);
                    eq_after += w == v && h > g;
                }
                o(pos) = (uint32_t)g | (eq_after == 0 ? LAST : 0u);
            }
        }
    }
}

// Fine-tune workload of a cell: the reference rows of its first-round candidates (0 when it has at
// most one candidate and needs no round).
__global__ void ft_keys_kernel(int n, const int32_t* list, int L, const uint8_t* flags, const uint32_t* ctidx,
                               int64_t* keys, int32_t* ncand) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int q = list ? list[i] : i;
    const uint8_t* f = flags + (int64_t)q * L;
    int64_t w = 0;
    int c = 0;
    for (int l = 0; l < L; ++l)
        if (f[l]) {
            ++c;
            w += ctidx[2 * l + 1];
        }
    keys[i] = c >= 2 ? w : 0;
    ncand[i] = c;
}

struct FtShared {
    int cell, ntop, nS, kq, rounds, done;
    int64_t nq;
    double rq;
};

// Candidates of a cell: its flagged labels in ascending order (src/cusingler.cu:1305-1312).  Warp.
__device__ int warp_flagged_labels(const uint8_t* flags, int L, uint8_t* top, int lane) {
    int n = 0;
    for (int base = 0; base < L; base += 32) {
        const int l = base + lane;
        const bool f = l < L && flags[l] != 0;
        const unsigned m = __ballot_sync(FULL, f);
        if (f) top[n + __popc(m & ((1u << lane) - 1u))] = (uint8_t)l;
        n += __popc(m);
    }
    return n;
}

// Gene set S of a candidate list: union over ordered pairs of the first min(len, gene_thre(n))
// genes of the pair's fine-tune list (src/cusingler.cu:1141-1156), as bits over the thre pool.
// CTA-wide; returns |S| to every thread.
template <int NW>
__device__ int cta_gene_set(const FtPersistentArgs& a, const uint8_t* top, int ntop, uint32_t* bits, int* red) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwords = (a.Wt + 31) / 32;
    for (int w = tid; w < nwords; w += NW * 32) bits[w] = 0u;
    __syncthreads();
    const int gthre = a.gene_thre[ntop];
    const int np = ntop * ntop;
    if (np <= 4 * NW) {
        // few pairs: warps take pairs round robin, and with more warps than pairs each pair's list is
        // cut into interleaved segments, so that every warp has loads in flight
        const int segs = max(1, NW / np);
        for (int u = warp; u < np * segs; u += NW) {
            const int pr = u % np, seg = u / np;
            const int i = pr / ntop, j = pr % ntop;
            if (i == j) continue;
            const size_t pi = (size_t)top[i] * a.L + top[j];
            const uint32_t pos = a.ft_idx[2 * pi];
            const int len = min((int)a.ft_idx[2 * pi + 1], gthre);
#pragma unroll 4
            for (int e = seg * 32 + lane; e < len; e += 32 * segs) {
                const uint32_t g = __ldg(a.ft_genes + pos + e);
                atomicOr(&bits[g >> 5], 1u << (g & 31));
            }
        }
    }
    // many pairs: a warp takes ppw ordered pairs at a time (at most 32, and few enough that every warp
    // gets some): each lane fetches one pair's list, then the warp walks the lists together so that the
    // gene loads of several pairs are in flight at once
    const int ppw = min(32, (np + NW - 1) / NW);
    for (int base = warp * ppw; np > 4 * NW && base < np; base += NW * ppw) {
        const int pr = base + lane;
        uint32_t pos = 0;
        int len = 0;
        if (lane < ppw && pr < np) {
            const int i = pr / ntop, j = pr % ntop;
            if (i != j) {
                const size_t pi = (size_t)top[i] * a.L + top[j];
                pos = a.ft_idx[2 * pi];
                len = min((int)a.ft_idx[2 * pi + 1], gthre);
            }
        }
        const int maxn = __reduce_max_sync(FULL, len);
        for (int e0 = 0; e0 < maxn; e0 += 32) {
#pragma unroll 8
            for (int t = 0; t < ppw; ++t) {
                const uint32_t p = __shfl_sync(FULL, pos, t);
                const int n = __shfl_sync(FULL, len, t);
                const int e = e0 + lane;
                if (e < n) {
                    const uint32_t g = __ldg(a.ft_genes + p + e);
                    atomicOr(&bits[g >> 5], 1u << (g & 31));
                }
            }
        }
    }
    __syncthreads();
    int cnt = 0;
    for (int w = tid; w < nwords; w += NW * 32) cnt += __popc(bits[w]);
    cnt = __reduce_add_sync(FULL, cnt);
    if (lane == 0) red[warp] = cnt;
    __syncthreads();
    int t = 0;
    for (int w = 0; w < NW; ++w) t += red[w];
    __syncthreads();
    return t;
}

// The query's e-values over S: 0 at genes of S it does not store, |S| - k + 2 #less + #equal at
// stored ones, SENT outside S.  CTA-wide (the ranking itself by warp 0); sets *kq, *nq, *rq.
template <int NW>
__device__ void cta_query_ranks(const FtPersistentArgs& a, int cell, int nS, const uint32_t* bits, int* eqv,
                                uint64_t* qkeys, uint32_t* qvals, int* qhist, int* kq_out, int64_t* nq_out,
                                double* rq_out) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int beg = a.qf_ptr[cell], end = a.qf_ptr[cell + 1];
    for (int g = tid; g < a.Wt; g += NW * 32) eqv[g] = (bits[g >> 5] >> (g & 31)) & 1u ? 0 : SENT;
    if (tid == 0) {
        eqv[a.Wt] = SENT;  // the pad entries' gene id
        qhist[0] = 0;
    }
    __syncthreads();
    // the query's stored entries inside S, gathered by the whole CTA in any order (the ranks below
    // count #less / #equal, which do not depend on it)
    for (int i = beg + tid; i < end; i += NW * 32) {
        const int g = a.qf_idx[i];
        if ((bits[g >> 5] >> (g & 31)) & 1u) {
            const uint64_t key = ((uint64_t)ord_key(canon_zero(a.qf_data[i])) << 32) | (uint32_t)g;
            const int o = atomicAdd(&qhist[0], 1);
            if (o < a.capq) qkeys[o] = key;
        }
    }
    __syncthreads();
    const int k = qhist[0];
    __syncthreads();  // qhist is the ranking's scratch below
    if (warp == 0) {
        int64_t sq = 0;
        if (k <= a.capq) {
            // #less / #equal through 256 value buckets (as in the score step's rank kernel)
            int* cnt = qhist;
            int* cursor = qhist + 256;
            uint32_t kmin = 0xffffffffu, kmax = 0u;
            for (int j = lane; j < k; j += 32) {
                const uint32_t u = (uint32_t)(qkeys[j] >> 32);
                kmin = min(kmin, u);
                kmax = max(kmax, u);
            }
            kmin = __reduce_min_sync(FULL, kmin);
            kmax = __reduce_max_sync(FULL, kmax);
            const float fmin = key_float(kmin), span = key_float(kmax) - fmin;
            const float scale = (span > 0.f && span < 1e30f) ? 256.0f / span : 0.f;
            auto bucket = [&](uint32_t u) {
                const float t = (key_float(u) - fmin) * scale;
                return t >= 0.f ? min(255, (int)t) : 0;
            };
            for (int b = lane; b < 256; b += 32) cnt[b] = 0;
            __syncwarp();
            for (int j = lane; j < k; j += 32) atomicAdd(&cnt[bucket((uint32_t)(qkeys[j] >> 32))], 1);
            __syncwarp();
            int c[8], sum = 0;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                c[t] = cnt[8 * lane + t];
                sum += c[t];
            }
            int acc = warp_incl_scan(sum, lane) - sum;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                cursor[8 * lane + t] = acc;
                acc += c[t];
            }
            __syncwarp();
            for (int j = lane; j < k; j += 32) {
                const uint32_t u = (uint32_t)(qkeys[j] >> 32);
                qvals[atomicAdd(&cursor[bucket(u)], 1)] = u;
            }
            __syncwarp();
            for (int j = lane; j < k; j += 32) {
                const uint64_t key = qkeys[j];
                const uint32_t hv = (uint32_t)(key >> 32);
                const int b = bucket(hv), end_b = cursor[b];
                int less = end_b - cnt[b], eq = 0;
                for (int t = end_b - cnt[b]; t < end_b; ++t) {
                    less += qvals[t] < hv;
                    eq += qvals[t] == hv;
                }
                const int e = nS - k + 2 * less + eq;
                eqv[(int)(uint32_t)key] = e;
                sq += (int64_t)(e - k) * (e - k);
            }
        } else {
            for (int i = beg + lane; i < end; i += 32) {
                const int g = a.qf_idx[i];
                if (!((bits[g >> 5] >> (g & 31)) & 1u)) continue;
                const float v = canon_zero(a.qf_data[i]);
                int less = 0, eq = 0;
                for (int j = beg; j < end; ++j) {
                    const int h = a.qf_idx[j];
                    if (!((bits[h >> 5] >> (h & 31)) & 1u)) continue;
                    const float w = canon_zero(a.qf_data[j]);
                    less += w < v;
                    eq += w == v;
                }
                const int e = nS - k + 2 * less + eq;
                eqv[g] = e;
                sq += (int64_t)(e - k) * (e - k);
            }
        }
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(FULL, sq, o);
        if (lane == 0) {
            const int64_t nq = sq + (int64_t)(nS - k) * k * k;
            *kq_out = k;
            *nq_out = nq;
            *rq_out = nq > 0 ? 1.0 / sqrt((double)nq) : 0.0;
        }
    }
    __syncthreads();
}

// Reference-row slot layout of a candidate list: label i's rows are [off[i], off[i] + len), each
// label's range padded to a multiple of 32 slots so that a warp's 32 slots are one row block.
// Thread 0.
__device__ void label_offsets(const FtPersistentArgs& a, const uint8_t* top, int ntop, int* off) {
    int o = 0;
    for (int i = 0; i < ntop; ++i) {
        off[i] = o;
        o += ((int)a.ctidx[2 * top[i] + 1] + 31) & ~31;
    }
    off[ntop] = o;
}

// Walks a row's n4 16-byte entry vectors (32 vectors apart: the rows of a block are interleaved)
// with PF loads in flight: PF = 1 where many warps hide the latency (the work queue), deeper where
// few rows are scored at once (the late rounds of the spread path).
template <int PF, class F>
__device__ __forceinline__ void scan_words(const uint4* p, int n4, F&& fn) {
    uint4 buf[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) buf[u] = u < n4 ? __ldg(p + 32 * u) : make_uint4(0u, 0u, 0u, 0u);
    for (int t0 = 0; t0 < n4; t0 += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int t = t0 + u;
            if (t < n4) {
                const uint4 w4 = buf[u];
                if (t + PF < n4) buf[u] = __ldg(p + 32 * (t + PF));
                fn(w4);
            }
        }
    }
}

// Exact correlation over S of the query (eqv, kq, nq) with reference row slot f of the list.
// One thread: one pass over the row's value-sorted entries (see the top of this file).
// The rows of a label are scanned in the order of their 32-row blocks (rows sorted by length inside
// the label, so that a block's rows are of similar length); *dest receives the score's slot in the
// label's original row order, which the quantile's NaN-order rules depend on.
template <int PF>
__device__ float row_score(const FtPersistentArgs& a, const uint8_t* top, const int* off, int ntop, int f,
                           const int* eqv, int nS, int kq, int64_t nq, double rq, int* dest) {
    int lo = 0, hi = ntop - 1;  // label slot: off[lo] <= f < off[lo+1]
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= f) lo = mid;
        else hi = mid - 1;
    }
    const int lab = top[lo], j = f - off[lo];
    *dest = f;
    if (j >= (int)a.ctidx[2 * lab + 1]) return 0.f;  // padding slot of the label's range
    if (a.row_perm) *dest = off[lo] + (int)a.row_perm[a.ctidx[2 * lab] + j];
    const int blk = a.blk_base[lab] + (j >> 5);
    const int beg = a.ell_off[blk], n4 = (a.ell_off[blk + 1] - beg) >> 7;
    const uint4* p = reinterpret_cast<const uint4*>(a.ref_sorted + beg) + (j & 31);
    // Per entry: b, sum of the open run; at a run's last entry (flag bit 31) the run is closed.
    // Bounds (|S| <= Wt <= 40000, e <= 2|S|): sum, Y, z * sum / z < 2^32, b^3 < 2^63.
    uint32_t ka = 0, Y = 0;
    uint64_t X = 0, T = 0;
    if (a.pack_shift) {
        // packed e-values: (1 << shift) + e at genes of S, 0 elsewhere, so one add per entry keeps
        // the run's count (high bits) and e-sum (low bits); the host chose shift so that neither
        // field of a run can overflow
        const uint32_t* ep = reinterpret_cast<const uint32_t*>(eqv);
        const int sh = a.pack_shift;
        const uint32_t low = (1u << sh) - 1u;
        uint32_t acc = 0;
        if (a.narrow) {
            // X, sum b^3 fit 32 bits (the host checked 4 k^2 Wt < 2^32 and k^3 < 2^32 for the longest
            // row k): a run end is applied with masks, the same instructions for every lane, and
            // T = sum b^3 - k_r at the end
            uint32_t X32 = 0, B3 = 0;
            scan_words<PF>(p, n4, [&](const uint4 w4) {
                const uint32_t ws[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t ent = ws[u];
                    acc += ep[ent & 0xffffu];
                    const uint32_t m = (uint32_t)((int32_t)ent >> 31);  // all ones at a run's last entry
                    const uint32_t b = (acc >> sh) & m, sum = acc & low & m;
                    X32 += (2 * ka + b) * sum;
                    Y += sum;
                    B3 += b * b * b;
                    ka += b;
                    acc &= ~m;
                }
            });
            X = X32;
            T = (uint64_t)(B3 - ka);
        } else {
            scan_words<PF>(p, n4, [&](const uint4 w4) {
                const uint32_t ws[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t ent = ws[u];
                    acc += ep[ent & 0xffffu];
                    if ((int32_t)ent < 0) {  // last entry of its value run
                        const uint32_t b = acc >> sh, sum = acc & low;
                        X += (uint64_t)(2 * ka + b) * sum;
                        Y += sum;
                        T += (uint64_t)b * (b * b - 1u);
                        ka += b;
                        acc = 0;
                    }
                }
            });
        }
    } else {
        uint32_t b = 0, sum = 0;
        scan_words<PF>(p, n4, [&](const uint4 w4) {
            const uint32_t ws[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t ent = ws[u];
                const int v = eqv[ent & 0xffffu];
                b += v >= 0 ? 1u : 0u;
                sum += (uint32_t)max(v, 0);
                if ((int32_t)ent < 0) {  // last entry of its value run
                    X += (uint64_t)(2 * ka + b) * sum;
                    Y += sum;
                    T += (uint64_t)b * (b * b - 1u);
                    ka += b;
                    b = 0;
                    sum = 0;
                }
            }
        });
    }
    const int64_t kr = ka;
    const int64_t N = (int64_t)X + ((int64_t)nS - kr) * (int64_t)Y - (int64_t)nS * kq * kr;
    const int64_t c = (int64_t)nS - 2 * kr;
    const int64_t Z1 = kr * kr;
    const int64_t Z2 = (4 * kr * kr * kr - kr - (int64_t)T) / 3;
    const int64_t nr = Z2 + 2 * c * Z1 + kr * c * c + ((int64_t)nS - kr) * kr * kr;
    if (nq == 0 || nr == 0) return __int_as_float(0x7fffffff);
    return (float)(((double)N * rq) * (1.0 / sqrt((double)nr)));
}

// Per-label quantiles of the scores laid out by off[] (warps over labels).  CTA-wide.
template <int NW>
__device__ void cta_label_quantiles(const FtPersistentArgs& a, const uint8_t* top, const int* off, int ntop,
                                    const float* scores, float* lsc, int* hist, float* nan_scratch) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = warp; i < ntop; i += NW) {
        LabelQ q = a.lq_label[top[i]];
        const float v = quantile_warp(scores + off[i], q, a.p, hist + 256 * warp,
                                      nan_scratch + (size_t)warp * a.max_label, lane, a.status);
        if (lane == 0) lsc[i] = v;
    }
    (void)tid;
    __syncthreads();
}

// The reference's keep / drop rule (src/cusingler.cu:1270-1295) on the list order: returns the new
// list length, the new list in top.  One thread.
__device__ int decide_top(const float* lsc, int ntop, uint8_t* top, uint8_t* tmp, float thre) {
    int mn, mx;
    stl::minmax(lsc, ntop, &mn, &mx);
    const float lo = lsc[mn], hi = lsc[mx];
    const float t = __fsub_rn(hi, thre);
    int n = 0;
    if (!(hi != hi)) {
        for (int i = 0; i < ntop; ++i) {
            const float s = lsc[i];
            if (s <= lo || s < t) continue;
            if (s == hi) {
                for (int j = n; j > 0; --j) tmp[j] = tmp[j - 1];
                tmp[0] = top[i];
            } else {
                tmp[n] = top[i];
            }
            ++n;
        }
    }
    if (n == 0) {
        tmp[0] = top[0];
        n = 1;
    }
    for (int i = 0; i < n; ++i) top[i] = tmp[i];
    return n;
}

template <int NW>
__global__ void __launch_bounds__(NW * 32) ft_persistent_kernel(FtPersistentArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int Wt = a.Wt, L = a.L;
    const int nwords = (Wt + 31) / 32;
    int* eqv = reinterpret_cast<int*>(smem);                                     // Wt + 1
    uint32_t* bits = reinterpret_cast<uint32_t*>(eqv + ((Wt + 4) & ~3));         // nwords
    uint64_t* qkeys = reinterpret_cast<uint64_t*>(bits + ((nwords + 3) & ~3));   // capq (8-byte aligned)
    uint32_t* qvals = reinterpret_cast<uint32_t*>(qkeys + a.capq);                // capq
    int* hist = reinterpret_cast<int*>(qvals + a.capq);                           // NW * 256 (>= 512)
    float* lsc = reinterpret_cast<float*>(hist + NW * 256);                      // 256
    int* off = reinterpret_cast<int*>(lsc + 256);                                // 257
    int* red = off + 257;                                                        // NW
    uint8_t* top = reinterpret_cast<uint8_t*>(red + NW);                         // 256
    uint8_t* ntopv = top + 256;                                                  // 256
    __shared__ FtShared sh;

    float* scores = a.scratch + (size_t)blockIdx.x * a.scratch_per_cta;
    float* nan_scratch = scores + a.max_rcand;

    for (;;) {
        if (tid == 0) {
            const int i = atomicAdd(a.next_cell, 1);
            const int n = a.cell_list ? *a.n_list : a.Q;
            sh.cell = i < n ? (a.cell_list ? a.cell_list[i] : i) : -1;
        }
        __syncthreads();
        const int cell = sh.cell;
        if (cell < 0) break;
        if (warp == 0) {
            const int n = warp_flagged_labels(a.flags + (size_t)cell * L, L, top, lane);
            if (lane == 0) {
                sh.ntop = n;
                sh.rounds = 0;
            }
        }
        __syncthreads();
        int times_used = 0;
        for (;;) {
            const int ntop = sh.ntop;
            if (!(ntop > 1 && (a.times == 0 || times_used++ < a.times))) break;
            const int nS = cta_gene_set<NW>(a, top, ntop, bits, red);
            if (tid == 0) sh.rounds++;
            if (nS < 20) {  // keep the first candidate (src/cusingler.cu:1158-1159)
                if (tid == 0) sh.ntop = 1;
                __syncthreads();
                continue;
            }
            cta_query_ranks<NW>(a, cell, nS, bits, eqv, qkeys, qvals, hist, &sh.kq, &sh.nq, &sh.rq);
            if (a.pack_shift)
                for (int g = tid; g <= Wt; g += NW * 32) eqv[g] = pack_e(eqv[g], a.pack_shift);
            if (tid == 0) label_offsets(a, top, ntop, off);
            __syncthreads();
            const int total = off[ntop];
            const int kq = sh.kq;
            const int64_t nq = sh.nq;
            const double rq = sh.rq;
            for (int f = tid; f < total; f += NW * 32) {
                int dst;
                const float v = row_score<1>(a, top, off, ntop, f, eqv, nS, kq, nq, rq, &dst);
                scores[dst] = v;
            }
            __syncthreads();
            cta_label_quantiles<NW>(a, top, off, ntop, scores, lsc, hist, nan_scratch);
            if (tid == 0) sh.ntop = decide_top(lsc, ntop, top, ntopv, a.thre);
            __syncthreads();
        }
        if (tid == 0) {
            a.final_labels[cell] = sh.ntop > 0 ? (int32_t)top[0] : 0;
            if (a.rounds) a.rounds[cell] = sh.rounds;
        }
        __syncthreads();
    }
}

// ---- split path: the rounds of many heavy cells spread over the whole GPU ----------------------
//
// State per heavy cell i (device arrays of FtSplit): candidate list, its length, rounds, times used,
// state; per round: the query's e-values, |S|, k_q, n_q, label offsets and the scores.  A round is
// two launches: the scan of the 256-row chunks of every active cell (a compact chunk list, filled by
// the previous launch), then per cell the quantiles, the keep / drop rule and the setup of its next
// round (gene set, query ranks, its chunks appended to the other list).  The cells that take many
// rounds keep many candidates for most of them, so the scan stays the bulk of the work: chunks are
// spread over a grid of 16 CTAs per SM, rows scanned with four loads in flight, and the scores of a
// round are staged in shared memory for the quantiles.

constexpr int SPLIT_STAGE = 21504;  // rows of a round whose scores are staged for the quantiles
constexpr int SPLIT_NW = 16;        // warps of the setup and decision CTAs
constexpr int SPLIT_SCAN_PF = 4;    // entry vectors in flight per row in the spread scan
constexpr int SPLIT_SCAN_CTAS = 16; // scan CTAs per SM

// Cell i is done: its first candidate is the final label.  One thread.
__device__ void split_finish(const FtPersistentArgs& a, const FtSplit& sp, int i, int cell, int ntop) {
    a.final_labels[cell] = ntop > 0 ? (int32_t)sp.top[(size_t)i * 256] : 0;
    if (a.rounds) a.rounds[cell] = sp.rounds[i];
    sp.state[i] = 2;
    sp.total[i] = 0;
}

// Setup of cell i's next round, CTA-wide (256 threads): the round condition, gene set, the query's
// ranks (e-values into sp.eqv), label offsets, and the round's chunks appended to chunk list q.
// smem: split_prepare_smem bytes.
__device__ void split_setup_round(const FtPersistentArgs& a, const FtSplit& sp, int i, int q, unsigned char* smem) {
    constexpr int NW = SPLIT_NW;
    const int tid = threadIdx.x;
    const int Wt = a.Wt;
    const int nwords = (Wt + 31) / 32;
    int* eqv = reinterpret_cast<int*>(smem);
    uint32_t* bits = reinterpret_cast<uint32_t*>(eqv + ((Wt + 4) & ~3));
    uint64_t* qkeys = reinterpret_cast<uint64_t*>(bits + ((nwords + 3) & ~3));
    uint32_t* qvals = reinterpret_cast<uint32_t*>(qkeys + a.capq);
    int* qhist = reinterpret_cast<int*>(qvals + a.capq);  // 512
    int* red = qhist + 512;
    __shared__ int s_go, s_kq;
    __shared__ int64_t s_nq;
    __shared__ double s_rq;
    const int cell = sp.cells[i];
    const uint8_t* top = sp.top + (size_t)i * 256;
    const int ntop = sp.ntop[i];
    if (tid == 0) {
        bool go = sp.state[i] == 1 && ntop > 1;
        if (go && a.times != 0) go = sp.times[i]++ < a.times;
        if (go) sp.rounds[i]++;
        else split_finish(a, sp, i, cell, ntop);
        s_go = go;
    }
    __syncthreads();
    if (!s_go) return;
    const int nS = cta_gene_set<NW>(a, top, ntop, bits, red);
    if (nS < 20) {  // keep the first candidate (src/cusingler.cu:1158-1159)
        if (tid == 0) {
            sp.ntop[i] = 1;
            split_finish(a, sp, i, cell, 1);
        }
        return;
    }
    cta_query_ranks<NW>(a, cell, nS, bits, eqv, qkeys, qvals, qhist, &s_kq, &s_nq, &s_rq);
    int* geqv = sp.eqv + (size_t)i * Wt;
    for (int g = tid; g < Wt; g += NW * 32) geqv[g] = eqv[g];
    if (tid == 0) {
        int* off = sp.off + (size_t)i * 257;
        label_offsets(a, top, ntop, off);
        const int total = off[ntop];
        sp.nS[i] = nS;
        sp.kq[i] = s_kq;
        sp.nq[i] = s_nq;
        sp.rq[i] = s_rq;
        sp.total[i] = total;
        atomicAdd(sp.rows_scored, (unsigned long long)total);
        const int nch = (total + 255) / 256;
        const int base = atomicAdd(sp.n_items + q, nch);
        int* items = sp.items + (size_t)q * sp.max_items;
        for (int c = 0; c < nch; ++c) items[base + c] = i * sp.max_chunks + c;
    }
}

// First round of every heavy cell: candidates from the flags, then the round's setup (chunk list 0).
// grid = H.
__global__ void __launch_bounds__(SPLIT_NW * 32) split_first_kernel(FtPersistentArgs a, FtSplit sp) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int i = blockIdx.x, lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
        const int n = warp_flagged_labels(a.flags + (size_t)sp.cells[i] * a.L, a.L, sp.top + (size_t)i * 256, lane);
        if (lane == 0) {
            sp.ntop[i] = n;
            sp.rounds[i] = 0;
            sp.times[i] = 0;
            sp.state[i] = 1;
            sp.total[i] = 0;
        }
    }
    __syncthreads();
    split_setup_round(a, sp, i, 0, smem);
}

// Scores of the chunks on list q (item i * max_chunks + c: rows [256 c, 256 c + 256) of cell i's
// round); also clears the other list's count for the setups that follow.  Fixed grid striding over
// the items; a CTA reloads the cell's tables (e-values, offsets, candidates) when the cell changes.
__global__ void __launch_bounds__(256) split_scan_kernel(FtPersistentArgs a, FtSplit sp, int q) {
    extern __shared__ __align__(16) unsigned char smem[];
    int* eqv = reinterpret_cast<int*>(smem);
    int* off = eqv + ((a.Wt + 4) & ~3);
    uint8_t* top = reinterpret_cast<uint8_t*>(off + 260);
    __shared__ int s_ntop;
    if (blockIdx.x == 0 && threadIdx.x == 0) sp.n_items[q ^ 1] = 0;
    const int n = sp.n_items[q];
    const int* items = sp.items + (size_t)q * sp.max_items;
    int cur = -1;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const int it = items[t];
        const int i = it / sp.max_chunks, c = it % sp.max_chunks;
        if (i != cur) {
            __syncthreads();  // the previous cell's tables are no longer read
            const int* geqv = sp.eqv + (size_t)i * a.Wt;
            const int ntop = sp.ntop[i];
            if (a.pack_shift) {
                for (int g = threadIdx.x; g < a.Wt; g += 256) eqv[g] = pack_e(geqv[g], a.pack_shift);
            } else {
                for (int g = threadIdx.x; g < a.Wt; g += 256) eqv[g] = geqv[g];
            }
            if (threadIdx.x == 0) {
                eqv[a.Wt] = a.pack_shift ? 0 : SENT;
                s_ntop = ntop;
            }
            for (int u = threadIdx.x; u <= ntop; u += 256) off[u] = sp.off[(size_t)i * 257 + u];
            for (int u = threadIdx.x; u < ntop; u += 256) top[u] = sp.top[(size_t)i * 256 + u];
            __syncthreads();
            cur = i;
        }
        const int f = c * 256 + (int)threadIdx.x;
        if (f < sp.total[i]) {
            int dst;
            const float v = row_score<SPLIT_SCAN_PF>(a, top, off, s_ntop, f, eqv, sp.nS[i], sp.kq[i], sp.nq[i],
                                                     sp.rq[i], &dst);
            sp.scores[(size_t)i * sp.max_rcand + dst] = v;
        }
    }
}

// Per cell scanned this round: quantiles (from shared memory when the round's scores fit), the keep /
// drop rule, then the setup of its next round (chunks appended to list q).  grid = H.
__global__ void __launch_bounds__(SPLIT_NW * 32) split_decide_kernel(FtPersistentArgs a, FtSplit sp, int q) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int NW = SPLIT_NW;
    __shared__ int hist[NW * 256];
    __shared__ float lsc[256];
    __shared__ int off[257];
    __shared__ uint8_t top[256], tmp[256];
    const int i = blockIdx.x;
    const int total = sp.total[i];
    if (total == 0) return;  // finished
    const int ntop = sp.ntop[i];
    for (int t = threadIdx.x; t <= ntop; t += NW * 32) off[t] = sp.off[(size_t)i * 257 + t];
    for (int t = threadIdx.x; t < ntop; t += NW * 32) top[t] = sp.top[(size_t)i * 256 + t];
    const float* scores = sp.scores + (size_t)i * sp.max_rcand;
    if (total <= SPLIT_STAGE) {  // total is a multiple of 32 (label ranges are padded to 32 rows)
        float4* st = reinterpret_cast<float4*>(smem);
        const float4* src = reinterpret_cast<const float4*>(scores);
        for (int t = threadIdx.x; t < total / 4; t += NW * 32) st[t] = src[t];
        scores = reinterpret_cast<const float*>(smem);
    }
    __syncthreads();
    cta_label_quantiles<NW>(a, top, off, ntop, scores, lsc, hist, sp.nan_scratch + (size_t)i * NW * a.max_label);
    if (threadIdx.x == 0) {
        const int n = decide_top(lsc, ntop, top, tmp, a.thre);
        for (int t = 0; t < n; ++t) sp.top[(size_t)i * 256 + t] = top[t];
        sp.ntop[i] = n;
    }
    __syncthreads();
    split_setup_round(a, sp, i, q, smem);
}

}  // namespace

size_t split_prepare_smem(int Wt, int capq) {
    const int nwords = (Wt + 31) / 32;
    return sizeof(int) * ((Wt + 4) & ~3) + sizeof(uint32_t) * ((nwords + 3) & ~3) + sizeof(uint64_t) * capq +
           sizeof(uint32_t) * capq + sizeof(int) * (512 + 16);
}

namespace {
size_t split_decide_smem(int Wt, int capq) {
    return std::max(split_prepare_smem(Wt, capq), sizeof(float) * SPLIT_STAGE);
}
size_t split_scan_smem(int Wt) { return sizeof(int) * (((Wt + 4) & ~3) + 260) + 256; }
}  // namespace

void split_round_setup(const FtPersistentArgs& a) {
    SGR_CUDA(cudaFuncSetAttribute(split_first_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)split_prepare_smem(a.Wt, a.capq)));
    SGR_CUDA(cudaFuncSetAttribute(split_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)split_scan_smem(a.Wt)));
    SGR_CUDA(cudaFuncSetAttribute(split_decide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)split_decide_smem(a.Wt, a.capq)));
}

void launch_split_first(const FtPersistentArgs& a, const FtSplit& sp, int H, cudaStream_t s) {
    split_first_kernel<<<H, SPLIT_NW * 32, split_prepare_smem(a.Wt, a.capq), s>>>(a, sp);
    SGR_LAUNCH_CHECK();
    count_launch(1);
}

void launch_split_round(const FtPersistentArgs& a, const FtSplit& sp, int H, int q, cudaStream_t s) {
    split_scan_kernel<<<SPLIT_SCAN_CTAS * device_sm_count(), 256, split_scan_smem(a.Wt), s>>>(a, sp, q);
    SGR_LAUNCH_CHECK();
    split_decide_kernel<<<H, SPLIT_NW * 32, split_decide_smem(a.Wt, a.capq), s>>>(a, sp, q ^ 1);
    SGR_LAUNCH_CHECK();
    count_launch(2);
}

void launch_ft_keys(int n, const int32_t* list, int L, const uint8_t* flags, const uint32_t* ctidx, int64_t* keys,
                    int32_t* ncand, cudaStream_t s) {
    if (n <= 0) return;
    ft_keys_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, list, L, flags, ctidx, keys, ncand);
    SGR_LAUNCH_CHECK();
    count_launch();
}

size_t ft_persistent_smem(int Wt, int capq, int nw) {
    const int nwords = (Wt + 31) / 32;
    size_t b = 0;
    b += sizeof(int) * ((Wt + 4) & ~3);
    b += sizeof(uint32_t) * ((nwords + 3) & ~3);
    b += sizeof(uint64_t) * capq + sizeof(uint32_t) * capq;
    b += sizeof(int) * (size_t)nw * 256 + sizeof(float) * 256 + sizeof(int) * (257 + nw) + 512;
    return (b + 15) & ~size_t(15);
}

void launch_ref_presort(const float* data, const int32_t* idx, const int32_t* ptr, const int32_t* ell_base,
                        const int32_t* ell_len, uint32_t n_rows, int cap, uint32_t pad_gene, uint32_t* out,
                        cudaStream_t s) {
    if (!n_rows) return;
    int wpb = std::max(1, std::min(8, (200 * 1024) / (cap * 8)));
    const size_t smem = (size_t)wpb * cap * 8;
    SGR_CUDA(cudaFuncSetAttribute(ref_presort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned blocks = std::min<unsigned>((n_rows + wpb - 1) / wpb, device_sm_count() * 8);
    ref_presort_kernel<<<blocks, 32 * wpb, smem, s>>>(data, idx, ptr, ell_base, ell_len, n_rows, cap, pad_gene, out);
    SGR_LAUNCH_CHECK();
    count_launch();
}

namespace {
template <int NW>
int ft_grid_t(size_t smem) {
    SGR_CUDA(cudaFuncSetAttribute(ft_persistent_kernel<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ft_persistent_kernel<NW>, NW * 32, smem);
    if (per_sm < 1) per_sm = 1;
    return device_sm_count() * per_sm;
}
}  // namespace

int ft_persistent_grid(size_t smem, int nw) { return nw == 32 ? ft_grid_t<32>(smem) : ft_grid_t<8>(smem); }

void launch_ft_persistent(const FtPersistentArgs& a, int grid, size_t smem, int nw, cudaStream_t s) {
    if (nw == 32) {
        SGR_CUDA(cudaFuncSetAttribute(ft_persistent_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ft_persistent_kernel<32><<<grid, 1024, smem, s>>>(a);
    } else {
        SGR_CUDA(cudaFuncSetAttribute(ft_persistent_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ft_persistent_kernel<8><<<grid, 256, smem, s>>>(a);
    }
    SGR_LAUNCH_CHECK();
    count_launch();
}

}  // namespace sgr
