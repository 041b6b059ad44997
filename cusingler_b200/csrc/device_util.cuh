// Device helpers shared by the kernels: ordered float keys, warp sorts and searches, and the
// per-label quantile of the reference's percentile() (src/cusingler.cu:947-978 of
// STOmics/cusingler) by radix selection, with libstdc++'s sort order for NaN-bearing lists.
#pragma once

#include <climits>
#include <cstdint>

#include "kernels.cuh"
#include "stl_order.h"

namespace sgr {
namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t ord_key(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float key_float(uint32_t k) {
    uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// -0 and +0 are one value (the reference keys its per-row value codes with std::set<float>).
__device__ __forceinline__ float canon_zero(float v) {
    uint32_t u = __float_as_uint(v);
    return (u << 1) == 0 ? 0.0f : v;
}

// d = 128*h + l with l in [-64, 63]; s = h + l (the Karatsuba limb).
// Int8 limbs of a doubled centred rank d, written as planes (p0, l, s), with d = m * p0 + s:
//   w = 0: d = 128 h + l, l in [-64, 63], p0 = h, s = h + l (m = 127);
//   w > 0: d = C h + l with C = w^2 + 1, l in [-C/2, C - 1 - C/2], p0 = w h, s = h + l (m = w).
// The second split lets the exact product use two accumulators: d d' = C (p0 p0' + s s') - (C-1) l l'.
// The host picks w so that every limb of |d| < G fits int8.
__device__ __forceinline__ void split_limbs(int d, int w, int& p0, int& l, int& s) {
    if (w == 0) {
        l = ((d + 64) & 127) - 64;
        p0 = (d - l) >> 7;
        s = p0 + l;
        return;
    }
    const int C = w * w + 1, hc = C >> 1;
    const int h = (d + hc + 4096 * C) / C - 4096;  // floor((d + hc) / C) for |d| < 4096 C
    l = d - C * h;
    s = h + l;
    p0 = w * h;
}


__device__ __forceinline__ int64_t warp_sum_i64(int64_t v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ int lower_hi(const uint64_t* keys, int n, uint32_t hv) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if ((uint32_t)(keys[mid] >> 32) < hv) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ int upper_hi(const uint64_t* keys, int n, uint32_t hv) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if ((uint32_t)(keys[mid] >> 32) <= hv) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Ascending bitonic sort of n (power of two) keys in shared memory by one warp.
__device__ void warp_bitonic(uint64_t* keys, int n, int lane) {
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < (n >> 1); t += 32) {
                int i = 2 * t - (t & (stride - 1));
                int j = i + stride;
                uint64_t a = keys[i], b = keys[j];
                bool up = (i & size) == 0;
                if ((a > b) == up) {
                    keys[i] = b;
                    keys[j] = a;
                }
            }
            __syncwarp();
        }
    }
}

__device__ __forceinline__ float interp(float p, float prev_index, float step, float a, float b) {
    // (p - prev_index) * (b - a) / step + a, each operation rounded once (src/cusingler.cu:975)
    return __fadd_rn(__fdiv_rn(__fmul_rn(__fsub_rn(p, prev_index), __fsub_rn(b, a)), step), a);
}

__device__ __forceinline__ int warp_incl_scan(int x, int lane) {
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Key of the j-th smallest (0-based) of v[0..n) by 4 passes of an 8-bit radix histogram.
// `common` high bits are shared by every key (from the list's minimum and maximum): the radix
// passes start below them.
__device__ uint32_t warp_select(const float* v, int n, int j, int* hist, int lane, uint32_t kmin = 0,
                                int common = 0) {
    uint32_t mask = common ? ~0u << (32 - common) : 0u;
    uint32_t prefix = kmin & mask;
    const int low = 32 - common;  // bits still to resolve
    int shift = low - 8;
    for (;; shift -= 8) {
        if (shift < 0) shift = 0;
        for (int b = lane; b < 256; b += 32) hist[b] = 0;
        __syncwarp();
        for (int i = lane; i < n; i += 32) {
            const uint32_t u = ord_key(v[i]);
            if ((u & mask) == prefix) atomicAdd(&hist[(u >> shift) & 255], 1);
        }
        __syncwarp();
        int c[8], s = 0;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            c[t] = hist[8 * lane + t];
            s += c[t];
        }
        const int incl = warp_incl_scan(s, lane), excl = incl - s;
        const unsigned own = __ballot_sync(FULL, excl <= j && j < incl);
        const int src = __ffs(own) - 1;
        int bin = 0, before = 0;
        if (lane == src) {
            int acc = excl;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                if (j < acc + c[t]) {
                    bin = 8 * lane + t;
                    before = acc;
                    break;
                }
                acc += c[t];
            }
        }
        bin = __shfl_sync(FULL, bin, src);
        before = __shfl_sync(FULL, before, src);
        j -= before;
        prefix |= (uint32_t)bin << shift;
        mask |= 0xffu << shift;
        __syncwarp();
        if (shift == 0) break;
    }
    return prefix;
}

__device__ __forceinline__ uint32_t warp_min_u32(uint32_t x) { return __reduce_min_sync(FULL, x); }
__device__ __forceinline__ uint32_t warp_max_u32(uint32_t x) { return __reduce_max_sync(FULL, x); }

// Keys of order statistics j and j+1 (0-based) of v[0..n) (no NaN, kmin < kmax) by one warp: a
// 256-bin histogram over a monotone linear map of [min, max] locates the bin holding statistic j;
// that bin's keys (at most 256) are compacted into `buf` (the histogram's memory) and sorted.
// Returns false (nothing decided) when the bin is larger than 256 or the range is degenerate.
__device__ bool bucket_select(const float* v, int n, int j, int* hist, int lane, uint32_t kmin, uint32_t kmax,
                              uint32_t* ka, uint32_t* kb) {
    const float fmin = key_float(kmin), fmax = key_float(kmax);
    const float span = fmax - fmin;
    if (!(span > 1e-30f) || !(span < 1e30f)) return false;
    const float scale = __fdividef(256.0f, span);  // any positive scale keeps the map monotone
    // The bin of x is round-to-nearest((x - min) * scale), read from the bits of one FMA whose result
    // lies in [2^23, 2^24), where floats are the integers: bits(y) = 0x4B000000 + y - 2^23.  The map
    // from x to those bits is monotone non-decreasing, which is all the selection needs (both passes
    // use the same map).  Clamped both ways on the bits, so that a value outside [min, max] (extremes
    // that do not match the list) still lands in a bin rather than outside the histogram.
    constexpr int B0 = 0x4B000000;
    const float shift = fmaf(-fmin, scale, 8388608.0f);
    auto bin_bits = [&](float x) { return __float_as_int(fmaf(x, scale, shift)); };
    auto bin_of = [&](float x) { return min(max(bin_bits(x), B0), B0 + 255) - B0; };
    for (int b = lane; b < 256; b += 32) hist[b] = 0;
    __syncwarp();
    int i = lane;
    for (; i + 96 < n; i += 128) {  // four independent loads in flight per lane
        const float x0 = v[i], x1 = v[i + 32], x2 = v[i + 64], x3 = v[i + 96];
        atomicAdd(&hist[bin_of(x0)], 1);
        atomicAdd(&hist[bin_of(x1)], 1);
        atomicAdd(&hist[bin_of(x2)], 1);
        atomicAdd(&hist[bin_of(x3)], 1);
    }
    for (; i < n; i += 32) atomicAdd(&hist[bin_of(v[i])], 1);
    __syncwarp();
    int c[8], s = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        c[t] = hist[8 * lane + t];
        s += c[t];
    }
    const int incl = warp_incl_scan(s, lane), excl = incl - s;
    const unsigned own = __ballot_sync(FULL, excl <= j && j < incl);
    const int src = __ffs(own) - 1;
    int bin = 0, before = 0, cnt = 0;
    if (lane == src) {
        int acc = excl;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            if (j < acc + c[t]) {
                bin = 8 * lane + t;
                before = acc;
                cnt = c[t];
                break;
            }
            acc += c[t];
        }
    }
    bin = __shfl_sync(FULL, bin, src);
    before = __shfl_sync(FULL, before, src);
    cnt = __shfl_sync(FULL, cnt, src);
    if (cnt > 256) return false;
    // when statistic j is the last of its bin and j + 1 exists, statistic j + 1 is the smallest value
    // of the next non-empty bin: collect that bin too (the bins between are empty)
    int nb = -1, total = cnt;
    if (j + 1 >= before + cnt && j + 1 < n) {
        int cand = 256, ccand = 0;
#pragma unroll
        for (int t = 0; t < 8; ++t)
            if (cand == 256 && 8 * lane + t > bin && c[t] > 0) {
                cand = 8 * lane + t;
                ccand = c[t];
            }
        nb = __reduce_min_sync(FULL, cand);
        const int cnb = __reduce_add_sync(FULL, cand == nb ? ccand : 0);
        if (cnt + cnb <= 256) total = cnt + cnb;
        else nb = -1;
    }
    __syncwarp();
    // Collect the values of bins bin..last (the bins between bin and nb are empty), compared on the
    // map's bits: bin(x) >= bin holds for every x when bin is 0, else exactly when bits >= B0 + bin;
    // bin(x) <= last likewise.  Raw float bits are stored and turned into order keys afterwards.
    const int last = nb >= 0 ? nb : bin;
    const int lo = bin == 0 ? INT_MIN : B0 + bin, hi = last == 255 ? INT_MAX : B0 + last;
    uint32_t* buf = reinterpret_cast<uint32_t*>(hist);
    int w = 0;
    const unsigned lt = (1u << lane) - 1u;
    int base = 0;
    for (; base + 64 <= n; base += 64) {  // two 32-value chunks per step
        const float x0 = v[base + lane], x1 = v[base + 32 + lane];
        const int y0 = bin_bits(x0), y1 = bin_bits(x1);
        const bool in0 = y0 >= lo && y0 <= hi, in1 = y1 >= lo && y1 <= hi;
        const unsigned m0 = __ballot_sync(FULL, in0), m1 = __ballot_sync(FULL, in1);
        if (in0) buf[w + __popc(m0 & lt)] = __float_as_uint(x0);
        if (in1) buf[w + __popc(m0) + __popc(m1 & lt)] = __float_as_uint(x1);
        w += __popc(m0) + __popc(m1);
    }
    for (; base < n; base += 32) {
        const int i0 = base + lane;
        const float x0 = i0 < n ? v[i0] : 0.f;
        const int y0 = bin_bits(x0);
        const bool in0 = i0 < n && y0 >= lo && y0 <= hi;
        const unsigned m0 = __ballot_sync(FULL, in0);
        if (in0) buf[w + __popc(m0 & lt)] = __float_as_uint(x0);
        w += __popc(m0);
    }
    __syncwarp();
    const int r = j - before;  // statistic j is the r-th smallest collected key (r < cnt <= total)
    bool have_b = r + 1 < total;
    if (total <= 32) {
        // one key per lane; its rank among the collected keys (ties by position) picks r and r + 1
        const uint32_t key = lane < total ? ord_key(__uint_as_float(buf[lane])) : 0xffffffffu;
        int rank = 0;
        for (int t = 0; t < total; ++t) {
            const uint32_t kt = __shfl_sync(FULL, key, t);
            rank += (kt < key) | ((kt == key) & (t < lane));
        }
        *ka = __shfl_sync(FULL, key, __ffs(__ballot_sync(FULL, lane < total && rank == r)) - 1);
        const unsigned mb = __ballot_sync(FULL, lane < total && rank == r + 1);
        if (have_b) *kb = __shfl_sync(FULL, key, __ffs(mb) - 1);
    } else {
        for (int i = lane; i < total; i += 32) buf[i] = ord_key(__uint_as_float(buf[i]));
        int np = 1;
        while (np < total) np <<= 1;
        for (int i = total + lane; i < np; i += 32) buf[i] = 0xffffffffu;
        __syncwarp();
        for (int size = 2; size <= np; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int t = lane; t < (np >> 1); t += 32) {
                    const int a = 2 * t - (t & (stride - 1)), b = a + stride;
                    const uint32_t x = buf[a], y = buf[b];
                    if ((x > y) == ((a & size) == 0)) {
                        buf[a] = y;
                        buf[b] = x;
                    }
                }
                __syncwarp();
            }
        *ka = buf[r];
        if (have_b) *kb = buf[r + 1];
    }
    if (!have_b) {  // statistic j + 1 lies beyond the collected bins: the smallest key above ka
        uint32_t nxt = 0xffffffffu;
        for (int i = lane; i < n; i += 32) {
            const uint32_t u = ord_key(v[i]);
            if (u > *ka) nxt = min(nxt, u);
        }
        *kb = __reduce_min_sync(FULL, nxt);
    }
    __syncwarp();
    return true;
}

// quantile_warp after its min / max / NaN pass: kmin, kmax are the warp-wide extreme order keys of
// the list and nan whether it holds a NaN (all lanes agree).  Lists holding NaN are sorted exactly as
// libstdc++ would, in `scratch` (n floats), by lane 0.
__device__ float quantile_warp_core(const float* v, const LabelQ& lq, float p, int* hist, float* scratch, int lane,
                                    int* status, uint32_t kmin, uint32_t kmax, bool nan) {
    const int n = lq.len;
    if (nan) {
        float r = 0.f;
        if (scratch == nullptr) {
            if (lane == 0) atomicOr(status, 8);
            return __int_as_float(0x7fffffff);
        }
        for (int i = lane; i < n; i += 32) scratch[i] = v[i];
        __syncwarp();
        if (lane == 0) {
            int oob = 0;
            stl::sort(scratch, n, &oob);
            if (oob) atomicOr(status, 4);
            if (lq.kind == 1) r = scratch[0];
            else if (lq.kind == 2) r = scratch[n - 1];
            else r = interp(p, lq.prev_index, lq.step, scratch[lq.k - 1], scratch[lq.k]);
        }
        __syncwarp();
        return __shfl_sync(FULL, r, 0);
    }
    if (lq.kind == 1) return key_float(kmin);
    if (lq.kind == 2) return key_float(kmax);
    if (kmin == kmax) return interp(p, lq.prev_index, lq.step, key_float(kmin), key_float(kmin));
    uint32_t ka, kb;
    if (bucket_select(v, n, lq.k - 1, hist, lane, kmin, kmax, &ka, &kb))
        return interp(p, lq.prev_index, lq.step, key_float(ka), key_float(kb));
    ka = warp_select(v, n, lq.k - 1, hist, lane);
    int le = 0;
    uint32_t nxt = 0xffffffffu;
    for (int i = lane; i < n; i += 32) {
        const uint32_t u = ord_key(v[i]);
        le += u <= ka;
        if (u > ka) nxt = min(nxt, u);
    }
    le = __reduce_add_sync(FULL, le);
    nxt = warp_min_u32(nxt);
    kb = le > lq.k ? ka : nxt;
    return interp(p, lq.prev_index, lq.step, key_float(ka), key_float(kb));
}

// The reference's percentile(v, n, p) (src/cusingler.cu:947-978) for one score list, by one warp.
__device__ float quantile_warp(const float* v, const LabelQ& lq, float p, int* hist, float* scratch, int lane,
                               int* status) {
    const int n = lq.len;
    if (lq.kind == 0) return v[0];
    bool nan = false;
    uint32_t mn0 = 0xffffffffu, mn1 = 0xffffffffu, mx0 = 0u, mx1 = 0u;
    int i = lane;
    for (; i + 32 < n; i += 64) {  // two independent chains per lane
        const float x0 = v[i], x1 = v[i + 32];
        nan |= (x0 != x0) | (x1 != x1);
        const uint32_t u0 = ord_key(x0), u1 = ord_key(x1);
        mn0 = min(mn0, u0);
        mx0 = max(mx0, u0);
        mn1 = min(mn1, u1);
        mx1 = max(mx1, u1);
    }
    if (i < n) {
        const float x = v[i];
        nan |= x != x;
        const uint32_t u = ord_key(x);
        mn0 = min(mn0, u);
        mx0 = max(mx0, u);
    }
    nan = __any_sync(FULL, nan);
    const uint32_t kmin = __reduce_min_sync(FULL, min(mn0, mn1));
    const uint32_t kmax = __reduce_max_sync(FULL, max(mx0, mx1));
    return quantile_warp_core(v, lq, p, hist, scratch, lane, status, kmin, kmax, nan);
}


}  // namespace
}  // namespace sgr
