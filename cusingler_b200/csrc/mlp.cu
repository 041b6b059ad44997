// Learned proposal: a small MLP that predicts a cell's final fine-tuned label from its first-round
// per-label quantile scores, so that confident cells can skip the fine-tune loop.  It has no
// counterpart in the reference; it is trained on labels the plain method produces.
//
// Network: x = (scores - max(scores)) / 0.05 clipped at -8 (L inputs) -> 256 -> GELU -> 256 -> GELU
// -> L -> softmax.
// Weights are kept as FP32 master copies (updated by AdamW) and BF16 working copies (used by the
// forward and backward products); every product accumulates in FP32.  All kernels are hand-written:
// a tiled CUDA-core GEMM with strided operands for training, fused bias + GELU epilogues, softmax
// cross-entropy, bias reductions and AdamW.  Inference (predict) runs the three products on the
// tensor cores instead.

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "kernels.cuh"
#include "mlp.h"
#include "sgr_internal.h"

namespace sgr {
namespace {

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }

// C[m][n] (ldc) = sum_k A(m,k) B(k,n) (+ bias[n]) with A(m,k) = A[m*am + k*ak], B(k,n) = B[k*bk + n*bn].
// epi 0: plain store; 1: + bias; 2: + bias, store pre-activation to Z and GELU to C.
template <class TA, class TB>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const TA* A, int64_t am, int64_t ak,
                                                   const TB* B, int64_t bk, int64_t bn, float* C, int64_t ldc,
                                                   const float* bias, float* Z, int epi) {
    __shared__ float As[16][64 + 1];
    __shared__ float Bs[16][64 + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int i = threadIdx.x; i < 16 * 64; i += 256) {
            const int kk = i / 64, mm = i % 64;
            const int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < M && k < K) ? to_f(A[m * am + k * ak]) : 0.f;
            const int n = n0 + mm;
            Bs[kk][mm] = (n < N && k < K) ? to_f(B[k * bk + n * bn]) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            float v = acc[i][j];
            if (epi >= 1) v += bias[n];
            if (epi == 2) {
                Z[m * ldc + n] = v;
                v = 0.5f * v * (1.f + erff(v * 0.70710678118654752f));
            }
            C[m * ldc + n] = v;
        }
    }
}

// Inference product on the tensor cores (mma.sync m16n8k16, BF16 inputs, FP32 accumulation):
// C[m][n] = act(sum_k A[m][k] W[n][k] + bias[n]) with A FP32 (row-major, lda) and W BF16 (row-major
// [N][K], ldw).  Each A value is split into BF16 hi + lo (a - hi - lo is within 2^-16 |a|), so two
// products per tile keep the FP32 activations' precision.  gelu: apply GELU after the bias.
// Block tile BM x BN with 8 warps in WARPS_M x WARPS_N, each warp 32 rows x BN / WARPS_N columns; one
// block spans every output column of a 256-wide layer, so each A row is loaded and split once.  K in
// steps of 64; shared rows padded to 72 values (36 words), so the fragment loads are conflict-free.
// 16-byte loads when rows and K allow them, element loads otherwise (the first layer's K = labels).
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ void split_store(__nv_bfloat16* hi, __nv_bfloat16* lo, float a) {
    const __nv_bfloat16 h = __float2bfloat16_rn(a);
    *hi = h;
    *lo = __float2bfloat16_rn(a - __bfloat162float(h));
}

template <int BN, int WARPS_N>
__global__ void __launch_bounds__(256, 2) gemm_tc_kernel(int M, int N, int K, const float* A, int64_t lda,
                                                         const __nv_bfloat16* W, int64_t ldw, const float* bias,
                                                         float* C, int64_t ldc, int gelu) {
    constexpr int WARPS_M = 8 / WARPS_N, BM = 32 * WARPS_M, WN = BN / WARPS_N, NT = WN / 8;
    constexpr int BK = 64, P = BK + 8;
    extern __shared__ __align__(16) __nv_bfloat16 sm[];
    __nv_bfloat16* Ahi = sm;
    __nv_bfloat16* Alo = Ahi + BM * P;
    __nv_bfloat16* Ws = Alo + BM * P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp / WARPS_N) * 32, wn = (warp % WARPS_N) * WN;
    const int m0 = blockIdx.x * BM;
    const bool vecA = (K % 4) == 0 && (lda % 4) == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0;
    const bool vecW = (K % 8) == 0 && (ldw % 8) == 0 && (reinterpret_cast<uintptr_t>(W) & 15) == 0;
    float acc[2][NT][4] = {};
    for (int k0 = 0; k0 < K; k0 += BK) {
        if (vecA) {
            for (int i = tid; i < BM * (BK / 4); i += 256) {
                const int r = i / (BK / 4), c = 4 * (i % (BK / 4));
                const int m = m0 + r, k = k0 + c;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (m < M && k < K) v = *reinterpret_cast<const float4*>(A + (int64_t)m * lda + k);
                __nv_bfloat16* h = Ahi + r * P + c;
                __nv_bfloat16* l = Alo + r * P + c;
                split_store(h, l, v.x);
                split_store(h + 1, l + 1, v.y);
                split_store(h + 2, l + 2, v.z);
                split_store(h + 3, l + 3, v.w);
            }
        } else {
            for (int i = tid; i < BM * BK; i += 256) {
                const int r = i / BK, c = i % BK;
                const int m = m0 + r, k = k0 + c;
                split_store(Ahi + r * P + c, Alo + r * P + c, (m < M && k < K) ? A[(int64_t)m * lda + k] : 0.f);
            }
        }
        if (vecW) {
            for (int i = tid; i < BN * (BK / 8); i += 256) {
                const int r = i / (BK / 8), c = 8 * (i % (BK / 8));
                const int k = k0 + c;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (r < N && k < K) v = *reinterpret_cast<const uint4*>(W + (int64_t)r * ldw + k);
                *reinterpret_cast<uint4*>(Ws + r * P + c) = v;
            }
        } else {
            for (int i = tid; i < BN * BK; i += 256) {
                const int r = i / BK, c = i % BK;
                const int k = k0 + c;
                Ws[r * P + c] = (r < N && k < K) ? W[(int64_t)r * ldw + k] : __float2bfloat16_rn(0.f);
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t bf[NT][2];
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const __nv_bfloat16* w = Ws + (wn + 8 * j + g) * P + kk + 2 * t;
                bf[j][0] = *reinterpret_cast<const uint32_t*>(w);
                bf[j][1] = *reinterpret_cast<const uint32_t*>(w + 8);
            }
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                const __nv_bfloat16* As = part ? Alo : Ahi;
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const __nv_bfloat16* a = As + (wm + 16 * i + g) * P + kk + 2 * t;
                    const uint32_t af[4] = {*reinterpret_cast<const uint32_t*>(a),
                                            *reinterpret_cast<const uint32_t*>(a + 8 * P),
                                            *reinterpret_cast<const uint32_t*>(a + 8),
                                            *reinterpret_cast<const uint32_t*>(a + 8 * P + 8)};
#pragma unroll
                    for (int j = 0; j < NT; ++j) mma_bf16(acc[i][j], af, bf[j]);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int m = m0 + wm + 16 * i + g + (e >= 2 ? 8 : 0);
                const int n = wn + 8 * j + 2 * t + (e & 1);
                if (m >= M || n >= N) continue;
                float v = acc[i][j][e] + bias[n];
                if (gelu) v = 0.5f * v * (1.f + erff(v * 0.70710678118654752f));
                C[(int64_t)m * ldc + n] = v;
            }
}

template <int BN, int WARPS_N>
constexpr size_t gemm_tc_smem() {
    return sizeof(__nv_bfloat16) * (2 * 32 * (8 / WARPS_N) + BN) * (64 + 8);
}

// dZ = dH * GELU'(Z), GELU'(z) = Phi(z) + z phi(z)
__global__ void gelu_back_kernel(const float* dH, const float* Z, float* dZ, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float z = Z[i];
        const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
        const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
        dZ[i] = dH[i] * (cdf + z * pdf);
    }
}

// column sums: db[n] = sum_m dZ[m][n]
__global__ void colsum_kernel(const float* dZ, int M, int N, float* db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int m = 0; m < M; ++m) s += dZ[(int64_t)m * N + n];
    db[n] = s;
}

// softmax cross-entropy over rows of logits; writes dlogits = (p - onehot) / B and per-row loss.
__global__ void softmax_xent_kernel(const float* logits, const int32_t* y, int B, int L, float* dlogits,
                                    float* row_loss) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B) return;
    const float* z = logits + (int64_t)r * L;
    float mx = -INFINITY;
    for (int l = 0; l < L; ++l) mx = fmaxf(mx, z[l]);
    float s = 0.f;
    for (int l = 0; l < L; ++l) s += expf(z[l] - mx);
    const float lse = mx + logf(s);
    row_loss[r] = lse - z[y[r]];
    for (int l = 0; l < L; ++l) {
        const float pr = expf(z[l] - lse);
        dlogits[(int64_t)r * L + l] = (pr - (l == y[r] ? 1.f : 0.f)) / B;
    }
}

__global__ void adamw_kernel(float* w, const float* g, float* m, float* v, __nv_bfloat16* wb, int64_t n, float lr,
                             float b1, float b2, float eps, float wd, float c1, float c2, int decay) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float wi = w[i];
        if (decay) wi -= lr * wd * wi;
        wi -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void to_bf16_kernel(const float* w, __nv_bfloat16* wb, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

// Features: per cell, (scores - the cell's maximum) / 0.05, clipped below at -8, so that the labels
// within the fine-tune margin of the best fall in [-1, 0]; NaN anywhere marks the cell (bad = 1).
__global__ void features_kernel(const float* scores, int Q, int L, float* X, uint8_t* bad) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    const float* s = scores + (int64_t)q * L;
    float mx = -INFINITY;
    bool nan = false;
    for (int l = 0; l < L; ++l) {
        nan |= s[l] != s[l];
        mx = fmaxf(mx, s[l]);
    }
    for (int l = 0; l < L; ++l) X[(int64_t)q * L + l] = nan ? 0.f : fmaxf((s[l] - mx) * 20.f, -8.f);
    if (bad) bad[q] = nan ? 1 : 0;
}

// argmax and its softmax probability per row
__global__ void predict_kernel(const float* logits, int Q, int L, int32_t* label, float* conf) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    const float* z = logits + (int64_t)q * L;
    int best = 0;
    float mx = z[0];
    for (int l = 1; l < L; ++l)
        if (z[l] > mx) {
            mx = z[l];
            best = l;
        }
    float s = 0.f;
    for (int l = 0; l < L; ++l) s += expf(z[l] - mx);
    label[q] = best;
    conf[q] = 1.f / s;
}

__global__ void gather_rows_kernel(const float* X, const int32_t* yall, const int32_t* idx, int B, int L, float* Xb,
                                   int32_t* yb) {
    const int r = blockIdx.x;
    if (r >= B) return;
    const int src = idx[r];
    for (int l = threadIdx.x; l < L; l += blockDim.x) Xb[(int64_t)r * L + l] = X[(int64_t)src * L + l];
    if (threadIdx.x == 0) yb[r] = yall[src];
}

template <class TA, class TB>
void gemm(int M, int N, int K, const TA* A, int64_t am, int64_t ak, const TB* B, int64_t bk, int64_t bn, float* C,
          int64_t ldc, const float* bias, float* Z, int epi, cudaStream_t s) {
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    gemm_kernel<TA, TB><<<grid, 256, 0, s>>>(M, N, K, A, am, ak, B, bk, bn, C, ldc, bias, Z, epi);
    SGR_LAUNCH_CHECK();
    count_launch();
}

unsigned blocks_for(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16); }

// Per cell: 0 candidates -> final 0; 1 candidate -> that label; otherwise the MLP proposal when it
// is confident, among the candidates, the scores have no NaN and the cell is not in the check
// sample; every other cell goes to the plain list.  role: 0 decided without fine-tune, 1 plain
// (fallback), 2 plain (check sample; its proposal is kept in final_labels for the comparison).
__global__ void learned_route_kernel(int Q, int L, const uint8_t* flags, const uint8_t* bad, const int32_t* prop,
                                     const float* conf, float min_conf, uint32_t check_per_10k, uint64_t seed,
                                     uint64_t row0, int32_t* final_labels, int32_t* plain, int* n_plain,
                                     uint8_t* role) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    const uint8_t* f = flags + (int64_t)q * L;
    int n = 0, only = 0;
    for (int l = 0; l < L; ++l)
        if (f[l]) {
            ++n;
            only = l;
        }
    if (n <= 1) {
        final_labels[q] = n == 1 ? only : 0;
        role[q] = 0;
        return;
    }
    // the check sample is a hash of the cell's row in the whole query (row0: the batch's first row),
    // so that a query annotated in batches checks the same cells as in one call
    uint64_t z = seed ^ (0x9E3779B97F4A7C15ull * (row0 + (uint64_t)q + 1));
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const bool check = (uint32_t)(z % 10000u) < check_per_10k;
    const int p = prop[q];
    const bool ok = !bad[q] && conf[q] >= min_conf && p >= 0 && p < L && f[p];
    if (ok && !check) {
        final_labels[q] = p;
        role[q] = 0;
        return;
    }
    final_labels[q] = ok ? p : -1;
    role[q] = ok ? 2 : 1;
    plain[atomicAdd(n_plain, 1)] = q;
}

}  // namespace

void launch_learned_route(int Q, int L, const uint8_t* flags, const uint8_t* bad, const int32_t* prop,
                          const float* conf, float min_conf, uint32_t check_per_10k, uint64_t seed, uint64_t row0,
                          int32_t* final_labels, int32_t* plain, int* n_plain, uint8_t* role, cudaStream_t s) {
    if (Q <= 0) return;
    learned_route_kernel<<<(Q + 255) / 256, 256, 0, s>>>(Q, L, flags, bad, prop, conf, min_conf, check_per_10k, seed,
                                                         row0, final_labels, plain, n_plain, role);
    SGR_LAUNCH_CHECK();
    count_launch();
}

// ---- host side -------------------------------------------------------------------------------

void Mlp::init(int L_, int H_, uint64_t seed, cudaStream_t s) {
    L = L_;
    H = H_;
    const size_t n1 = (size_t)H * L, n2 = (size_t)H * H, n3 = (size_t)L * H;
    off_w1 = 0;
    off_b1 = off_w1 + n1;
    off_w2 = off_b1 + H;
    off_b2 = off_w2 + n2;
    off_w3 = off_b2 + H;
    off_b3 = off_w3 + n3;
    n_params = off_b3 + L;
    std::vector<float> p(n_params, 0.f);
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
    auto uni = [&]() {  // splitmix64 -> [0, 1)
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](size_t off, size_t n, int fan_in) {
        const double a = 1.0 / std::sqrt((double)fan_in);
        for (size_t i = 0; i < n; ++i) p[off + i] = (float)((2 * uni() - 1) * a);
    };
    fill(off_w1, n1, L);
    fill(off_w2, n2, H);
    fill(off_w3, n3, H);
    set_params(p.data(), s);
    ready = true;
}

void Mlp::set_params(const float* host, cudaStream_t s) {
    w.upload(host, n_params, s);
    wb.ensure(n_params);
    to_bf16_kernel<<<blocks_for(n_params), 256, 0, s>>>(w.p, wb.p, (int64_t)n_params);
    SGR_LAUNCH_CHECK();
    count_launch();
    m.ensure(n_params);
    v.ensure(n_params);
    g.ensure(n_params);
    SGR_CUDA(cudaMemsetAsync(m.p, 0, n_params * sizeof(float), s));
    SGR_CUDA(cudaMemsetAsync(v.p, 0, n_params * sizeof(float), s));
    step = 0;
}

// Forward of B rows of X (device, B x L) into logits (B x L); keeps activations for backward.
void Mlp::forward(const float* X, int B, cudaStream_t s) {
    z1.ensure((size_t)B * H);
    h1.ensure((size_t)B * H);
    z2.ensure((size_t)B * H);
    h2.ensure((size_t)B * H);
    logits.ensure((size_t)B * L);
    const __nv_bfloat16* W = wb.p;
    gemm<float, __nv_bfloat16>(B, H, L, X, L, 1, W + off_w1, 1, L, h1.p, H, w.p + off_b1, z1.p, 2, s);
    gemm<float, __nv_bfloat16>(B, H, H, h1.p, H, 1, W + off_w2, 1, H, h2.p, H, w.p + off_b2, z2.p, 2, s);
    gemm<float, __nv_bfloat16>(B, L, H, h2.p, H, 1, W + off_w3, 1, H, logits.p, L, w.p + off_b3, nullptr, 1, s);
}

// Backward of the mean cross-entropy of the last forward into g (flat, same layout as w).
void Mlp::backward(const float* X, const int32_t* y, int B, cudaStream_t s) {
    dlogits.ensure((size_t)B * L);
    row_loss.ensure(B);
    dh.ensure((size_t)B * H);
    dz.ensure((size_t)B * H);
    softmax_xent_kernel<<<(B + 255) / 256, 256, 0, s>>>(logits.p, y, B, L, dlogits.p, row_loss.p);
    SGR_LAUNCH_CHECK();
    count_launch();
    const __nv_bfloat16* W = wb.p;
    float* G = g.p;
    // layer 3: dW3[L x H] = dlogits^T h2, db3, dh2 = dlogits W3
    gemm<float, float>(L, H, B, dlogits.p, 1, L, h2.p, H, 1, G + off_w3, H, nullptr, nullptr, 0, s);
    colsum_kernel<<<(L + 255) / 256, 256, 0, s>>>(dlogits.p, B, L, G + off_b3);
    count_launch();
    gemm<float, __nv_bfloat16>(B, H, L, dlogits.p, L, 1, W + off_w3, H, 1, dh.p, H, nullptr, nullptr, 0, s);
    gelu_back_kernel<<<blocks_for((int64_t)B * H), 256, 0, s>>>(dh.p, z2.p, dz.p, (int64_t)B * H);
    count_launch();
    // layer 2: dW2[H x H] = dz2^T h1, db2, dh1 = dz2 W2
    gemm<float, float>(H, H, B, dz.p, 1, H, h1.p, H, 1, G + off_w2, H, nullptr, nullptr, 0, s);
    colsum_kernel<<<(H + 255) / 256, 256, 0, s>>>(dz.p, B, H, G + off_b2);
    count_launch();
    gemm<float, __nv_bfloat16>(B, H, H, dz.p, H, 1, W + off_w2, H, 1, dh.p, H, nullptr, nullptr, 0, s);
    gelu_back_kernel<<<blocks_for((int64_t)B * H), 256, 0, s>>>(dh.p, z1.p, dz.p, (int64_t)B * H);
    count_launch();
    // layer 1: dW1[H x L] = dz1^T X, db1
    gemm<float, float>(H, L, B, dz.p, 1, H, X, L, 1, G + off_w1, L, nullptr, nullptr, 0, s);
    colsum_kernel<<<(H + 255) / 256, 256, 0, s>>>(dz.p, B, H, G + off_b1);
    count_launch();
    SGR_LAUNCH_CHECK();
}

void Mlp::adamw(float lr, float b1, float b2, float eps, float wd, cudaStream_t s) {
    ++step;
    const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
    // weights decay, biases do not
    struct Seg {
        size_t off, n;
        int decay;
    } segs[6] = {{off_w1, (size_t)H * L, 1}, {off_b1, (size_t)H, 0}, {off_w2, (size_t)H * H, 1},
                 {off_b2, (size_t)H, 0},     {off_w3, (size_t)L * H, 1}, {off_b3, (size_t)L, 0}};
    for (auto& sg : segs) {
        adamw_kernel<<<blocks_for(sg.n), 256, 0, s>>>(w.p + sg.off, g.p + sg.off, m.p + sg.off, v.p + sg.off,
                                                      wb.p + sg.off, (int64_t)sg.n, lr, b1, b2, eps, wd, c1, c2,
                                                      sg.decay);
        count_launch();
    }
    SGR_LAUNCH_CHECK();
}

void Mlp::features(const float* scores, int Q, float* X, uint8_t* bad, cudaStream_t s) {
    if (Q <= 0) return;
    features_kernel<<<(Q + 255) / 256, 256, 0, s>>>(scores, Q, L, X, bad);
    SGR_LAUNCH_CHECK();
    count_launch();
}

// Inference forward of B rows of X into logits on the tensor cores (no activations kept).
void Mlp::forward_infer(const float* X, int B, cudaStream_t s) {
    h1.ensure((size_t)B * H);
    h2.ensure((size_t)B * H);
    logits.ensure((size_t)B * L);
    const __nv_bfloat16* W = wb.p;
    // one block spans up to 256 output columns (64 rows x 256, or 256 rows x 32 for narrow layers);
    // wider layers take several column blocks
    auto run = [&](int N, int K, const float* A, const __nv_bfloat16* w, const float* b, float* C, int gelu) {
        if (N <= 32) {
            constexpr size_t smem = gemm_tc_smem<32, 1>();
            SGR_CUDA(cudaFuncSetAttribute(gemm_tc_kernel<32, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
            gemm_tc_kernel<32, 1><<<(B + 255) / 256, 256, smem, s>>>(B, N, K, A, K, w, K, b, C, N, gelu);
            SGR_LAUNCH_CHECK();
            count_launch();
            return;
        }
        constexpr size_t smem = gemm_tc_smem<256, 4>();
        SGR_CUDA(cudaFuncSetAttribute(gemm_tc_kernel<256, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        for (int n0 = 0; n0 < N; n0 += 256) {
            gemm_tc_kernel<256, 4><<<(B + 63) / 64, 256, smem, s>>>(B, std::min(256, N - n0), K, A, K,
                                                                     w + (size_t)n0 * K, K, b + n0, C + n0, N,
                                                                     gelu);
            SGR_LAUNCH_CHECK();
            count_launch();
        }
    };
    run(H, L, X, W + off_w1, w.p + off_b1, h1.p, 1);
    run(H, H, h1.p, W + off_w2, w.p + off_b2, h2.p, 1);
    run(L, H, h2.p, W + off_w3, w.p + off_b3, logits.p, 0);
}

void Mlp::predict(const float* X, int Q, int32_t* label, float* conf, cudaStream_t s) {
    const int chunk = 1 << 16;
    for (int q0 = 0; q0 < Q; q0 += chunk) {
        const int n = std::min(chunk, Q - q0);
        forward_infer(X + (size_t)q0 * L, n, s);
        predict_kernel<<<(n + 255) / 256, 256, 0, s>>>(logits.p, n, L, label + q0, conf + q0);
        SGR_LAUNCH_CHECK();
        count_launch();
    }
}

void Mlp::gather(const float* X, const int32_t* y, const int32_t* idx, int B, float* Xb, int32_t* yb, cudaStream_t s) {
    gather_rows_kernel<<<B, 64, 0, s>>>(X, y, idx, B, L, Xb, yb);
    SGR_LAUNCH_CHECK();
    count_launch();
}

}  // namespace sgr
