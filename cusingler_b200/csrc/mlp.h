// Learned-proposal MLP state (weights, optimizer moments, activations) on one device.
#pragma once

#include <cuda_bf16.h>

#include "sgr_internal.h"

namespace sgr {

struct Mlp {
    int L = 0, H = 0;
    bool ready = false;
    size_t off_w1 = 0, off_b1 = 0, off_w2 = 0, off_b2 = 0, off_w3 = 0, off_b3 = 0, n_params = 0;
    int step = 0;
    DevBuf<float> w, g, m, v;       // FP32 master parameters, gradients, AdamW moments
    DevBuf<__nv_bfloat16> wb;       // BF16 working copy used by the products
    DevBuf<float> z1, h1, z2, h2, logits, dlogits, row_loss, dh, dz;

    void init(int L, int H, uint64_t seed, cudaStream_t s);
    void set_params(const float* host, cudaStream_t s);
    void forward(const float* X, int B, cudaStream_t s);
    // Inference forward on the tensor cores (BF16 hi/lo split of the activations); logits only.
    void forward_infer(const float* X, int B, cudaStream_t s);
    void backward(const float* X, const int32_t* y, int B, cudaStream_t s);
    void adamw(float lr, float b1, float b2, float eps, float wd, cudaStream_t s);
    void features(const float* scores, int Q, float* X, uint8_t* bad, cudaStream_t s);
    void predict(const float* X, int Q, int32_t* label, float* conf, cudaStream_t s);
    void gather(const float* X, const int32_t* y, const int32_t* idx, int B, float* Xb, int32_t* yb, cudaStream_t s);
};

// Route cells for the learned form: cells whose proposal is confident, a candidate, and not
// sampled for checking keep the proposal; the rest are appended to `plain` (device list).
void launch_learned_route(int Q, int L, const uint8_t* flags, const uint8_t* bad, const int32_t* prop,
                          const float* conf, float min_conf, uint32_t check_per_10k, uint64_t seed, uint64_t row0,
                          int32_t* final_labels, int32_t* plain, int* n_plain, uint8_t* role, cudaStream_t s);

}  // namespace sgr
