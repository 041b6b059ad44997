// Internal declarations shared by the host and device sources of libsgr.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sgr.h"

namespace sgr {

struct Error : std::runtime_error {
    sgr_status code;
    Error(sgr_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(sgr_status c, const std::string& m) { throw Error(c, m); }

#define SGR_CUDA(call)                                                                                   \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            if (e_ == cudaErrorMemoryAllocation) {                                                       \
                cudaGetLastError();                                                                      \
                ::sgr::fail(SGR_ERR_OUT_OF_MEMORY, std::string(#call) + ": " + cudaGetErrorString(e_));  \
            }                                                                                            \
            ::sgr::fail(SGR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + " (" +        \
                                          __FILE__ + ":" + std::to_string(__LINE__) + ")");              \
        }                                                                                                \
    } while (0)

#define SGR_LAUNCH_CHECK() SGR_CUDA(cudaGetLastError())

// Owning device buffer (cudaMalloc'ed, grows, never shrinks unless freed).
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    T* ensure(size_t count) {
        if (count > n) {
            release();
            size_t bytes = (count ? count : 1) * sizeof(T);
            SGR_CUDA(cudaMalloc(reinterpret_cast<void**>(&p), bytes));
            n = count;
        }
        return p;
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        ensure(count);
        if (count) SGR_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), h.size(), s); }
};

// ---- host marker training (train.cpp) ---------------------------------------------------------

struct HostCsr {
    uint32_t n_rows = 0, n_cols = 0;
    const float* data = nullptr;
    const int32_t* indices = nullptr;
    const int32_t* indptr = nullptr;
};

struct Markers {
    uint32_t n_labels = 0;
    uint32_t W = 0;                    // gene space = reference column count as given
    bool filter_genes = false;
    std::vector<int32_t> ref_colmap;   // reference column -> gene id (identity or intersection rank)
    std::vector<int32_t> qry_colmap;   // query column -> gene id, -1 when dropped
    std::vector<uint32_t> ref_order;   // regrouped row -> original reference row
    std::vector<uint32_t> ctidx;       // (start, len) per label in the regrouped reference
    std::vector<uint32_t> common;      // score-step marker genes, ascending
    std::vector<uint32_t> thre;        // fine-tune gene pool, ascending
    std::vector<uint32_t> pair_genes;  // positive-difference genes per ordered pair, concatenated
    std::vector<uint32_t> pair_idx;    // (start, len) per ordered pair, diagonal (0, 0)
    std::vector<uint32_t> ft_genes;    // pair lists restricted to thre, as thre-compact ids
    std::vector<uint32_t> ft_idx;      // (start, len) per ordered pair
};

// Gene-name intersection, label regrouping and marker training on the host (see train.cpp):
// prepare_markers (intersection, regrouping: colmaps, ref_order, ctidx) then rank_markers_host
// (medians, per-pair lists, gene sets).
void train_markers(const HostCsr& ref, const int32_t* celltypes, uint32_t n_labels,
                   const char* const* ref_genes, const char* const* qry_genes, uint32_t n_qry_genes,
                   int cores, Markers& out);
void prepare_markers(const HostCsr& ref, const int32_t* celltypes, uint32_t n_labels,
                     const char* const* ref_genes, const char* const* qry_genes, uint32_t n_qry_genes, Markers& m);
void rank_markers_host(const HostCsr& ref, int cores, Markers& m);
// From pair_genes / pair_idx and the score-step and fine-tune gene flags (W each): the gene sets
// common and thre and the fine-tune pair lists.
void finish_markers(Markers& m, const uint8_t* in_common, const uint8_t* in_thre);
// The medians and per-pair lists on the device (train_gpu.cu) from the label-grouped reference CSR
// in device memory (rows in m.ref_order order, original columns); fills pair_genes, pair_idx and,
// through finish_markers, the gene sets.
void rank_markers_device(const float* data, const int32_t* indices, const int32_t* indptr, uint32_t R,
                         uint32_t ref_cols, int64_t nnz, Markers& m, cudaStream_t s);

// Reference's marker-count formula round(500 * (2/3)^log2(n)) (src/io.cpp:209,
// src/cusingler.cu:1142).
int marker_count(size_t n_labels);

}  // namespace sgr
