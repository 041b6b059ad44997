// Allocation-free variant of the score-step label selection (per-label quantile, first label,
// candidate flags) for callers that must not allocate device memory.
//
// Who needs it: code that runs while another runtime owns the device memory (a serving process
// whose framework allocates everything from its own pool and budget), code that is being recorded
// into a CUDA graph, or latency-bound code where a cudaMalloc/cudaFree would synchronise the device
// and stall every other stream.  Such callers pass device buffers they already own for the inputs
// and outputs; this entry point itself calls no cudaMalloc, cudaFree or allocating library routine.
//
// The only temporary space the selection needs is a sort buffer for score lists that hold NaN
// (constant rows).  It lives in one file-scope device array of kNoallocScratchFloats floats
// (1,048,576 floats, 4 MiB) that every GPU loading this library holds until the process exits.  Host code cannot pass
// the array's name to a kernel (in host code it is only a stand-in, not a device address), so the
// first call on each device looks its address up with cudaGetSymbolAddress, with that device
// current, and caches it.

#include <algorithm>
#include <mutex>

#include "device_util.cuh"
#include "kernels.cuh"
#include "sgr_internal.h"

namespace sgr {
namespace {

constexpr int kNoallocScratchFloats = 1 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_noalloc_scratch[kNoallocScratchFloats];

struct LabelTable {
    LabelQ q[256];
};

__global__ void __launch_bounds__(256) select_noalloc_kernel(const float* scores, int64_t ld, int nq, int L,
                                                             const __grid_constant__ LabelTable lt, float p,
                                                             float thre, float* label_scores, int32_t* first,
                                                             uint8_t* flags, float* scratch, int spw) {
    __shared__ float ls[256];
    __shared__ int hist[8][256];
    __shared__ int s_mx;
    // Status bits of the selection are not reported by this entry point: it only enqueues work and
    // has no context to return them through.  Bit 8 (no sort scratch) cannot arise, the scratch is
    // always present; bit 4 (a NaN-bearing list on which libstdc++ would read outside the array,
    // sorted within bounds instead) is not reported by the main path either.
    __shared__ int ignored_status;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) ignored_status = 0;
    __syncthreads();
    float* my_scratch = scratch + (size_t)(blockIdx.x * 8 + warp) * spw;
    for (int q = blockIdx.x; q < nq; q += gridDim.x) {
        const float* row = scores + (size_t)q * ld;
        for (int l = warp; l < L; l += 8) {
            const LabelQ d = lt.q[l];
            // a constant query row makes every score NaN: the quantile of an all-NaN list is NaN for
            // every grid position, so such lists skip the sort (checked only when the first score is NaN)
            bool all_nan = false;
            if (row[d.start] != row[d.start]) {
                bool any = false;
                for (int i = lane; i < d.len; i += 32) any |= row[d.start + i] == row[d.start + i];
                all_nan = !__any_sync(0xffffffffu, any);
            }
            const float r = all_nan ? __int_as_float(0x7fffffff)
                                    : quantile_warp(row + d.start, d, p, hist[warp], my_scratch, lane, &ignored_status);
            if (lane == 0) ls[l] = r;
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

std::mutex g_mu;
float* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per device).
float* scratch_address(int dev) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        float* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            fail(SGR_ERR_CUDA, std::string("cudaGetSymbolAddress of the selection scratch: ") + cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = p;
    }
    return g_scratch_ptr[dev];
}

}  // namespace

}  // namespace sgr

extern "C" sgr_status sgr_select_labels_noalloc(const float* d_scores, int64_t ld, uint32_t n_rows,
                                                const uint32_t* label_ranges, uint32_t n_labels, float quantile,
                                                float finetune_thre, float* d_label_scores,
                                                int32_t* d_first_labels, uint8_t* d_flags, void* stream) {
    using namespace sgr;
    if (n_rows == 0) return SGR_OK;
    if (!d_scores || !label_ranges || !d_label_scores || !d_first_labels) return SGR_ERR_INVALID_ARGUMENT;
    if (n_labels == 0 || n_labels > 256) return SGR_ERR_UNSUPPORTED;
    LabelTable lt{};
    uint32_t max_len = 1;
    for (uint32_t l = 0; l < n_labels; ++l) {
        const uint32_t start = label_ranges[2 * l], len = label_ranges[2 * l + 1];
        if (len == 0) return SGR_ERR_EMPTY_LABEL;
        if ((uint64_t)start + len > (uint64_t)ld) return SGR_ERR_INVALID_ARGUMENT;
        max_len = std::max(max_len, len);
        // the reference's float index grid (src/cusingler.cu:947-978 of STOmics/cusingler)
        lt.q[l] = make_lq((int)start, (int)len, quantile);
    }
    // eight warps per block, each with its own max_len-float slice of the fixed scratch array
    const long fit_blocks = (long)kNoallocScratchFloats / (8L * max_len);
    if (fit_blocks < 1) return SGR_ERR_UNSUPPORTED;  // a label with more than 131072 reference cells
    try {
        int dev = 0;
        SGR_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kMaxDevices) return SGR_ERR_UNSUPPORTED;
        float* scratch = scratch_address(dev);
        const unsigned blocks =
            (unsigned)std::min<long>({(long)n_rows, fit_blocks, (long)device_sm_count() * 2});
        select_noalloc_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(
            d_scores, ld, (int)n_rows, (int)n_labels, lt, quantile, finetune_thre, d_label_scores, d_first_labels,
            d_flags, scratch, (int)max_len);
        SGR_CUDA(cudaGetLastError());
        count_launch();
    } catch (const Error& e) {
        return e.code;
    }
    return SGR_OK;
}
