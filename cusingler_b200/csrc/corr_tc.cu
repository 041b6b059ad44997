// Score-step rank correlation on the 5th-generation tensor cores (tcgen05, kind::i8), exact.
//
// The reference computes every (query, reference) Spearman correlation with one FP32 fused
// multiply-add chain per pair on CUDA cores (spearman, src/cusingler.cu:918-945 of
// STOmics/cusingler).  Doubled centred ranks d = 2*rank - (G+1) are integers with |d| < G, so the
// numerator N = sum_g d_q d_r is computed exactly here from int8 limbs (split_limbs): planes
// P0 | L | S with d = m * p0 + s, written by the rank kernel (3 * Kp bytes per row, Kp a multiple
// of 128, one TMA tensor map per operand over all three planes).  Then
//     score = float((N * (1/sqrt(n_q))) * (1/sqrt(n_r)))   (FP64); a zero norm has a NaN
//             reciprocal, so the score of a constant row is NaN as in the reference.
// Three forms of the exact product (all bit-identical):
//   corr_wide_hold_kernel (default) and corr_wide_kernel<8|16>: 128 x 256 tiles, two-accumulator
//       split d = C h + l, C = w^2 + 1: A1 = P0.P0' + S.S', A2 = L.L', N = C A1 - (C - 1) A2;
//   corr_tc_kernel: 128 x 160 tiles, three accumulators P1 = P0.P0', P3 = S.S', P2 = L.L',
//       N = C (k1 P1 + P3) - (C - 1) P2 with (k1, C) = (127, 128) for the base-128 split
//       d = 128 h + l and (1, w^2 + 1) for the two-accumulator one;
//   its SM-pair form (PAIR), and an FP16-operand variant of the 128 x 160 and 128 x 256 tiles.
//
// corr_tc_kernel: per tile the K loop runs plane by plane in the order P0, S, L into three TMEM
// accumulators of BN = 160 columns (P1, P3, P2; 480 of 512 columns).

// Structure: persistent kernel, one CTA per SM, 384 threads:
//   warp 0      TMA producer (128 x 128-byte A boxes, 160 x 128-byte B boxes, 128B swizzle,
//               STAGES-deep ring)
//   warp 1      TMEM allocator and single-thread tcgen05.mma issuer (M = 128, N = 160, K = 32)
//   warps 4..11 epilogue, two warps per TMEM lane quadrant (warp % 4), one column half each:
//               tcgen05.ld 32x32b of P1 and P3 into T = k1 P1 + P3 (registers), release of those
//               two accumulators (the next tile's P0 and S planes may start), then P2, the exact
//               recombination, scores into a 128 x 160 staging tile in shared memory, release of
//               P2, and row-contiguous 16-byte stores from the staging tile; with LabelExtremes it
//               also keeps each (query, label) list's min / max for the selection
// A second instantiation (F16) is the FP16-operand variant benchmarked beside the exact one: d as
// IEEE half (exact for |d| <= 2048), one kind::f16 accumulator with FP32 sums (not exact).
// A third (PAIR) runs the exact product on SM pairs: a cluster of two CTAs issues
// tcgen05.mma.cta_group::2 with M = 256 (each CTA holds 128 query rows of A and 80 of the tile's 160
// reference rows of B, and receives its 128 x 160 accumulators in its own TMEM).  Per SM the MMA
// then reads A and half of B from shared memory, so each SM's TMA writes and MMA operand reads per
// tile drop from 995 KB to 718 KB.  The leader CTA (rank 0) issues the MMAs; both CTAs' TMA loads
// signal the leader's stage barriers, each MMA commit arrives on the matching barrier of both CTAs
// (one commit per CTA), and both CTAs' epilogues release the accumulators on the leader's barriers.
// Tiles are visited in groups of `gm` row bands (band fastest), so that the CTAs working at the
// same time share a few bands of A and a slab of B in L2 instead of streaming all of B per band.
// No TMA multicast is used.  Every mbarrier wait is bounded: on timeout the kernel records
// SGR_TC_TIMEOUT in *status, drains its own TMA copies (bounded), frees TMEM and returns.

#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdint>

#include "kernels.cuh"
#include "sgr_internal.h"

namespace sgr {
namespace {

constexpr int BM = 128;
constexpr int BN = 160;  // 3 x 160 accumulator columns fit TMEM's 512
constexpr int HALF = BN / 2;       // columns per epilogue warp
constexpr int CH = HALF / 16;      // 16-column TMEM chunks per epilogue warp
constexpr int BK = 128;  // bytes of K per stage (one 128-byte swizzle row)
constexpr int STAGES = 5;
constexpr int A_BYTES = BM * BK;
constexpr int B_BYTES = BN * BK;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int TMEM_COLS = 512;
constexpr int EPI_WARPS = 8;                // warps 4 .. 11
constexpr int THREADS = 32 * (4 + EPI_WARPS);
// per epilogue warp, one 32-row x 16-column chunk of scores on its way to global memory
constexpr int CHUNK_BYTES = 32 * 16 * 4;
constexpr int STAGING_BYTES = EPI_WARPS * CHUNK_BYTES;
// SM-pair form: per CTA 128 rows of A and BN / 2 rows of B per stage
constexpr int B_HALF_BYTES = (BN / 2) * BK;
constexpr int PAIR_STAGE_BYTES = A_BYTES + B_HALF_BYTES;  // 26 KB, a multiple of 1024
constexpr int PAIR_STAGES = 7;
constexpr int MAX_STAGES = PAIR_STAGES > STAGES ? PAIR_STAGES : STAGES;
static_assert(PAIR_STAGE_BYTES % 1024 == 0, "stage buffers must keep 1024-byte alignment");
constexpr long long WAIT_CYCLES = 4000000000LL;  // about 2 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// try_wait with cluster-scope acquire (phases completed by the peer CTA's arrivals)
__device__ __forceinline__ bool mbar_try_cluster(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; false on timeout (or when another role already gave up).
template <bool CLUSTER = false>
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    const long long t0 = clock64();
    for (uint32_t i = 0;; ++i) {
        if (CLUSTER ? mbar_try_cluster(bar, parity) : mbar_try(bar, parity)) return true;
        if ((i & 63) == 63) {
            if (*abort_flag) return false;
            if (clock64() - t0 > WAIT_CYCLES) return false;
        }
    }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Arrival on a barrier given by its shared::cluster address (this CTA's or the peer's).
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t cluster_id_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t n_clusters_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}

// shared::cluster address of the variable at shared::cta address `addr` in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t mapa(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// L2 policy: keep the lines of a reused operand over streaming data
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_load_2d_hint(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar,
                                                 uint64_t policy) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, %3}], "
        "[%4], %5;" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar), "l"(policy)
        : "memory");
}

// Load into this CTA's shared memory whose completion is counted on a barrier of either CTA of the
// pair (bar: shared::cluster address).  No multicast.
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar,
                                                 uint64_t policy) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], "
        "[%1, {%2, %3}], [%4], %5;" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar), "l"(policy)
        : "memory");
}

// K-major operand tile in shared memory with 128-byte swizzle: rows of 128 bytes, 8-row groups
// 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::i8 instruction descriptor: S32 accumulator, signed A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// kind::f16 instruction descriptor: F32 accumulator, F16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N) {
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_c, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_c),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_c, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_c),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_i8_pair(uint32_t tmem_c, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}" ::"r"(tmem_c),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0), "r"(0));
}

// Completion of this thread's earlier MMAs arrives on the barrier at shared::cluster address `bar`
// (a barrier of either CTA of the pair); one commit per barrier.
__device__ __forceinline__ void umma_commit_pair(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// Order key of a float (unsigned compare = float compare for non-NaN values).
__device__ __forceinline__ uint32_t ord_key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

struct __align__(8) TcShared {
    uint64_t full[MAX_STAGES];
    uint64_t empty[MAX_STAGES];
    uint64_t acc_full[3];   // accumulator region g (P1, P3, P2; the F16 one is 0) holds its plane's sums
    uint64_t acc_empty[3];  // ... and has been read by every epilogue warp
    uint64_t drain;
    uint32_t tmem_base;
    int abort_flag;
};

// Tile t of the visiting order -> (row band, column tile): groups of `gm` bands, band fastest.
__device__ __forceinline__ void tile_coords(int t, int tiles_m, int tiles_n, int gm, int& mb, int& nb) {
    const int group = gm * tiles_n;
    const int g = t / group, first = g * gm;
    const int gme = min(gm, tiles_m - first);
    const int local = t - g * group;
    mb = first + local % gme;
    nb = local / gme;
}

// F16: the FP16-operand variant -- one plane of d as half (2 * Kp bytes per row), kind::f16 with
// FP32 accumulation into one accumulator, score = float((acc * 1/sqrt(n_q)) * 1/sqrt(n_r)).
// PAIR: the exact product on a cluster of two CTAs (tcgen05 cta_group::2, M = 256).
template <bool F16, bool PAIR>
__global__ void __launch_bounds__(THREADS, 1)
    corr_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int nq, int R,
                   int Kp, const double* __restrict__ rq, const double* __restrict__ rr,
                   const int64_t* __restrict__ nq2, const int64_t* __restrict__ nr2, float* __restrict__ out,
                   int64_t ld, int* status, LabelExtremes ext, int gm, int k1, int cbase) {
    static_assert(!(F16 && PAIR), "the SM-pair form is exact only");
    constexpr int NST = PAIR ? PAIR_STAGES : STAGES;
    constexpr int SBYTES = PAIR ? PAIR_STAGE_BYTES : STAGE_BYTES;
    constexpr int MT = PAIR ? 2 * BM : BM;  // query rows of a tile
    constexpr int NEPI = PAIR ? 2 * EPI_WARPS : EPI_WARPS;  // epilogue warps releasing an accumulator
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ TcShared sh;
    // stage buffers must start on a 1024-byte boundary (128B swizzle atoms)
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = PAIR ? cluster_rank() : 0;
    const int unit = PAIR ? (int)cluster_id_x() : (int)blockIdx.x;        // this CTA's (pair's) tile stream
    const int n_units = PAIR ? (int)n_clusters_x() : (int)gridDim.x;
    const int tiles_n = (R + BN - 1) / BN, tiles_m = (nq + MT - 1) / MT;
    const int n_tiles = tiles_m * tiles_n;
    const int kblocks = (F16 ? 2 : 3) * Kp / BK, seg_blocks = F16 ? kblocks : Kp / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < NST; ++s) {
            mbar_init(smem_u32(&sh.full[s]), 1);
            mbar_init(smem_u32(&sh.empty[s]), 1);
        }
        for (int g = 0; g < 3; ++g) {
            mbar_init(smem_u32(&sh.acc_full[g]), 1);
            mbar_init(smem_u32(&sh.acc_empty[g]), NEPI);
        }
        mbar_init(smem_u32(&sh.drain), 1);
        sh.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        if (PAIR) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             smem_u32(&sh.tmem_base)),
                         "r"(TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             smem_u32(&sh.tmem_base)),
                         "r"(TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
    }
    __syncthreads();
    if (PAIR) cluster_sync();  // both CTAs' barriers are initialised before either signals the other's
    tc_fence_after();
    const uint32_t tmem = sh.tmem_base;
    volatile int* abort_flag = &sh.abort_flag;
    // gives up this CTA's waits and, in a pair, the peer's
    auto give_up = [&]() {
        atomicOr(status, SGR_TC_TIMEOUT);
        sh.abort_flag = 1;
        if (PAIR)
            asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(mapa(smem_u32(&sh.abort_flag), rank ^ 1u)), "r"(1)
                         : "memory");
    };

    if (warp == 0) {
        // ---- TMA producer ------------------------------------------------------------------
        if (lane == 0) {
            const uint64_t keep = policy_evict_last();  // the reference operand is read by every band
            uint32_t it = 0;
            bool ok = true;
            for (int t = unit; t < n_tiles && ok; t += n_units) {
                int mb, nb;
                tile_coords(t, tiles_m, tiles_n, gm, mb, nb);
                const int m0 = mb * MT + (PAIR ? BM * (int)rank : 0);
                const int n0 = nb * BN + (PAIR ? (BN / 2) * (int)rank : 0);
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    const int s = it % NST;
                    const uint32_t ph = (it / NST) & 1;
                    if (!mbar_wait<PAIR>(smem_u32(&sh.empty[s]), ph ^ 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint32_t a_dst = smem_u32(smem + s * SBYTES);
                    const uint32_t b_dst = a_dst + A_BYTES;
                    // planes in the order H, S, L (the MMA's accumulator order)
                    const int grp = kb / seg_blocks, seg = F16 ? 0 : (grp == 0 ? 0 : (grp == 1 ? 2 : 1));
                    const int kx = F16 ? kb * BK : (seg * seg_blocks + kb % seg_blocks) * BK;
                    if (PAIR) {
                        // both CTAs' copies complete on the leader's stage barrier
                        const uint32_t fb = mapa(smem_u32(&sh.full[s]), 0);
                        if (rank == 0) mbar_expect_tx(smem_u32(&sh.full[s]), 2 * PAIR_STAGE_BYTES);
                        tma_load_2d_pair(a_dst, &tmA, kx, m0, fb, keep);
                        tma_load_2d_pair(b_dst, &tmB, kx, n0, fb, keep);
                    } else {
                        const uint32_t fb = smem_u32(&sh.full[s]);
                        mbar_expect_tx(fb, STAGE_BYTES);
                        tma_load_2d(a_dst, &tmA, kx, m0, fb);
                        tma_load_2d_hint(b_dst, &tmB, kx, n0, fb, keep);
                    }
                }
            }
            if (!ok) give_up();
            // drain: every issued stage's copies land before the CTA can exit (in a pair the leader
            // sees both CTAs' copies on its barriers; both CTAs leave only through the final cluster
            // barrier)
            if (!PAIR || rank == 0)
                for (uint32_t j = (it > (uint32_t)NST ? it - NST : 0); j < it; ++j) {
                    const uint32_t s = j % NST, ph = (j / NST) & 1;
                    const long long t0 = clock64();
                    while (!mbar_try(smem_u32(&sh.full[s]), ph) && clock64() - t0 < WAIT_CYCLES) {
                    }
                }
        }
    } else if (warp == 1) {
        // ---- MMA issuer (the leader CTA of a pair) ---------------------------------------------
        if (lane == 0 && rank == 0) {
            constexpr uint32_t idesc = F16 ? idesc_f16(BM, BN) : idesc_i8(MT, BN);
            uint32_t it = 0, tile_iter = 0;
            bool ok = true;
            // arrival on a barrier of both CTAs (pair) or this CTA
            auto commit = [&](uint64_t* bar) {
                if (PAIR) {
                    umma_commit_pair(mapa(smem_u32(bar), 0));
                    umma_commit_pair(mapa(smem_u32(bar), 1));
                } else {
                    umma_commit(smem_u32(bar));
                }
            };
            for (int t = unit; t < n_tiles && ok; t += n_units, ++tile_iter) {
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    // groups of k-blocks: H plane -> P1 (region 0), S plane -> P3 (region 1),
                    // L plane -> P2 (region 2); a region is written once the previous tile's epilogue
                    // has read it, and signalled as soon as its plane is done, so the epilogue drains
                    // P1 and P3 while the later planes are still being multiplied
                    const int grp = kb / seg_blocks;
                    const bool first = (kb % seg_blocks) == 0;
                    if (first) {
                        if (!mbar_wait<PAIR>(smem_u32(&sh.acc_empty[grp]), (tile_iter & 1) ^ 1, abort_flag)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                    }
                    const int s = it % NST;
                    const uint32_t ph = (it / NST) & 1;
                    if (!mbar_wait<PAIR>(smem_u32(&sh.full[s]), ph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(smem + s * SBYTES);
                    const uint64_t da = smem_desc(a_addr), db = smem_desc(a_addr + A_BYTES);
                    const uint32_t tc = tmem + grp * BN;
#pragma unroll
                    for (int k = 0; k < BK / 32; ++k) {  // 32 bytes of K per MMA (32 int8 or 16 half)
                        const uint32_t acc = (first && k == 0) ? 0u : 1u;
                        if (F16)
                            umma_f16(tc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc, acc);
                        else if (PAIR)
                            umma_i8_pair(tc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc, acc);
                        else
                            umma_i8(tc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc, acc);
                    }
                    commit(&sh.empty[s]);
                    if (kb % seg_blocks == seg_blocks - 1) commit(&sh.acc_full[grp]);
                }
                if (!ok) break;
            }
            if (!ok) give_up();
            // every MMA this thread issued has finished before TMEM is freed (in both CTAs of a pair)
            commit(&sh.drain);
        }
        if (lane == 0) {
            const long long t0 = clock64();
            while (!mbar_try_cluster(smem_u32(&sh.drain), 0) && clock64() - t0 < WAIT_CYCLES) {
            }
        }
    } else if (warp >= 4) {
        // ---- epilogue ------------------------------------------------------------------------
        // Lane = tile row (32 * quarter + lane); this warp scores its 80 columns in chunks of 16.
        // Each chunk goes through the warp's 32 x 16 staging buffer: lane r writes row r's four
        // 16-byte pieces at position u ^ ((r >> 1) & 3) (conflict-free), and the warp then stores
        // 8 rows x 64 contiguous bytes per instruction.
        const int quarter = warp & 3, half = (warp - 4) >> 2;
        float4* chunk = reinterpret_cast<float4*>(smem + NST * SBYTES + (warp - 4) * CHUNK_BYTES);
        const bool vec_store = (ld % 4) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
        const int row = 32 * quarter + lane;
        // the accumulators are released on the leader's barriers (this CTA's own when alone)
        auto release = [&](int g) {
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                if (PAIR) mbar_arrive_cluster(mapa(smem_u32(&sh.acc_empty[g]), 0));
                else mbar_arrive(smem_u32(&sh.acc_empty[g]));
            }
        };
        auto acquire = [&](int g, uint32_t parity) {
            const bool got = __all_sync(0xffffffffu, mbar_wait<PAIR>(smem_u32(&sh.acc_full[g]), parity, abort_flag));
            if (got) tc_fence_after();
            return got;
        };
        uint32_t tile_iter = 0;
        for (int t = unit; t < n_tiles; t += n_units, ++tile_iter) {
            int mb, nb;
            tile_coords(t, tiles_m, tiles_n, gm, mb, nb);
            const int m0 = mb * MT + (PAIR ? BM * (int)rank : 0), n0 = nb * BN;
            // norms of this tile's rows and columns, loaded while the accumulator is still being computed
            const int q = m0 + row;
            const double rqv = q < nq ? rq[q] : 0.0;  // NaN when the query row is constant
            double rrv[CH];
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const int r = n0 + half * HALF + c * 16 + lane;
                rrv[c] = (lane < 16 && r < R) ? rr[r] : 0.0;  // NaN for a constant reference row
            }
            const uint32_t par = tile_iter & 1;
            const uint32_t lane_base = tmem + ((uint32_t)(32 * quarter) << 16);
            // phase 1: T = 127 P1 + P3 for this warp's columns; P1 is released as soon as it is read,
            // P3 likewise, while the MMA works on the later planes
            int T[CH][16];
            bool got = true;
            if (!F16) {
                got = acquire(0, par);
                if (got) {
#pragma unroll
                    for (int c = 0; c < CH; ++c) {
                        uint32_t pa[16];
                        tmem_ld16(lane_base + half * HALF + c * 16, pa);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 16; ++j) T[c][j] = k1 * (int)pa[j];
                    }
                    release(0);
                    got = acquire(1, par);
                }
                if (got) {
#pragma unroll
                    for (int c = 0; c < CH; ++c) {
                        uint32_t pb[16];
                        tmem_ld16(lane_base + BN + half * HALF + c * 16, pb);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 16; ++j) T[c][j] += (int)pb[j];
                    }
                    release(1);
                }
            }
            if (got) got = acquire(F16 ? 0 : 2, par);
            if (!got) {
                if (lane == 0) give_up();
                break;
            }
            // per-(query, label) extremes of this warp's columns, flushed at label ends (labels are
            // column ranges, the same for every lane, so the flushes are warp-uniform)
            int lab = 0, lab_end = 0;
            float mnf = __int_as_float(0x7f800000), mxf = -__int_as_float(0x7f800000);
            bool seen = false;
            if (ext.kmin) {
                const int cb = n0 + half * HALF;
                int lo = 0, hi = ext.L - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (__ldg(ext.lstart + mid) <= cb) lo = mid;
                    else hi = mid - 1;
                }
                lab = lo;
                lab_end = __ldg(ext.lstart + lab + 1);
            }
            // phase 2: P2 (the F16 accumulator), reads one chunk ahead of the arithmetic; each chunk of
            // scores is staged and stored before the next
            const uint32_t base2 = lane_base + (F16 ? 0 : 2 * BN);
            constexpr int last_region = F16 ? 0 : 2;
            uint32_t p2[2][16];
            tmem_ld16(base2 + half * HALF, p2[0]);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const int col0 = half * HALF + c * 16;
                if (c + 1 < CH) tmem_ld16(base2 + col0 + 16, p2[(c + 1) & 1]);
                float v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const double N = F16 ? (double)__uint_as_float(p2[c & 1][j])
                                         : (double)((int64_t)cbase * T[c][j] -
                                                    (int64_t)(cbase - 1) * (int)p2[c & 1][j]);
                    const double rrj = __shfl_sync(0xffffffffu, rrv[c], j);
                    v[j] = (float)((N * rqv) * rrj);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    chunk[lane * 4 + (u ^ ((lane >> 1) & 3))] =
                        make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
                if (ext.kmin && n0 + col0 + 16 <= min(lab_end, R)) {  // the chunk lies in one label
                    float a0 = fminf(fminf(v[0], v[1]), fminf(v[2], v[3]));
                    float b0 = fmaxf(fmaxf(v[0], v[1]), fmaxf(v[2], v[3]));
#pragma unroll
                    for (int j = 4; j < 16; j += 4) {
                        a0 = fminf(a0, fminf(fminf(v[j], v[j + 1]), fminf(v[j + 2], v[j + 3])));
                        b0 = fmaxf(b0, fmaxf(fmaxf(v[j], v[j + 1]), fmaxf(v[j + 2], v[j + 3])));
                    }
                    mnf = fminf(mnf, a0);
                    mxf = fmaxf(mxf, b0);
                    seen = true;
                } else if (ext.kmin) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int col = n0 + col0 + j;
                        if (col >= R) break;
                        if (col >= lab_end) {  // label boundary
                            if (seen && q < nq) {
                                atomicMin(ext.kmin + (size_t)q * ext.L + lab, ord_key(mnf));
                                atomicMax(ext.kmax + (size_t)q * ext.L + lab, ord_key(mxf));
                            }
                            mnf = __int_as_float(0x7f800000);
                            mxf = -__int_as_float(0x7f800000);
                            do {
                                ++lab;
                                lab_end = __ldg(ext.lstart + lab + 1);
                            } while (col >= lab_end);
                        }
                        mnf = fminf(mnf, v[j]);
                        mxf = fmaxf(mxf, v[j]);
                        seen = true;
                    }
                }
                if (c + 1 < CH) tmem_wait_ld();
                else release(last_region);  // all of this warp's TMEM reads are done
                // the chunk's 32 rows x 16 columns: lane l stores piece l % 4 of row l / 4 (+ 8 i)
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = 8 * i + (lane >> 2), u = lane & 3;
                    const int qq = m0 + 32 * quarter + r, col = n0 + col0 + 4 * u;
                    const float4 val = chunk[r * 4 + (u ^ ((r >> 1) & 3))];
                    if (qq >= nq || col >= R) continue;
                    float* dst = out + (size_t)qq * ld + col;
                    // streaming stores (evict first): the scores are read once, later, and must not
                    // push the reference operand out of L2
                    if (vec_store && col + 3 < R) {
                        __stcs(reinterpret_cast<float4*>(dst), val);
                    } else {
                        __stcs(dst, val.x);
                        if (col + 1 < R) __stcs(dst + 1, val.y);
                        if (col + 2 < R) __stcs(dst + 2, val.z);
                        if (col + 3 < R) __stcs(dst + 3, val.w);
                    }
                }
                __syncwarp();  // the next chunk may overwrite the staging buffer
            }
            if (ext.kmin && seen && q < nq) {
                atomicMin(ext.kmin + (size_t)q * ext.L + lab, ord_key(mnf));
                atomicMax(ext.kmax + (size_t)q * ext.L + lab, ord_key(mxf));
            }
        }
    }
    __syncthreads();
    // a pair leaves together: no CTA exits while the other may still signal its barriers or read its
    // shared memory through the MMA
    if (PAIR) cluster_sync();
    if (warp == 1) {
        tc_fence_after();
        if (PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
        else
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ---- wide form: 128 x 256 tiles, two accumulators ----------------------------------------------
//
// With the split d = C h + l, C = w^2 + 1 (split_limbs with w > 0; planes P0 = w h, L = l, S = h + l):
//     A1 = P0_q . P0_r + S_q . S_r,   A2 = L_q . L_r,   N = C A1 - (C - 1) A2   (exact in int64).
// The two 256-column accumulators fill TMEM's 512 columns, so every tcgen05.mma has N = 256: the
// time of one M = 128, K = 32 instruction measured the same at N = 128, 160 and 256, so this tile
// gets the most products out of each.  Per tile the K loop multiplies the P0 and S planes into A1,
// then the L plane into A2.  No second accumulator set fits, so the epilogue's walk over the tile
// (TMEM loads one 16-column chunk ahead of the arithmetic) holds up the next tile's MMAs until its
// last loads; EW epilogue warps (8 or 16: two or four per TMEM lane quadrant) shorten that walk.
constexpr int WBN = 256;
constexpr int WSTAGES = 4;
constexpr int WSTAGE_BYTES = A_BYTES + WBN * BK;  // 48 KB, a multiple of 1024
static_assert(WSTAGES <= MAX_STAGES, "barrier arrays");

template <int EW>
__global__ void __launch_bounds__(32 * (4 + EW), 1)
    corr_wide_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int nq, int R,
                     int Kp, const double* __restrict__ rq, const double* __restrict__ rr, float* __restrict__ out,
                     int64_t ld, int* status, LabelExtremes ext, int gm, int cbase) {
    constexpr int QW = EW / 4;         // epilogue warps per TMEM lane quadrant
    constexpr int WCOLS = WBN / QW;    // columns per epilogue warp
    constexpr int WCH = WCOLS / 16;    // 16-column chunks per epilogue warp
    static_assert(EW == 8 || EW == 16, "two or four epilogue warps per lane quadrant");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ TcShared sh;
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_n = (R + WBN - 1) / WBN, tiles_m = (nq + BM - 1) / BM;
    const int n_tiles = tiles_m * tiles_n;
    const int segb = Kp / BK, kblocks = 3 * segb;

    if (threadIdx.x == 0) {
        for (int s = 0; s < WSTAGES; ++s) {
            mbar_init(smem_u32(&sh.full[s]), 1);
            mbar_init(smem_u32(&sh.empty[s]), 1);
        }
        for (int g = 0; g < 2; ++g) {
            mbar_init(smem_u32(&sh.acc_full[g]), 1);
            mbar_init(smem_u32(&sh.acc_empty[g]), EW);
        }
        mbar_init(smem_u32(&sh.drain), 1);
        sh.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh.tmem_base)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sh.tmem_base;
    volatile int* abort_flag = &sh.abort_flag;
    auto give_up = [&]() {
        atomicOr(status, SGR_TC_TIMEOUT);
        sh.abort_flag = 1;
    };

    if (warp == 0) {
        // ---- TMA producer ------------------------------------------------------------------
        if (lane == 0) {
            const uint64_t keep = policy_evict_last();  // the reference operand is read by every band
            uint32_t it = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
                int mb, nb;
                tile_coords(t, tiles_m, tiles_n, gm, mb, nb);
                const int m0 = mb * BM, n0 = nb * WBN;
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    const int s = it % WSTAGES;
                    const uint32_t ph = (it / WSTAGES) & 1;
                    if (!mbar_wait(smem_u32(&sh.empty[s]), ph ^ 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint32_t a_dst = smem_u32(smem + s * WSTAGE_BYTES);
                    const uint32_t b_dst = a_dst + A_BYTES;
                    // planes in the MMA's order: P0 and S (into A1), then L (into A2)
                    const int grp = kb / segb, plane = grp == 0 ? 0 : (grp == 1 ? 2 : 1);
                    const int kx = (plane * segb + kb % segb) * BK;
                    const uint32_t fb = smem_u32(&sh.full[s]);
                    mbar_expect_tx(fb, WSTAGE_BYTES);
                    tma_load_2d(a_dst, &tmA, kx, m0, fb);
                    tma_load_2d_hint(b_dst, &tmB, kx, n0, fb, keep);
                }
            }
            if (!ok) give_up();
            // drain: every issued stage's copies land before the CTA can exit
            for (uint32_t j = (it > (uint32_t)WSTAGES ? it - WSTAGES : 0); j < it; ++j) {
                const uint32_t s = j % WSTAGES, ph = (j / WSTAGES) & 1;
                const long long t0 = clock64();
                while (!mbar_try(smem_u32(&sh.full[s]), ph) && clock64() - t0 < WAIT_CYCLES) {
                }
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer --------------------------------------------------------------------------
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_i8(BM, WBN);
            uint32_t it = 0, tile_iter = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x, ++tile_iter) {
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    const int region = kb < 2 * segb ? 0 : 1;  // A1 (P0 and S planes), A2 (L plane)
                    const bool first = kb == 0 || kb == 2 * segb;
                    if (first) {
                        if (!mbar_wait(smem_u32(&sh.acc_empty[region]), (tile_iter & 1) ^ 1, abort_flag)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                    }
                    const int s = it % WSTAGES;
                    const uint32_t ph = (it / WSTAGES) & 1;
                    if (!mbar_wait(smem_u32(&sh.full[s]), ph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(smem + s * WSTAGE_BYTES);
                    const uint64_t da = smem_desc(a_addr), db = smem_desc(a_addr + A_BYTES);
                    const uint32_t tc = tmem + region * WBN;
#pragma unroll
                    for (int k = 0; k < BK / 32; ++k)
                        umma_i8(tc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc,
                                (first && k == 0) ? 0u : 1u);
                    umma_commit(smem_u32(&sh.empty[s]));
                    if (kb == 2 * segb - 1) umma_commit(smem_u32(&sh.acc_full[0]));
                    if (kb == kblocks - 1) umma_commit(smem_u32(&sh.acc_full[1]));
                }
            }
            if (!ok) give_up();
            umma_commit(smem_u32(&sh.drain));  // every MMA has finished before TMEM is freed
        }
        if (lane == 0) {
            const long long t0 = clock64();
            while (!mbar_try(smem_u32(&sh.drain), 0) && clock64() - t0 < WAIT_CYCLES) {
            }
        }
    } else if (warp >= 4) {
        // ---- epilogue ------------------------------------------------------------------------
        // Lane = tile row 32 * quarter + lane; this warp scores columns [part * WCOLS, + WCOLS) in
        // 16-column chunks, staged through its 32 x 16 buffer as in corr_tc_kernel.
        const int ew = warp - 4, quarter = warp & 3, part = ew >> 2;
        float4* chunk = reinterpret_cast<float4*>(smem + WSTAGES * WSTAGE_BYTES + ew * CHUNK_BYTES);
        const bool vec_store = (ld % 4) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
        const int row = 32 * quarter + lane;
        const int64_t c1 = cbase, c2 = cbase - 1;
        auto release = [&](int g) {
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&sh.acc_empty[g]));
        };
        uint32_t tile_iter = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++tile_iter) {
            int mb, nb;
            tile_coords(t, tiles_m, tiles_n, gm, mb, nb);
            const int m0 = mb * BM, n0 = nb * WBN;
            const int q = m0 + row;
            const double rqv = q < nq ? rq[q] : 0.0;  // NaN when the query row is constant
            double rrv[WCH];
#pragma unroll
            for (int c = 0; c < WCH; ++c) {
                const int r = n0 + part * WCOLS + c * 16 + lane;
                rrv[c] = (lane < 16 && r < R) ? rr[r] : 0.0;  // NaN for a constant reference row
            }
            int lab = 0, lab_end = 0;
            float mnf = __int_as_float(0x7f800000), mxf = -__int_as_float(0x7f800000);
            bool seen = false;
            if (ext.kmin) {
                const int cb = n0 + part * WCOLS;
                int lo = 0, hi = ext.L - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (__ldg(ext.lstart + mid) <= cb) lo = mid;
                    else hi = mid - 1;
                }
                lab = lo;
                lab_end = __ldg(ext.lstart + lab + 1);
            }
            const uint32_t par = tile_iter & 1;
            bool got = __all_sync(0xffffffffu, mbar_wait(smem_u32(&sh.acc_full[0]), par, abort_flag));
            if (got) got = __all_sync(0xffffffffu, mbar_wait(smem_u32(&sh.acc_full[1]), par, abort_flag));
            if (!got) {
                if (lane == 0) give_up();
                break;
            }
            tc_fence_after();
            const uint32_t lane_base = tmem + ((uint32_t)(32 * quarter) << 16);
            const uint32_t b1 = lane_base + part * WCOLS, b2 = lane_base + WBN + part * WCOLS;
            uint32_t x1[2][16], x2[2][16];
            tmem_ld16(b1, x1[0]);
            tmem_ld16(b2, x2[0]);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < WCH; ++c) {
                const int col0 = part * WCOLS + c * 16;
                if (c + 1 < WCH) {
                    tmem_ld16(b1 + 16 * (c + 1), x1[(c + 1) & 1]);
                    tmem_ld16(b2 + 16 * (c + 1), x2[(c + 1) & 1]);
                } else {
                    release(0);  // every TMEM read of this warp has completed
                    release(1);
                }
                float v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const double N = (double)(c1 * (int)x1[c & 1][j] - c2 * (int)x2[c & 1][j]);
                    const double rrj = __shfl_sync(0xffffffffu, rrv[c], j);
                    v[j] = (float)((N * rqv) * rrj);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    chunk[lane * 4 + (u ^ ((lane >> 1) & 3))] =
                        make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
                if (ext.kmin && n0 + col0 + 16 <= min(lab_end, R)) {  // the chunk lies in one label
                    float a0 = fminf(fminf(v[0], v[1]), fminf(v[2], v[3]));
                    float b0 = fmaxf(fmaxf(v[0], v[1]), fmaxf(v[2], v[3]));
#pragma unroll
                    for (int j = 4; j < 16; j += 4) {
                        a0 = fminf(a0, fminf(fminf(v[j], v[j + 1]), fminf(v[j + 2], v[j + 3])));
                        b0 = fmaxf(b0, fmaxf(fmaxf(v[j], v[j + 1]), fmaxf(v[j + 2], v[j + 3])));
                    }
                    mnf = fminf(mnf, a0);
                    mxf = fmaxf(mxf, b0);
                    seen = true;
                } else if (ext.kmin) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int col = n0 + col0 + j;
                        if (col >= R) break;
                        if (col >= lab_end) {  // label boundary
                            if (seen && q < nq) {
                                atomicMin(ext.kmin + (size_t)q * ext.L + lab, ord_key(mnf));
                                atomicMax(ext.kmax + (size_t)q * ext.L + lab, ord_key(mxf));
                            }
                            mnf = __int_as_float(0x7f800000);
                            mxf = -__int_as_float(0x7f800000);
                            do {
                                ++lab;
                                lab_end = __ldg(ext.lstart + lab + 1);
                            } while (col >= lab_end);
                        }
                        mnf = fminf(mnf, v[j]);
                        mxf = fmaxf(mxf, v[j]);
                        seen = true;
                    }
                }
                // the chunk's 32 rows x 16 columns: lane l stores piece l % 4 of row l / 4 (+ 8 i)
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = 8 * i + (lane >> 2), u = lane & 3;
                    const int qq = m0 + 32 * quarter + r, col = n0 + col0 + 4 * u;
                    const float4 val = chunk[r * 4 + (u ^ ((r >> 1) & 3))];
                    if (qq >= nq || col >= R) continue;
                    float* dst = out + (size_t)qq * ld + col;
                    // streaming stores (evict first): the scores are read once, later, and must not
                    // push the reference operand out of L2
                    if (vec_store && col + 3 < R) {
                        __stcs(reinterpret_cast<float4*>(dst), val);
                    } else {
                        __stcs(dst, val.x);
                        if (col + 1 < R) __stcs(dst + 1, val.y);
                        if (col + 2 < R) __stcs(dst + 2, val.z);
                        if (col + 3 < R) __stcs(dst + 3, val.w);
                    }
                }
                __syncwarp();  // the next chunk may overwrite the staging buffer
                if (c + 1 < WCH) tmem_wait_ld();
            }
            if (ext.kmin && seen && q < nq) {
                atomicMin(ext.kmin + (size_t)q * ext.L + lab, ord_key(mnf));
                atomicMax(ext.kmax + (size_t)q * ext.L + lab, ord_key(mxf));
            }
        }
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// Overlapped wide form: the 16 epilogue warps are warps 0-15 (warp % 4 is the TMEM lane quadrant
// again), the TMA producer warp 16 and the MMA warp 17 (registers are allocated per four warps, so
// the CTA's 18 warps leave 96 registers per thread).  Each epilogue warp takes its 64 columns of A1
// into registers as soon as A1 is complete (while the MMA multiplies the L plane into A2) and
// releases A1 at once, so the next tile's P0 and S
// planes are multiplied while the warp walks A2 and stores the scores; A2 is released when its last
// chunk has been read, well before the next tile's L plane.
constexpr int HOLD_THREADS = 32 * 18;

__global__ void __launch_bounds__(HOLD_THREADS, 1)
    corr_wide_hold_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int nq,
                          int R, int Kp, const double* __restrict__ rq, const double* __restrict__ rr,
                          float* __restrict__ out, int64_t ld, int* status, LabelExtremes ext, int gm, int cbase) {
    constexpr int EW = 16, WCOLS = 64, WCH = 4;
    constexpr int PRODUCER = 16, ISSUER = 17;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ TcShared sh;
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_n = (R + WBN - 1) / WBN, tiles_m = (nq + BM - 1) / BM;
    const int n_tiles = tiles_m * tiles_n;
    const int segb = Kp / BK, kblocks = 3 * segb;

    if (threadIdx.x == 0) {
        for (int s = 0; s < WSTAGES; ++s) {
            mbar_init(smem_u32(&sh.full[s]), 1);
            mbar_init(smem_u32(&sh.empty[s]), 1);
        }
        for (int g = 0; g < 2; ++g) {
            mbar_init(smem_u32(&sh.acc_full[g]), 1);
            mbar_init(smem_u32(&sh.acc_empty[g]), EW);
        }
        mbar_init(smem_u32(&sh.drain), 1);
        sh.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == ISSUER) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh.tmem_base)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sh.tmem_base;
    volatile int* abort_flag = &sh.abort_flag;
    auto give_up = [&]() {
        atomicOr(status, SGR_TC_TIMEOUT);
        sh.abort_flag = 1;
    };

    if (warp == PRODUCER) {
        if (lane == 0) {
            const uint64_t keep = policy_evict_last();  // the reference operand is read by every band
            uint32_t it = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
                int mb, nb;
                tile_coords(t, tiles_m, tiles_n, gm, mb, nb);
                const int m0 = mb * BM, n0 = nb * WBN;
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    const int s = it % WSTAGES;
                    const uint32_t ph = (it / WSTAGES) & 1;
                    if (!mbar_wait(smem_u32(&sh.empty[s]), ph ^ 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint32_t a_dst = smem_u32(smem + s * WSTAGE_BYTES);
                    const uint32_t b_dst = a_dst + A_BYTES;
                    const int grp = kb / segb, plane = grp == 0 ? 0 : (grp == 1 ? 2 : 1);  // P0, S, L
                    const int kx = (plane * segb + kb % segb) * BK;
                    const uint32_t fb = smem_u32(&sh.full[s]);
                    mbar_expect_tx(fb, WSTAGE_BYTES);
                    tma_load_2d(a_dst, &tmA, kx, m0, fb);
                    tma_load_2d_hint(b_dst, &tmB, kx, n0, fb, keep);
                }
            }
            if (!ok) give_up();
            for (uint32_t j = (it > (uint32_t)WSTAGES ? it - WSTAGES : 0); j < it; ++j) {
                const uint32_t s = j % WSTAGES, ph = (j / WSTAGES) & 1;
                const long long t0 = clock64();
                while (!mbar_try(smem_u32(&sh.full[s]), ph) && clock64() - t0 < WAIT_CYCLES) {
                }
            }
        }
    } else if (warp == ISSUER) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_i8(BM, WBN);
            uint32_t it = 0, tile_iter = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x, ++tile_iter) {
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    const int region = kb < 2 * segb ? 0 : 1;  // A1 (P0 and S planes), A2 (L plane)
                    const bool first = kb == 0 || kb == 2 * segb;
                    if (first) {
                        if (!mbar_wait(smem_u32(&sh.acc_empty[region]), (tile_iter & 1) ^ 1, abort_flag)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                    }
                    const int s = it % WSTAGES;
                    const uint32_t ph = (it / WSTAGES) & 1;
                    if (!mbar_wait(smem_u32(&sh.full[s]), ph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(smem + s * WSTAGE_BYTES);
                    const uint64_t da = smem_desc(a_addr), db = smem_desc(a_addr + A_BYTES);
                    const uint32_t tc = tmem + region * WBN;
#pragma unroll
                    for (int k = 0; k < BK / 32; ++k)
                        umma_i8(tc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc,
                                (first && k == 0) ? 0u : 1u);
                    umma_commit(smem_u32(&sh.empty[s]));
                    if (kb == 2 * segb - 1) umma_commit(smem_u32(&sh.acc_full[0]));
                    if (kb == kblocks - 1) umma_commit(smem_u32(&sh.acc_full[1]));
                }
            }
            if (!ok) give_up();
            umma_commit(smem_u32(&sh.drain));  // every MMA has finished before TMEM is freed
        }
        if (lane == 0) {
            const long long t0 = clock64();
            while (!mbar_try(smem_u32(&sh.drain), 0) && clock64() - t0 < WAIT_CYCLES) {
            }
        }
    } else {
        // ---- epilogue: warps 0-15 --------------------------------------------------------------
        const int quarter = warp & 3, part = warp >> 2;
        float4* chunk = reinterpret_cast<float4*>(smem + WSTAGES * WSTAGE_BYTES + warp * CHUNK_BYTES);
        const bool vec_store = (ld % 4) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
        const int row = 32 * quarter + lane;
        const int64_t c1 = cbase, c2 = cbase - 1;
        auto release = [&](int g) {
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&sh.acc_empty[g]));
        };
        const uint32_t lane_base = tmem + ((uint32_t)(32 * quarter) << 16);
        const uint32_t b1 = lane_base + part * WCOLS, b2 = lane_base + WBN + part * WCOLS;
        uint32_t tile_iter = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++tile_iter) {
            int mb, nb;
            tile_coords(t, tiles_m, tiles_n, gm, mb, nb);
            const int m0 = mb * BM, n0 = nb * WBN;
            const int q = m0 + row;
            const uint32_t par = tile_iter & 1;
            // A1: all 64 columns into registers, then release it for the next tile's first planes
            if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&sh.acc_full[0]), par, abort_flag))) {
                if (lane == 0) give_up();
                break;
            }
            tc_fence_after();
            uint32_t a1[WCH][16];
#pragma unroll
            for (int c = 0; c < WCH; ++c) tmem_ld16(b1 + 16 * c, a1[c]);
            tmem_wait_ld();
            release(0);
            const double rqv = q < nq ? rq[q] : 0.0;  // NaN when the query row is constant
            int lab = 0, lab_end = 0;
            float mnf = __int_as_float(0x7f800000), mxf = -__int_as_float(0x7f800000);
            bool seen = false;
            if (ext.kmin) {
                const int cb = n0 + part * WCOLS;
                int lo = 0, hi = ext.L - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (__ldg(ext.lstart + mid) <= cb) lo = mid;
                    else hi = mid - 1;
                }
                lab = lo;
                lab_end = __ldg(ext.lstart + lab + 1);
            }
            if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&sh.acc_full[1]), par, abort_flag))) {
                if (lane == 0) give_up();
                break;
            }
            tc_fence_after();
            // reference norms of this warp's columns, lanes 0-15 of chunk c; the next chunk's loaded
            // while this one is scored (NaN for a constant reference row)
            auto norm_of = [&](int c) {
                const int rcol = n0 + part * WCOLS + c * 16 + lane;
                return (lane < 16 && rcol < R) ? rr[rcol] : 0.0;
            };
            double rr_next = norm_of(0);
#pragma unroll
            for (int c = 0; c < WCH; ++c) {
                const int col0 = part * WCOLS + c * 16;
                const double rrl = rr_next;
                if (c + 1 < WCH) rr_next = norm_of(c + 1);
                uint32_t x2[16];
                tmem_ld16(b2 + 16 * c, x2);
                tmem_wait_ld();
                if (c + 1 == WCH) release(1);  // every TMEM read of this warp has completed
                float v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const double N = (double)(c1 * (int)a1[c][j] - c2 * (int)x2[j]);
                    const double rrj = __shfl_sync(0xffffffffu, rrl, j);
                    v[j] = (float)((N * rqv) * rrj);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    chunk[lane * 4 + (u ^ ((lane >> 1) & 3))] =
                        make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
                if (ext.kmin && n0 + col0 + 16 <= min(lab_end, R)) {  // the chunk lies in one label
                    float a0 = fminf(fminf(v[0], v[1]), fminf(v[2], v[3]));
                    float b0 = fmaxf(fmaxf(v[0], v[1]), fmaxf(v[2], v[3]));
#pragma unroll
                    for (int j = 4; j < 16; j += 4) {
                        a0 = fminf(a0, fminf(fminf(v[j], v[j + 1]), fminf(v[j + 2], v[j + 3])));
                        b0 = fmaxf(b0, fmaxf(fmaxf(v[j], v[j + 1]), fmaxf(v[j + 2], v[j + 3])));
                    }
                    mnf = fminf(mnf, a0);
                    mxf = fmaxf(mxf, b0);
                    seen = true;
                } else if (ext.kmin) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int col = n0 + col0 + j;
                        if (col >= R) break;
                        if (col >= lab_end) {  // label boundary
                            if (seen && q < nq) {
                                atomicMin(ext.kmin + (size_t)q * ext.L + lab, ord_key(mnf));
                                atomicMax(ext.kmax + (size_t)q * ext.L + lab, ord_key(mxf));
                            }
                            mnf = __int_as_float(0x7f800000);
                            mxf = -__int_as_float(0x7f800000);
                            do {
                                ++lab;
                                lab_end = __ldg(ext.lstart + lab + 1);
                            } while (col >= lab_end);
                        }
                        mnf = fminf(mnf, v[j]);
                        mxf = fmaxf(mxf, v[j]);
                        seen = true;
                    }
                }
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = 8 * i + (lane >> 2), u = lane & 3;
                    const int qq = m0 + 32 * quarter + r, col = n0 + col0 + 4 * u;
                    const float4 val = chunk[r * 4 + (u ^ ((r >> 1) & 3))];
                    if (qq >= nq || col >= R) continue;
                    float* dst = out + (size_t)qq * ld + col;
                    // streaming stores (evict first): the scores are read once, later, and must not
                    // push the reference operand out of L2
                    if (vec_store && col + 3 < R) {
                        __stcs(reinterpret_cast<float4*>(dst), val);
                    } else {
                        __stcs(dst, val.x);
                        if (col + 1 < R) __stcs(dst + 1, val.y);
                        if (col + 2 < R) __stcs(dst + 2, val.z);
                        if (col + 3 < R) __stcs(dst + 3, val.w);
                    }
                }
                __syncwarp();  // the next chunk may overwrite the staging buffer
            }
            if (ext.kmin && seen && q < nq) {
                atomicMin(ext.kmin + (size_t)q * ext.L + lab, ord_key(mnf));
                atomicMax(ext.kmax + (size_t)q * ext.L + lab, ord_key(mxf));
            }
        }
    }
    __syncthreads();
    if (warp == ISSUER) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// FP16-operand variant on 128 x 256 tiles (not exact: see corr_tc_kernel<true>).  One plane of d
// as IEEE half, kind::f16 MMAs with FP32 accumulation into one 256-column accumulator, so two
// accumulators fit TMEM and the epilogue of tile t reads one while the MMAs of tile t + 1 fill the
// other.  Warp roles and the epilogue's staging as in corr_wide_hold_kernel.
__global__ void __launch_bounds__(HOLD_THREADS, 1)
    corr_wide_f16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int nq,
                         int R, int Kp, const double* __restrict__ rq, const double* __restrict__ rr,
                         float* __restrict__ out, int64_t ld, int* status, LabelExtremes ext, int gm) {
    constexpr int EW = 16, WCOLS = 64, WCH = 4;
    constexpr int PRODUCER = 16, ISSUER = 17;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ TcShared sh;
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_n = (R + WBN - 1) / WBN, tiles_m = (nq + BM - 1) / BM;
    const int n_tiles = tiles_m * tiles_n;
    const int kblocks = 2 * Kp / BK;  // one plane of 2 * Kp bytes

    if (threadIdx.x == 0) {
        for (int s = 0; s < WSTAGES; ++s) {
            mbar_init(smem_u32(&sh.full[s]), 1);
            mbar_init(smem_u32(&sh.empty[s]), 1);
        }
        for (int g = 0; g < 2; ++g) {
            mbar_init(smem_u32(&sh.acc_full[g]), 1);
            mbar_init(smem_u32(&sh.acc_empty[g]), EW);
        }
        mbar_init(smem_u32(&sh.drain), 1);
        sh.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == ISSUER) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh.tmem_base)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sh.tmem_base;
    volatile int* abort_flag = &sh.abort_flag;
    auto give_up = [&]() {
        atomicOr(status, SGR_TC_TIMEOUT);
        sh.abort_flag = 1;
    };

    if (warp == PRODUCER) {
        if (lane == 0) {
            const uint64_t keep = policy_evict_last();
            uint32_t it = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
                int mb, nb;
                tile_coords(t, tiles_m, tiles_n, gm, mb, nb);
                const int m0 = mb * BM, n0 = nb * WBN;
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    const int s = it % WSTAGES;
                    const uint32_t ph = (it / WSTAGES) & 1;
                    if (!mbar_wait(smem_u32(&sh.empty[s]), ph ^ 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint32_t a_dst = smem_u32(smem + s * WSTAGE_BYTES);
                    const uint32_t fb = smem_u32(&sh.full[s]);
                    mbar_expect_tx(fb, WSTAGE_BYTES);
                    tma_load_2d(a_dst, &tmA, kb * BK, m0, fb);
                    tma_load_2d_hint(a_dst + A_BYTES, &tmB, kb * BK, n0, fb, keep);
                }
            }
            if (!ok) give_up();
            for (uint32_t j = (it > (uint32_t)WSTAGES ? it - WSTAGES : 0); j < it; ++j) {
                const uint32_t s = j % WSTAGES, ph = (j / WSTAGES) & 1;
                const long long t0 = clock64();
                while (!mbar_try(smem_u32(&sh.full[s]), ph) && clock64() - t0 < WAIT_CYCLES) {
                }
            }
        }
    } else if (warp == ISSUER) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_f16(BM, WBN);
            uint32_t it = 0, tile_iter = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x, ++tile_iter) {
                const int region = tile_iter & 1;  // the two accumulators alternate between tiles
                const uint32_t use = tile_iter >> 1;
                if (!mbar_wait(smem_u32(&sh.acc_empty[region]), (use & 1) ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    const int s = it % WSTAGES;
                    const uint32_t ph = (it / WSTAGES) & 1;
                    if (!mbar_wait(smem_u32(&sh.full[s]), ph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(smem + s * WSTAGE_BYTES);
                    const uint64_t da = smem_desc(a_addr), db = smem_desc(a_addr + A_BYTES);
                    const uint32_t tc = tmem + region * WBN;
#pragma unroll
                    for (int k = 0; k < BK / 32; ++k)  // 32 bytes of K (16 halves) per MMA
                        umma_f16(tc, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc,
                                 (kb == 0 && k == 0) ? 0u : 1u);
                    umma_commit(smem_u32(&sh.empty[s]));
                    if (kb == kblocks - 1) umma_commit(smem_u32(&sh.acc_full[region]));
                }
            }
            if (!ok) give_up();
            umma_commit(smem_u32(&sh.drain));
        }
        if (lane == 0) {
            const long long t0 = clock64();
            while (!mbar_try(smem_u32(&sh.drain), 0) && clock64() - t0 < WAIT_CYCLES) {
            }
        }
    } else {
        // ---- epilogue: warps 0-15 --------------------------------------------------------------
        const int quarter = warp & 3, part = warp >> 2;
        float4* chunk = reinterpret_cast<float4*>(smem + WSTAGES * WSTAGE_BYTES + warp * CHUNK_BYTES);
        const bool vec_store = (ld % 4) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
        const int row = 32 * quarter + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * quarter) << 16);
        uint32_t tile_iter = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++tile_iter) {
            int mb, nb;
            tile_coords(t, tiles_m, tiles_n, gm, mb, nb);
            const int m0 = mb * BM, n0 = nb * WBN;
            const int q = m0 + row;
            const int region = tile_iter & 1;
            const double rqv = q < nq ? rq[q] : 0.0;  // NaN when the query row is constant
            auto norm_of = [&](int c) {
                const int rcol = n0 + part * WCOLS + c * 16 + lane;
                return (lane < 16 && rcol < R) ? rr[rcol] : 0.0;
            };
            double rr_next = norm_of(0);
            int lab = 0, lab_end = 0;
            float mnf = __int_as_float(0x7f800000), mxf = -__int_as_float(0x7f800000);
            bool seen = false;
            if (ext.kmin) {
                const int cb = n0 + part * WCOLS;
                int lo = 0, hi = ext.L - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (__ldg(ext.lstart + mid) <= cb) lo = mid;
                    else hi = mid - 1;
                }
                lab = lo;
                lab_end = __ldg(ext.lstart + lab + 1);
            }
            if (!__all_sync(0xffffffffu,
                            mbar_wait(smem_u32(&sh.acc_full[region]), (tile_iter >> 1) & 1, abort_flag))) {
                if (lane == 0) give_up();
                break;
            }
            tc_fence_after();
            const uint32_t base = lane_base + region * WBN + part * WCOLS;
            uint32_t acc[2][16];
            tmem_ld16(base, acc[0]);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < WCH; ++c) {
                const int col0 = part * WCOLS + c * 16;
                const double rrl = rr_next;
                if (c + 1 < WCH) {
                    rr_next = norm_of(c + 1);
                    tmem_ld16(base + 16 * (c + 1), acc[(c + 1) & 1]);
                } else {
                    tc_fence_before();  // every TMEM read of this warp has completed
                    __syncwarp();
                    if (lane == 0) mbar_arrive(smem_u32(&sh.acc_empty[region]));
                }
                float v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const double rrj = __shfl_sync(0xffffffffu, rrl, j);
                    v[j] = (float)(((double)__uint_as_float(acc[c & 1][j]) * rqv) * rrj);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    chunk[lane * 4 + (u ^ ((lane >> 1) & 3))] =
                        make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
                if (ext.kmin && n0 + col0 + 16 <= min(lab_end, R)) {  // the chunk lies in one label
                    float a0 = fminf(fminf(v[0], v[1]), fminf(v[2], v[3]));
                    float b0 = fmaxf(fmaxf(v[0], v[1]), fmaxf(v[2], v[3]));
#pragma unroll
                    for (int j = 4; j < 16; j += 4) {
                        a0 = fminf(a0, fminf(fminf(v[j], v[j + 1]), fminf(v[j + 2], v[j + 3])));
                        b0 = fmaxf(b0, fmaxf(fmaxf(v[j], v[j + 1]), fmaxf(v[j + 2], v[j + 3])));
                    }
                    mnf = fminf(mnf, a0);
                    mxf = fmaxf(mxf, b0);
                    seen = true;
                } else if (ext.kmin) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int col = n0 + col0 + j;
                        if (col >= R) break;
                        if (col >= lab_end) {  // label boundary
                            if (seen && q < nq) {
                                atomicMin(ext.kmin + (size_t)q * ext.L + lab, ord_key(mnf));
                                atomicMax(ext.kmax + (size_t)q * ext.L + lab, ord_key(mxf));
                            }
                            mnf = __int_as_float(0x7f800000);
                            mxf = -__int_as_float(0x7f800000);
                            do {
                                ++lab;
                                lab_end = __ldg(ext.lstart + lab + 1);
                            } while (col >= lab_end);
                        }
                        mnf = fminf(mnf, v[j]);
                        mxf = fmaxf(mxf, v[j]);
                        seen = true;
                    }
                }
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = 8 * i + (lane >> 2), u = lane & 3;
                    const int qq = m0 + 32 * quarter + r, col = n0 + col0 + 4 * u;
                    const float4 val = chunk[r * 4 + (u ^ ((r >> 1) & 3))];
                    if (qq >= nq || col >= R) continue;
                    float* dst = out + (size_t)qq * ld + col;
                    if (vec_store && col + 3 < R) {
                        __stcs(reinterpret_cast<float4*>(dst), val);
                    } else {
                        __stcs(dst, val.x);
                        if (col + 1 < R) __stcs(dst + 1, val.y);
                        if (col + 2 < R) __stcs(dst + 2, val.z);
                        if (col + 3 < R) __stcs(dst + 3, val.w);
                    }
                }
                __syncwarp();  // the next chunk may overwrite the staging buffer
                if (c + 1 < WCH) tmem_wait_ld();
            }
            if (ext.kmin && seen && q < nq) {
                atomicMin(ext.kmin + (size_t)q * ext.L + lab, ord_key(mnf));
                atomicMax(ext.kmax + (size_t)q * ext.L + lab, ord_key(mxf));
            }
        }
    }
    __syncthreads();
    if (warp == ISSUER) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        SGR_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess) fail(SGR_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// Tensor map of a [rows x row_bytes] operand matrix, box_rows x 128-byte boxes, 128B swizzle.
CUtensorMap limb_map(const int8_t* base, int rows, int row_bytes, int box_rows) {
    CUtensorMap m;
    cuuint64_t dims[2] = {(cuuint64_t)row_bytes, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(base), dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(SGR_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

}  // namespace

size_t corr_tc_smem(bool pair) {
    return pair ? (size_t)PAIR_STAGES * PAIR_STAGE_BYTES + STAGING_BYTES + 1024
                : (size_t)STAGES * STAGE_BYTES + STAGING_BYTES + 1024;
}

size_t corr_wide_smem(int ew) { return (size_t)WSTAGES * WSTAGE_BYTES + (size_t)ew * CHUNK_BYTES + 1024; }

int pick_limb_w(int G) {
    const int D = std::max(G - 1, 0);
    for (int w = 1; w <= 15; ++w) {
        const int C = w * w + 1, hc = C / 2;
        bool ok = true;
        for (int d = -D; d <= D && ok; ++d) {
            const int h = (int)std::floor((double)(d + hc) / C), l = d - C * h, s = h + l;
            ok = std::abs(w * h) <= 127 && s >= -128 && s <= 127 && l >= -128 && l <= 127;
        }
        if (ok) return w;
    }
    return 0;
}

void launch_corr_tc(const int8_t* A, const int8_t* B, int nq, int R, int Kp, const double* ra, const double* rb,
                    const int64_t* na, const int64_t* nb, float* scores, int64_t ld, int* status, cudaStream_t s,
                    bool f16, LabelExtremes ext, bool pair, int gm, int limb_w, int wide_warps) {
    if (nq <= 0 || R <= 0) return;
    if (Kp % BK != 0 || (reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15))
        fail(SGR_ERR_INVALID_ARGUMENT, "tensor-core correlation: misaligned operands");
    pair = pair && !f16;
    gm = std::max(gm, 1);
    // recombination of the planes' products for the split the limbs were written with
    const int k1 = limb_w ? 1 : 127, cbase = limb_w ? limb_w * limb_w + 1 : 128;
    if (f16 && wide_warps != 0) {  // FP16 operands on 128 x 256 tiles
        const CUtensorMap ta = limb_map(A, nq, 2 * Kp, BM), tb = limb_map(B, R, 2 * Kp, WBN);
        const size_t fsmem = corr_wide_smem(16);
        const long tiles = (long)((nq + BM - 1) / BM) * ((R + WBN - 1) / WBN);
        const int grid = (int)std::min<long>(tiles, device_sm_count());
        SGR_CUDA(cudaFuncSetAttribute(corr_wide_f16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsmem));
        corr_wide_f16_kernel<<<grid, HOLD_THREADS, fsmem, s>>>(ta, tb, nq, R, Kp, ra, rb, scores, ld, status, ext, gm);
        SGR_LAUNCH_CHECK();
        count_launch();
        return;
    }
    if (!f16 && !pair && limb_w > 0 && (wide_warps == 8 || wide_warps == 16 || wide_warps == 18)) {
        const CUtensorMap ta = limb_map(A, nq, 3 * Kp, BM), tb = limb_map(B, R, 3 * Kp, WBN);
        const long tiles = (long)((nq + BM - 1) / BM) * ((R + WBN - 1) / WBN);
        const int grid = (int)std::min<long>(tiles, device_sm_count());
        int resident = 0;
        if (wide_warps == 18) {
            SGR_CUDA(cudaFuncSetAttribute(corr_wide_hold_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)corr_wide_smem(16)));
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, corr_wide_hold_kernel, HOLD_THREADS,
                                                              corr_wide_smem(16)) != cudaSuccess)
                resident = 0;
            cudaGetLastError();
            if (resident < 1) wide_warps = 16;  // its registers and shared memory do not fit one SM here
        }
        if (wide_warps == 18) {  // the overlapped form (18 warps per CTA)
            const size_t hsmem = corr_wide_smem(16);
            corr_wide_hold_kernel<<<grid, HOLD_THREADS, hsmem, s>>>(ta, tb, nq, R, Kp, ra, rb, scores, ld, status, ext,
                                                                    gm, cbase);
            SGR_LAUNCH_CHECK();
            count_launch();
            return;
        }
        auto kern = wide_warps == 16 ? corr_wide_kernel<16> : corr_wide_kernel<8>;
        const size_t smem = corr_wide_smem(wide_warps);
        SGR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, 32 * (4 + wide_warps), smem, s>>>(ta, tb, nq, R, Kp, ra, rb, scores, ld, status, ext, gm,
                                                        cbase);
        SGR_LAUNCH_CHECK();
        count_launch();
        return;
    }
    const int row_bytes = (f16 ? 2 : 3) * Kp;
    const CUtensorMap ta = limb_map(A, nq, row_bytes, BM), tb = limb_map(B, R, row_bytes, pair ? BN / 2 : BN);
    const size_t smem = corr_tc_smem(pair);
    const int mt = pair ? 2 * BM : BM;
    const long tiles = (long)((nq + mt - 1) / mt) * ((R + BN - 1) / BN);
    if (!pair) {
        auto kern = f16 ? corr_tc_kernel<true, false> : corr_tc_kernel<false, false>;
        SGR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int grid = (int)std::min<long>(tiles, device_sm_count());
        kern<<<grid, THREADS, smem, s>>>(ta, tb, nq, R, Kp, ra, rb, na, nb, scores, ld, status, ext, gm, k1, cbase);
        SGR_LAUNCH_CHECK();
        count_launch();
        return;
    }
    auto kern = corr_tc_kernel<false, true>;
    SGR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // as many pairs as can be resident at once (a pair needs two SMs of one GPC)
    cfg.gridDim = dim3(2 * (unsigned)std::max(1, device_sm_count() / 2));
    int max_pairs = 0;
    if (cudaOccupancyMaxActiveClusters(&max_pairs, kern, &cfg) != cudaSuccess || max_pairs < 1) {
        cudaGetLastError();
        max_pairs = std::max(1, device_sm_count() / 2);
    }
    cfg.gridDim = dim3(2 * (unsigned)std::min<long>(tiles, max_pairs));
    SGR_CUDA(cudaLaunchKernelEx(&cfg, kern, ta, tb, nq, R, Kp, ra, rb, na, nb, scores, ld, status, ext, gm, k1, cbase));
    count_launch();
}

}  // namespace sgr
