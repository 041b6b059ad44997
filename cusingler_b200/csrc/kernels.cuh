// Device kernels of the SingleR path and their launch helpers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace sgr {

int device_sm_count();

// Device status bits (ctx->status): 1 CSR column out of range, 2 NaN value, 4 NaN-bearing list where
// libstdc++ would have read out of bounds, 8 missing sort scratch, SGR_TC_TIMEOUT a bounded wait of
// the tensor-core kernel ran out.
constexpr int SGR_TC_TIMEOUT = 16;

// Kernels launched by this process's library (read before and after a call to count its launches).
uint64_t launch_count();
void count_launch(uint64_t n = 1);

// Grid caps of the selection kernels; their scratch (NaN-bearing lists) is sized per warp of the
// capped grid.
// Warps of the score-step selection that may use NaN-list scratch at once: 64 per SM (the warp-per-row
// form; the staged form runs at most two blocks of 16 warps per SM).
inline int select_warps_with_scratch() { return device_sm_count() * 64; }

// ---- gather + rank ----------------------------------------------------------------------------
//
// A "rank group" is one gene subset: a column map from input column to position in [0, G) (or -1),
// its width G, the padded width Kp (multiple of 128) and where its rows go.
struct RankGroup {
    const int32_t* colmap;  // input column -> position, -1 if not in the subset
    int32_t G;
    int32_t Kp;
    void* out;              // LIMBS: int8 [rows][3*Kp] planes p0|L|S (split_limbs); D16: int16 [rows][Kp]
    int64_t* n2;            // per row: sum of d^2 (exact)
    double* rinv;           // per row: 1/sqrt(n2), NaN when n2 == 0
    float* f32norm;         // per row, fp32 reference-order sum of x^2 (x = d/2), or nullptr
    int32_t limb_w = 0;     // LIMBS: the split of split_limbs (0: base 128)
};

struct RankItem {
    uint32_t row;    // input CSR row
    uint32_t group;  // index into the group table
    uint32_t slot;   // output row within the group
    uint32_t pad;
};

// LIMBS: int8 planes H | L | S (3 * Kp bytes per row); D16: int16 d; F16: d as IEEE half (exact for
// |d| <= 2048), the operand of the FP16 correlation variant.
enum RankOut { RANK_LIMBS = 0, RANK_D16 = 1, RANK_F16 = 2 };
enum F32Norm { NORM_NONE = 0, NORM_SEQ = 1, NORM_TREE128 = 2 };

struct RankLaunch {
    const float* data;
    const int32_t* indices;
    const int32_t* indptr;
    uint32_t n_cols;            // input column count (bounds check)
    const RankItem* items;      // nullptr: item i is row row0 + i of group 0, slot i
    uint32_t row0;
    uint32_t n_items;
    const RankGroup* groups;    // device array
    int out_mode;               // RankOut
    int norm_mode;              // F32Norm
    int max_Kp;                 // largest Kp over the groups (smem sizing)
    int cap;                    // sort capacity per warp (power of two)
    int* status;                // device flags: bit0 column out of range, bit1 NaN value
    // Two-tier launch: when `overflow` is set, launch_rank ranks rows of at most 384 marker entries
    // with a small sort buffer (more warps per SM) and appends the other rows to `overflow`
    // (capacity n_items), which a second launch with `cap` ranks; `n_overflow` is one device int.
    RankItem* overflow = nullptr;
    int* n_overflow = nullptr;
    const int* n_items_dev = nullptr;  // item count read from device memory (second tier)
    // Optional compact form of the (one) column map every group shares, kept in shared memory: bit c
    // of map_bits is set when column c is in the subset, and its position is map_prefix[c / 32] plus
    // the set bits below it in its word (the map must be increasing over the subset's columns).
    const uint32_t* map_bits = nullptr;
    const uint16_t* map_prefix = nullptr;
};

// map_bits / map_prefix (ceil(n_cols / 32) words each) of an increasing column map (-1 = not in the
// subset), on the host.
void column_bits(const int32_t* colmap, uint32_t n_cols, uint32_t* bits, uint16_t* prefix);

void launch_rank(const RankLaunch& a, cudaStream_t s);

// Compact a CSR to the columns with map[c] >= 0 (new column = map[c]); two passes.  row_max (may be
// null, not cleared here): atomic maximum of the kept entries per row.
void launch_filter_count(const int32_t* indptr, const int32_t* indices, uint32_t n_rows, uint32_t n_cols,
                         const int32_t* map, int32_t* counts, cudaStream_t s,
                         const uint8_t* row_mask = nullptr, int* row_max = nullptr);
// *out += sum of vals[list[i]] for i < *n (n read on the device; *out is not cleared; each value is
// below 2^32 and a warp's partial sum too).
void launch_sum_listed(const int32_t* list, const int* n, const int32_t* vals, unsigned long long* out,
                       cudaStream_t s);
// mask[list[i]] = 1 for i < n (list entries must be valid rows of mask).
void launch_mark_rows(const int32_t* list, int n, uint8_t* mask, cudaStream_t s);
// out[i] = in[0] + ... + in[i-1] for i <= n.  scratch (optional): 2 * ceil(n / 4096) + 1 ints, which
// lets blocks scan 4096-value tiles in parallel.
void launch_exclusive_scan(const int32_t* in, int32_t* out, uint32_t n, int32_t* scratch, cudaStream_t s);
void launch_filter_fill(const float* data, const int32_t* indptr, const int32_t* indices, uint32_t n_rows,
                        uint32_t n_cols, const int32_t* map, const int32_t* out_ptr, float* out_data,
                        int32_t* out_indices, cudaStream_t s,
                        const uint8_t* row_mask = nullptr);

// ---- score-step correlation on CUDA cores -------------------------------------------------------
//
// scores[q - q0][r] for q in [q0, q0 + nq), r in [0, R): A/B are LIMBS rows (3*Kp bytes).
// fp32ref: fused multiply-add chain over genes in order (the reference's spearman kernel order).
// exact:   FP64 accumulation of the integer products (exact), FP64 normalisation.
void launch_corr_simt(bool fp32ref, const int8_t* A, const int8_t* B, int nq, int R, int G, int Kp,
                      const float* fa, const float* fb, const double* ra, const double* rb,
                      const int64_t* na, const int64_t* nb, float* scores, int64_t ld, int limb_w, cudaStream_t s);

// ---- per-label quantile, argmax, candidate flags ------------------------------------------------
struct LabelQ {
    int32_t start;       // first column of the label's scores in a score row
    int32_t len;
    int32_t kind;        // 0 single value, 1 minimum, 2 maximum, 3 interpolate between k-1 and k
    int32_t k;
    float prev_index;    // index[k-1] of the reference's float index grid
    float step;          // the grid step 1/(len-1) as float
    int32_t has_nan;     // some reference row of the label has zero variance
    int32_t pad;
};

// LabelQ of a score list of `len` values at `start` for quantile p: the reference's float index
// grid i * step with step = 1/(len-1), lower_bound of p (src/cusingler.cu:947-978).  Host function.
LabelQ make_lq(int start, int len, float p);

// row_len: floats of a score row that the labels cover.  With `lorder` (label ids, longest first)
// and rows of at most 200 KB, each block stages its row in shared memory before selecting.
// ext_min / ext_max (optional, staged path): per (row, label) extreme order keys from the
// correlation epilogue, used instead of a min / max pass for lists that cannot hold NaN.  warps: 8 or 16
// warps per CTA of the staged form (a block per row), 0 the warp-per-row form (with `lorder`), 1 the
// warp-per-row form with 32 registers per thread (64 warps per SM).
void launch_select_first(const float* scores, int64_t ld, int nq, int L, const LabelQ* lq, float p,
                         float thre, const int64_t* qn2, float* label_scores, int32_t* first, uint8_t* flags,
                         float* scratch, int64_t scratch_per_warp, int* status, int row_len, const int32_t* lorder,
                         cudaStream_t s, const uint32_t* ext_min = nullptr, const uint32_t* ext_max = nullptr,
                         int warps = 16);

// ---- fine-tune ----------------------------------------------------------------------------------
struct FtGroup {
    int32_t G;             // genes of the round's subset
    int32_t Kp;            // padded row length of d16 rows
    int32_t n_cells;       // query cells in the group
    int32_t n_ref;         // reference rows of the candidate labels
    int64_t q_el;          // first element of the group's d16 query rows
    int64_t r_el;          // first element of the group's d16 reference rows
    int64_t q_row;         // first per-row norm index of the group's query rows
    int64_t r_row;         // first per-row norm index of the group's reference rows
    int64_t s_off;         // first score (floats) of the group's n_cells x n_ref block
    int32_t n_labels;      // candidate labels of the group
    int32_t lq_off;        // first LabelQ of the group (label segments inside a score row)
    int64_t out_off;       // first label score of the group's n_cells x n_labels block
};

struct FtCorrItem {
    uint32_t group;
    uint32_t ref;          // reference row within the group
    uint32_t q_begin, q_end;
};

void launch_ft_corr(bool fp32ref, const FtGroup* groups, const FtCorrItem* items, uint32_t n_items,
                    const int16_t* qd, const int16_t* rd, const float* qf, const float* rf, const double* qr,
                    const double* rr, const int64_t* qn, const int64_t* rn, float* scores, cudaStream_t s);

struct FtSelItem {
    uint32_t group;
    uint32_t cell;         // query cell within the group
};

void launch_ft_select(const FtGroup* groups, const FtSelItem* items, uint32_t n_items, const LabelQ* lq,
                      float p, const float* scores, float* label_scores, float* scratch,
                      int64_t scratch_per_warp, int* status, cudaStream_t s);

// Exact score-step correlation on the tensor cores (corr_tc.cu): A/B are LIMBS rows of 3 * Kp bytes.
// pair: tiles of 256 query rows on clusters of two CTAs (tcgen05 cta_group::2); exact mode only.
size_t corr_tc_smem(bool pair);
// Per-(query, label) extremes written by the correlation epilogue for the selection: label l's
// reference columns are [lstart[l], lstart[l+1]); kmin / kmax (Q x L order keys, preset to all ones /
// zero) receive atomicMin / atomicMax of each list's scores.  kmin = nullptr: not written.
struct LabelExtremes {
    const int32_t* lstart = nullptr;
    int L = 0;
    uint32_t* kmin = nullptr;
    uint32_t* kmax = nullptr;
};

// gm: row bands per group of the tile order (the bands of a group sweep the reference tiles together,
// so the CTAs at work share them through L2); 1 visits band after band.
// limb_w: the split of the exact limbs (split_limbs; 0 = base 128).  wide_warps 8 or 16 (with
// limb_w > 0, not f16 or pair) runs the 128 x 256-tile two-accumulator form with that many epilogue
// warps, 18 its overlapped form (18 warps per CTA: A1 held in registers while the next tile's MMAs
// run); 0 the 128 x 160 three-accumulator form.  With f16, any wide_warps but 0 runs the FP16
// operands on 128 x 256 tiles with two alternating accumulators.
void launch_corr_tc(const int8_t* A, const int8_t* B, int nq, int R, int Kp, const double* ra, const double* rb,
                    const int64_t* na, const int64_t* nb, float* scores, int64_t ld, int* status, cudaStream_t s,
                    bool f16 = false, LabelExtremes ext = LabelExtremes{}, bool pair = false, int gm = 1,
                    int limb_w = 0, int wide_warps = 0);
// Multiplier m of the limbs' reconstruction d = m * p0 + s (split_limbs with w; 0 = base 128).
__host__ __device__ inline int limb_mult(int w) { return w == 0 ? 127 : w; }
// Smallest w whose split (split_limbs) keeps every limb of |d| <= G - 1 in int8; 0 if none does.
int pick_limb_w(int G);
size_t corr_wide_smem(int ew);

// Persistent exact fine-tune (finetune.cu).
struct FtPersistentArgs {
    const uint32_t* ref_sorted;   // thre-pool entries by value, gene | run end << 31, in 32-row blocks
    const int32_t* blk_base;      // per label: its first row block
    const int32_t* ell_off;       // per row block: start in ref_sorted (blocks + 1 entries)
    const uint32_t* ctidx;        // (start, len) per label
    const uint32_t* ft_genes;     // fine-tune pair lists (thre ids)
    const uint32_t* ft_idx;       // (start, len) per ordered label pair
    const int32_t* gene_thre;     // marker count per candidate count n
    const LabelQ* lq_label;       // quantile grid per label (start 0)
    int L, Wt;
    const float* qf_data;         // query compacted to the thre pool
    const int32_t* qf_idx;
    const int32_t* qf_ptr;
    int Q;
    const uint8_t* flags;         // Q x L first-round candidate flags
    float p, thre;
    int times;
    const int32_t* cell_list;     // cells to fine-tune (nullptr: all Q cells)
    const int* n_list;            // device count of cell_list (read by the kernel)
    int* next_cell;               // work-queue counter (zeroed before launch)
    int32_t* final_labels;
    int32_t* rounds;
    float* scratch;               // per CTA: max_rcand scores + 8 * max_label sort space
    int64_t scratch_per_cta;
    int max_rcand, max_label, capq;
    int* status;
    int pack_shift;               // > 0: row scan on packed e-values (count << shift | e-sum); 0: plain
    int narrow;                   // with pack_shift: 32-bit run sums and masked run ends (bounds checked)
    const uint32_t* row_perm;     // per reference row slot in block order: its position in the label's row order
};

// Split path for heavy cells: state arrays of H cells (device), one round per launch_split_round.
struct FtSplit {
    const int32_t* cells;   // H query cells
    uint8_t* top;           // H x 256 candidate lists
    int* ntop;              // H
    int* rounds;            // H
    int* times;             // H
    int* state;             // H: 0 not started, 1 active, 2 finished
    int* nS;                // H
    int* kq;                // H
    int64_t* nq;            // H
    double* rq;             // H
    int* total;             // H: candidate reference rows of this round (0 when no scan)
    int* off;               // H x 257 label offsets
    int* eqv;               // H x Wt query e-values
    float* scores;          // H x max_rcand
    float* nan_scratch;     // H x 16 x max_label
    int max_rcand;
    unsigned long long* rows_scored;  // device counter: reference rows scored, summed over rounds
    int* items;             // 2 x max_items chunk lists (i * max_chunks + c)
    int* n_items;           // 2 list lengths
    int max_items;          // H * max_chunks
    int max_chunks;         // 256-row chunks of the longest possible round
};

// Function attributes of the split-round kernels; call once before launch_split_first (and before
// capturing rounds into a CUDA graph).
void split_round_setup(const FtPersistentArgs& a);
// First round's setup of the H cells (chunk list 0; n_items must be zero).
void launch_split_first(const FtPersistentArgs& a, const FtSplit& sp, int H, cudaStream_t s);
// One round: scan of chunk list q, then the decisions and the next round's setup (list q ^ 1).
void launch_split_round(const FtPersistentArgs& a, const FtSplit& sp, int H, int q, cudaStream_t s);

size_t ft_persistent_smem(int Wt, int capq, int nw);
void launch_ft_keys(int n, const int32_t* list, int L, const uint8_t* flags, const uint32_t* ctidx, int64_t* keys,
                    int32_t* ncand, cudaStream_t s);
// nw: warps per CTA (8 or 32)
int ft_persistent_grid(size_t smem, int nw);
void launch_ft_persistent(const FtPersistentArgs& a, int grid, size_t smem, int nw, cudaStream_t s);
// Value-sorted, run-flagged fine-tune lists of the reference rows in 32-row blocks: entry j of row r
// at ell_base[r] + (j / 4) * 128 + j % 4, padded to ell_len[r] entries with pad_gene entries.
void launch_ref_presort(const float* data, const int32_t* idx, const int32_t* ptr, const int32_t* ell_base,
                        const int32_t* ell_len, uint32_t n_rows, int cap, uint32_t pad_gene, uint32_t* out,
                        cudaStream_t s);

}  // namespace sgr
