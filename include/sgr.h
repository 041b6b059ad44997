/* sgr.h -- C ABI of the B200 SingleR annotation path (library: cusingler_b200/_lib/libsgr.so).
 *
 * The reference keeps its device path behind seven C++ free functions over file-scope globals
 * (src/cusingler.cuh:13-23 of STOmics/cusingler): initGPU, copyin_score, get_label, destroy_score,
 * copyin, cufinetune, destroy; the host stages live in DataParser (src/io.h:16-107).  This header
 * replaces that seam with an opaque context, plain pointers and sizes, and status codes instead
 * of exit().  Each entry point names the reference interface it replaces.
 *
 * Threading: one context is used by one host thread at a time.  Contexts are independent.
 * Memory: unless a sgr_csr says on_device = 1, every pointer is host memory; the library copies
 * what it needs and never keeps a caller pointer past the call.  A host query's rows are copied one
 * score block at a time on a stream of the context's own, overlapped with the scoring of the blocks
 * before; from page-locked host memory the copies run at the link's speed.
 */
#ifndef SGR_H_
#define SGR_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum sgr_status {
    SGR_OK = 0,
    SGR_ERR_INVALID_ARGUMENT = 1, /* malformed CSR, out-of-range code, bad size            */
    SGR_ERR_CUDA = 2,             /* a CUDA runtime call failed (message in last_error)    */
    SGR_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed                              */
    SGR_ERR_NO_INTERSECTION = 4,  /* reference and query share no gene name                */
    SGR_ERR_EMPTY_LABEL = 5,      /* a label name has no reference cell                    */
    SGR_ERR_UNSUPPORTED = 6,      /* a size beyond what the library supports               */
    SGR_ERR_STATE = 7,            /* call order violated (e.g. score before train)         */
    SGR_ERR_TIMEOUT = 8           /* a bounded device wait ran out                          */
} sgr_status;

/* Arithmetic of the rank correlation.
 *  SGR_MODE_EXACT   integer numerator on the INT8 tensor cores (doubled centred ranks split in two
 *                   int8 limbs, int32 accumulation, int64 recombination), FP64 normalisation,
 *                   rounded once to float.  Default.
 *  SGR_MODE_FP32REF the reference's own FP32 operation order, reproduced bit for bit (CUDA cores).
 */
typedef enum sgr_mode { SGR_MODE_EXACT = 0, SGR_MODE_FP32REF = 1 } sgr_mode;

/* A CSR matrix (rows = cells, columns = genes), the h5ad /X layout the reference reads
 * (test/test_basic.py:7-15).  Column indices of a row must be distinct; they need not be sorted. */
typedef struct sgr_csr {
    uint32_t n_rows;
    uint32_t n_cols;
    const float* data;      /* indptr[n_rows] values                                    */
    const int32_t* indices; /* indptr[n_rows] column ids                                */
    const int32_t* indptr;  /* n_rows + 1 offsets, indptr[0] == 0                       */
    int32_t on_device;      /* 0: host memory; 1: device memory of the context's GPU    */
} sgr_csr;

typedef struct sgr_ctx sgr_ctx;

/* Replaces initGPU (src/cusingler.cu:74-90): selects `gpuid`, creates a stream and the context.
 * `cores` is the host thread count for marker training (DataParser(thread_num), src/io.h:19).
 * gpuid == -1 makes a host-only context: sgr_train_ref then runs the marker training alone (for
 * inspection through sgr_get_info / sgr_get_u32) and the device stages return SGR_ERR_STATE. */
sgr_status sgr_create(int gpuid, int cores, sgr_ctx** out);

/* Replaces destroy / destroy_score (src/cusingler.cu:92-130): frees everything the context owns. */
sgr_status sgr_destroy(sgr_ctx* ctx);

/* Message of the last failed call on this context ("" if none).  Valid until the next call. */
const char* sgr_last_error(const sgr_ctx* ctx);

sgr_status sgr_set_mode(sgr_ctx* ctx, sgr_mode mode);

/* Replaces PyDataParser::prepareData + findIntersectionGenes + loadRefData + trainData
 * (src/io.cpp:792-821, 306-349, 351-370, 141-262) and the reference half of copyin_score /
 * copyin (src/cusingler.cu:283-521): intersects gene names, regroups reference rows by label,
 * trains the per-label-pair marker lists on the host, and leaves the ranked reference resident on
 * the device.  `celltypes[i]` is the label code of reference row i, narrowed to 8 bits as
 * src/io.cpp:813 does; `label_names` has n_labels entries.  The query gene names are needed here
 * because the gene intersection decides the reference's columns. */
sgr_status sgr_train_ref(sgr_ctx* ctx, const sgr_csr* ref, const int32_t* celltypes,
                         const char* const* label_names, uint32_t n_labels,
                         const char* const* ref_genes, const char* const* qry_genes,
                         uint32_t n_qry_genes);

/* Replaces copyin_score + get_label (src/cusingler.cu:283-413, 986-1136): per query cell, the
 * per-label `quantile` (a fraction, e.g. 0.8f) of its correlations with that label's reference
 * cells, the first label (last index of the maximum, as std::minmax_element gives) and the
 * candidate flags (score >= max - finetune_thre).  Outputs are host arrays:
 * first_labels[n_rows]; label_scores[n_rows * n_labels] and flags[n_rows * n_labels] may be NULL. */
sgr_status sgr_score_first(sgr_ctx* ctx, const sgr_csr* qry, float quantile, float finetune_thre,
                           int32_t* first_labels, float* label_scores, uint8_t* flags);

/* Replaces copyin + cufinetune (src/cusingler.cu:415-521, 1297-1333): starting from the candidate
 * flags (n_rows * n_labels, nonzero = candidate), repeats the fine-tune round until one label is
 * left (or finetune_times rounds when it is > 0) and writes final_labels[n_rows] (0 when a cell has
 * no candidate, as the reference does).  rounds (n_rows, may be NULL) receives the round count. */
sgr_status sgr_finetune(sgr_ctx* ctx, const sgr_csr* qry, const uint8_t* flags, float quantile,
                        float finetune_thre, int32_t finetune_times, int32_t* final_labels,
                        int32_t* rounds);

/* Both steps in one call (Pipeline::score + Pipeline::finetune, src/pipeline.cpp:47-111).
 * label_scores may be NULL. */
sgr_status sgr_annotate(sgr_ctx* ctx, const sgr_csr* qry, float quantile, float finetune_thre,
                        int32_t finetune_times, int32_t* first_labels, int32_t* final_labels,
                        float* label_scores);

/* Runs the context's work on `stream` (a cudaStream_t of the context's device; NULL restores the
 * context's own stream).  Calls stay synchronous: they return after their results are on the host. */
sgr_status sgr_set_stream(sgr_ctx* ctx, void* stream);

/* ---- Measurement --------------------------------------------------------------------------- */

/* Per-stage device times of the calls since the last sgr_reset_timings, measured with CUDA events
 * on the context's stream while profiling is on (sgr_set_profiling(ctx, 1)). */
typedef struct sgr_timings {
    double h2d_ms;          /* query upload (host inputs only; overlaps the score step)        */
    double rank_ms;         /* score-step gather + rank of the query                            */
    double corr_ms;         /* score-step correlation                                            */
    double select_ms;       /* score-step quantile / argmax / flags                              */
    double finetune_ms;     /* whole fine-tune (device time of its stages plus host decisions)   */
    double total_ms;        /* first to last event of the calls                                  */
    uint64_t launches;      /* kernels launched                                                  */
    uint64_t corr_launches;
    uint64_t rank_launches;
    uint64_t rank_bytes;    /* algorithmic bytes of the score-step gather + rank                 */
    uint64_t corr_ops;      /* algorithmic ops 2*Q*R*G of the score-step correlation             */
    uint64_t cells;         /* query cells annotated                                             */
    uint64_t ft_cell_rounds;/* fine-tune (cell, round) pairs                                     */
    double mlp_ms;          /* learned form: features, proposal network, routing                 */
    uint64_t select_launches;
    uint64_t select_bytes;  /* algorithmic bytes 4*Q*R read by the score-step selection          */
    uint64_t ft_queue_cells;/* fine-tune cells run whole by one CTA of the work-queue kernel      */
    uint64_t ft_split_cells;/* fine-tune cells whose rounds were spread over the GPU             */
    uint64_t ft_split_rounds;/* rounds of the spread path (each: prepare, scan, decide launches)  */
    uint64_t ft_split_rows; /* reference rows scored by the spread path, summed over its rounds   */
    uint64_t ft_cells;      /* cells that ran at least one fine-tune round                      */
    uint64_t ft_candidates; /* first-round candidate labels of those cells, summed               */
} sgr_timings;

sgr_status sgr_set_profiling(sgr_ctx* ctx, int on);

/* Launch-shape choices.  what 0: warps per CTA of the persistent fine-tune kernel (8 or 32);
 * what 1: candidate count from which a cell's fine-tune rounds are spread over the whole GPU
 * instead of one CTA (>= 2; large values disable the split path); what 2: MiB of score-step
 * correlations per block of queries (small blocks are read back from L2 by the selection); what 3:
 * 1 lets the fine-tune row scan keep each value run's count and e-sum in one packed 32-bit word when
 * the trained reference allows it, 2 (default) also keeps the run sums in 32 bits and applies run
 * ends with masks when the row lengths allow it, 0 always uses the two-register scan; what 5:
 * 1 runs the exact correlation on SM pairs (clusters of two CTAs, tcgen05 cta_group::2, 256-row
 * tiles), 0 one CTA per 128-row tile; what 6: row bands per group of the correlation's tile order
 * (1 to 4096; the bands of a group sweep the reference together so that the CTAs at work share
 * operand tiles in L2); what 7: the score-step selection's form: 8 or 16 warps per CTA that stages
 * a query row in shared memory, 0 for one warp per query row reading the scores directly, 1 the
 * same with 40 registers per thread (half again the warps per SM);
 * what 8: 1 trains the markers on the host instead of the device; what 9 (exact mode): 1 fine-tunes
 * each score block on a second stream while the next block is scored; what 10: the exact
 * correlation's tile: 8 or 16 for 128 x 256 tiles with two accumulators (when the trained marker
 * count allows the two-accumulator split, G <= 1921) and that many epilogue warps, 18 (default)
 * for the same tiles with the epilogue overlapping the next tile's products, 0 for 128 x 160 tiles
 * with three accumulators; what 11: 1 makes the next training write the base-128 limb split, which
 * only the 128 x 160 forms multiply.
 * No choice above changes any result.  what 4 (exact mode only; no counterpart in the reference):
 * 1 runs the score-step correlation on FP16 operands with FP32 accumulation (one tensor-core
 * product instead of three INT8 products; scores are not exact, their error against the exact
 * scores is reported by the benchmark), 0 (default) the exact INT8 form. */
sgr_status sgr_set_tuning(sgr_ctx* ctx, int what, int value);
sgr_status sgr_reset_timings(sgr_ctx* ctx);

/* Autotuner (no counterpart in the reference).  A host `sample` is first copied to the device once
 * (the trials then time the kernels, not the copy).  Phase 1 times the score step of `sample` for
 * every score-step shape -- correlation on one CTA or an SM pair per tile x tile
 * order of 1 or 16 bands per group x score block {256, 1024} MiB x selection form {warp per row at
 * 64 or 32 registers, 16-warp row-staging CTA}
 * (exact mode; fp32ref mode tunes the last two) -- and keeps the fastest; phase 2 then times the
 * whole annotation for every fine-tune shape -- pipelined or not (exact mode) x warps per CTA
 * {8, 32} x split-path threshold {4, 6, 9, 16, off} -- and keeps the fastest by wall time.  All choices stay set in the context.
 * learned = 1 tunes the learned form (sgr_annotate_learned with min_confidence / check_fraction), 0
 * the plain form.  Every candidate must give the same first (and, in phase 2, final) labels
 * (SGR_ERR_STATE otherwise).  The trials count in sgr_timings. */
typedef struct sgr_tuning {
    int32_t ft_warps;
    int32_t ft_heavy;       /* 1 << 30 when the split path is off */
    int32_t score_chunk_mb;
    int32_t trials;         /* phase-2 trials */
    double best_ms;         /* wall time of the chosen candidate on the sample */
    double worst_ms;        /* slowest phase-2 candidate */
    int32_t corr_pair;      /* 1: SM-pair correlation */
    int32_t corr_gm;        /* row bands per group of the correlation's tile order */
    int32_t select_warps;
    int32_t score_trials;   /* phase-1 trials */
    double score_best_ms;   /* wall time of the chosen score step on the sample */
    int32_t pipeline;       /* 1: each score block's fine-tune overlaps the next block's score step */
    int32_t corr_wide;      /* 8 / 16 / 18: 128 x 256-tile correlation (18: overlapped), 0: 128 x 160 */
} sgr_tuning;
sgr_status sgr_autotune(sgr_ctx* ctx, const sgr_csr* sample, float quantile, float finetune_thre,
                        int32_t finetune_times, int32_t learned, float min_confidence, float check_fraction,
                        sgr_tuning* out);
sgr_status sgr_get_timings(const sgr_ctx* ctx, sgr_timings* out);

/* ---- Learned proposal ------------------------------------------------------------------------ */

/* These entry points have no counterpart in the reference.  A small network (first-round
 * per-label scores minus their maximum -> 256 -> GELU -> 256 -> GELU -> labels, BF16 working weights,
 * FP32 master weights and accumulation, trained by the library's own CUDA kernels with AdamW)
 * proposes each cell's final label, so that confident cells can skip the fine-tune loop.  Its
 * inputs are (score - the cell's best score) / 0.05, clipped below at -8. */
typedef struct sgr_mlp_config {
    uint32_t hidden;        /* width of both hidden layers (default 256 when 0)        */
    uint32_t epochs;        /* passes over the training rows (default 20 when 0)       */
    uint32_t batch;         /* rows per step (default 4096 when 0)                     */
    float lr;               /* AdamW step size, e.g. 1e-3                              */
    float weight_decay;     /* decoupled weight decay on the weight matrices           */
    float beta1, beta2, eps;
    uint64_t seed;          /* initialisation and shuffling                            */
} sgr_mlp_config;

typedef struct sgr_learned_stats {
    uint64_t cells;         /* query cells                                              */
    uint64_t decided;       /* final label decided without fine-tune (0 or 1 candidate,
                               or a confident proposal)                                 */
    uint64_t finetuned;     /* cells that ran the plain fine-tune                      */
    uint64_t checked;       /* confident proposals re-run plain to measure agreement   */
    uint64_t check_agree;   /* ... of which the plain final label equals the proposal  */
} sgr_learned_stats;

/* Trains the proposal network on n rows of first-round label scores (host, n x n_labels, as
 * sgr_score_first returns them) and their plain-method final labels.  Rows holding NaN are skipped.
 * final_loss (may be NULL) receives the mean cross-entropy of the last step. */
sgr_status sgr_mlp_train(sgr_ctx* ctx, const float* label_scores, const int32_t* targets, uint32_t n,
                         const sgr_mlp_config* cfg, float* final_loss);

/* Proposed label and its softmax probability for n rows of label scores (host arrays). */
sgr_status sgr_mlp_predict(sgr_ctx* ctx, const float* label_scores, uint32_t n, int32_t* labels,
                           float* confidence);

/* Copies the FP32 parameters (layout W1[H][L], b1[H], W2[H][H], b2[H], W3[L][H], b3[L]) into `out`
 * (capacity `cap` floats, may be NULL to query sizes); sgr_mlp_load installs such a vector. */
sgr_status sgr_mlp_params(sgr_ctx* ctx, float* out, uint64_t cap, uint32_t* n_labels, uint32_t* hidden,
                          uint64_t* n_params);
sgr_status sgr_mlp_load(sgr_ctx* ctx, const float* params, uint32_t n_labels, uint32_t hidden);

/* One forward and backward pass (no update) on n rows of features (host, n x n_labels, already
 * centred) and targets: the mean loss and the flat gradient (same layout as the parameters). */
sgr_status sgr_mlp_debug_grads(sgr_ctx* ctx, const float* features, const int32_t* targets, uint32_t n,
                               float* grads, float* loss);

/* The learned form of sgr_annotate: score step, proposal, then the plain fine-tune only for cells
 * whose proposal is below `min_confidence`, is not one of their candidates, or whose scores hold
 * NaN; a `check_fraction` sample of the confident cells is re-run plain as well (their plain result
 * is returned) and counted in stats. */
sgr_status sgr_annotate_learned(sgr_ctx* ctx, const sgr_csr* qry, float quantile, float finetune_thre,
                                int32_t finetune_times, float min_confidence, float check_fraction,
                                int32_t* first_labels, int32_t* final_labels, sgr_learned_stats* stats);

/* ---- Streaming ----------------------------------------------------------------------------- */

/* Replaces the reference's query slicing (src/cusingler.cu:335-409: copyin_score cuts the query
 * into slices that fit the free device memory and get_label scores them one after another) for a
 * query that arrives as a sequence of host CSR batches, e.g. 65,536 cells each.  The reference stays
 * resident; batch i + 1 is uploaded on the context's copy stream into the second of two device
 * buffer sets while batch i is annotated, so with page-locked batches the upload is hidden behind
 * the previous batch's work.  learned = 0 runs the plain form (sgr_annotate), 1 the learned form
 * (sgr_annotate_learned with min_confidence / check_fraction; stats summed over batches, may be
 * NULL).  first_labels / final_labels hold the batches' rows one after another (sum of n_rows).
 * batch_ms (n_batches, may be NULL) receives, per batch, the time from the start of its upload to
 * its labels on the host. */
sgr_status sgr_annotate_stream(sgr_ctx* ctx, const sgr_csr* batches, uint32_t n_batches, float quantile,
                               float finetune_thre, int32_t finetune_times, int32_t learned,
                               float min_confidence, float check_fraction, int32_t* first_labels,
                               int32_t* final_labels, float* batch_ms, sgr_learned_stats* stats);

/* ---- Allocation-free selection -------------------------------------------------------------- */

/* This entry point has no counterpart in the reference.  It is for callers that cannot allocate
 * device memory: code running while another runtime owns the GPU's memory through its own pool and
 * budget, code being recorded into a CUDA graph, or latency-bound code where a cudaMalloc/cudaFree
 * would synchronise the device.  It does the score-step label selection of sgr_score_first (per
 * label the `quantile` of a query row's scores over that label's reference columns, the first
 * label, the candidate flags) on score rows the caller already holds on the device, and calls no
 * cudaMalloc, cudaFree or allocating library routine.
 *
 *   d_scores        n_rows x ld floats on the current device (row q: query q's correlations)
 *   label_ranges    host array, (start, len) of each label's columns, 2 * n_labels entries
 *   d_label_scores  n_rows x n_labels floats (device); d_first_labels n_rows (device);
 *   d_flags         n_rows x n_labels bytes (device) or NULL
 *   stream          cudaStream_t of the current device (NULL: the default stream)
 *
 * The call only enqueues work on `stream`; results are ready when the stream reaches that point.
 * Its temporary space is one fixed device array of 1,048,576 floats (4 MiB) inside the library,
 * which every GPU that loads the library holds until the process exits; each label may therefore
 * hold at most 131,072 reference columns (SGR_ERR_UNSUPPORTED beyond).  All calls share that
 * array, so calls that overlap on the GPU (other streams, other threads) race and must be
 * serialised by the caller.  The first call on a device looks the array's address up; make that
 * first call before any stream capture.  Because the call only enqueues, device-side conditions
 * that sgr_score_first reports through its status (a NaN input value, an out-of-range column) are
 * not checked here: the scores are the caller's, and a NaN-bearing list is sorted in libstdc++
 * order within its bounds, as in the main path. */
sgr_status sgr_select_labels_noalloc(const float* d_scores, int64_t ld, uint32_t n_rows,
                                     const uint32_t* label_ranges, uint32_t n_labels, float quantile,
                                     float finetune_thre, float* d_label_scores,
                                     int32_t* d_first_labels, uint8_t* d_flags, void* stream);

/* ---- Introspection (tests and tools) ------------------------------------------------------- */

typedef struct sgr_info {
    uint32_t n_labels;
    uint32_t n_genes;        /* gene space of the trained reference (its column count)        */
    uint32_t n_common;       /* marker genes of the score step (G)                             */
    uint32_t n_thre;         /* marker genes the fine-tune lists draw from                     */
    uint32_t filter_genes;   /* 1 when the gene names differed and were intersected             */
    uint32_t ref_rows;
    uint64_t n_pair_genes;   /* length of the concatenated per-pair marker lists               */
} sgr_info;

sgr_status sgr_get_info(const sgr_ctx* ctx, sgr_info* out);

/* what: 0 common genes (ascending), 1 thre genes (ascending), 2 per-pair positive marker lists
 * (concatenated, gene ids), 3 their (start, len) per ordered label pair (2 * L * L),
 * 4 fine-tune pair lists (thre-compact ids), 5 their (start, len) (2 * L * L), 6 (start, len) of
 * each label in the regrouped reference (2 * L), 7 original row of each regrouped reference row.
 * `cap` is the capacity of `out` in elements. */
sgr_status sgr_get_u32(const sgr_ctx* ctx, int what, uint32_t* out, uint64_t cap);

/* Doubled centred ranks d = 2 * rank - (G + 1) over the common genes, computed on the device by
 * the score-step gather kernel, for every row of `rows` (host copy, n_rows * n_common int32).
 * which: 0 the query rows given, 1 the trained reference (rows ignored). */
sgr_status sgr_debug_ranks(sgr_ctx* ctx, const sgr_csr* rows, int which, int32_t* d_out);

/* Raw score-step correlations (n_rows x ref_rows, float, host) of the query rows. */
sgr_status sgr_debug_scores(sgr_ctx* ctx, const sgr_csr* qry, float* out);

/* The device routines that restate libstdc++'s std::sort and std::minmax_element orders (used by
 * the quantile and argmax kernels for NaN-bearing score lists), run on the host for testing. */
void sgr_debug_stl_sort(float* v, int32_t n);
void sgr_debug_stl_minmax(const float* v, int32_t n, int32_t* min_idx, int32_t* max_idx);

#ifdef __cplusplus
}
#endif

#endif /* SGR_H_ */
