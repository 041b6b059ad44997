// C ABI (include/sgr.h) and the host orchestration of the SingleR path on one GPU.
//
// Reference flow restated (STOmics/cusingler): Pipeline::train / score / finetune
// (src/pipeline.cpp:128-156, 47-111), get_label (src/cusingler.cu:986-1136), cufinetune and
// finetune_round (src/cusingler.cu:1138-1333).  The reference keeps every stage's state in
// file-scope globals and exits on errors; here the state lives in sgr_ctx and errors come back as
// sgr_status.

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <map>
#include <random>
#include <set>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "mlp.h"
#include "sgr_internal.h"
#include "stl_order.h"

using namespace sgr;

namespace {

enum Stage { ST_H2D = 0, ST_RANK, ST_CORR, ST_SELECT, ST_FT, ST_MLP, ST_COUNT };

// CUDA-event spans on the context's stream; resolved after the call's final synchronisation.
struct Profiler {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    struct Span {
        int stage;
        cudaEvent_t a, b;
    };
    std::vector<Span> spans;
    sgr_timings acc{};
    // fine-tune rounds summed on the device (learned form), copied to pinned memory by the call
    unsigned long long* h_rounds = nullptr;
    bool rounds_pending = false;

    cudaEvent_t take() {
        if (used == pool.size()) {
            cudaEvent_t e;
            SGR_CUDA(cudaEventCreate(&e));
            pool.push_back(e);
        }
        return pool[used++];
    }
    int begin(int stage, cudaStream_t s) {
        if (!on) return -1;
        Span sp{stage, take(), take()};
        SGR_CUDA(cudaEventRecord(sp.a, s));
        spans.push_back(sp);
        return (int)spans.size() - 1;
    }
    void end(int id, cudaStream_t s) {
        if (id >= 0) SGR_CUDA(cudaEventRecord(spans[id].b, s));
    }
    // after the stream is synchronised
    void collect() {
        if (rounds_pending && h_rounds) acc.ft_cell_rounds += *h_rounds;
        rounds_pending = false;
        if (!on || spans.empty()) {
            spans.clear();
            used = 0;
            return;
        }
        double* slot[ST_COUNT] = {&acc.h2d_ms, &acc.rank_ms, &acc.corr_ms, &acc.select_ms, &acc.finetune_ms,
                                  &acc.mlp_ms};
        float first_last = 0.f;
        for (auto& sp : spans) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, sp.a, sp.b) == cudaSuccess) *slot[sp.stage] += ms;
        }
        if (cudaEventElapsedTime(&first_last, spans.front().a, spans.back().b) == cudaSuccess)
            acc.total_ms += first_last;
        cudaGetLastError();
        spans.clear();
        used = 0;
    }
    ~Profiler() {
        for (auto e : pool) cudaEventDestroy(e);
        if (h_rounds) cudaFreeHost(h_rounds);
    }
};

}  // namespace

struct sgr_ctx {
    int device = 0;
    int cores = 1;
    cudaStream_t stream = nullptr;      // the stream work runs on
    cudaStream_t own_stream = nullptr;  // created with the context
    cudaStream_t side = nullptr;        // fine-tune split path, concurrent with the work queue
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_state[2] = {nullptr, nullptr};  // split path: cell states copied to h_state
    cudaStream_t copy = nullptr;                    // host query rows, copied chunk by chunk
    std::vector<cudaEvent_t> up_ev;                 // one per copied chunk
    int32_t* h_state = nullptr;                     // pinned, two buffers of 1,024 cell states
    Profiler prof;
    sgr_mode mode = SGR_MODE_EXACT;
    std::string err;
    bool trained = false;        // reference resident on the device
    bool markers_ready = false;  // host marker training done

    Markers mk;
    uint32_t R = 0;      // reference rows
    uint32_t ref_cols = 0;
    int G = 0, Kp = 0;   // score-step genes and padded row length
    uint32_t Wt = 0;     // fine-tune gene pool

    // device reference: regrouped CSR (original columns), score-step ranks, thre-filtered CSR
    DevBuf<float> ref_data;
    DevBuf<int32_t> ref_indices, ref_indptr;
    DevBuf<int32_t> ref_map_common, qry_map_common, ref_map_thre, qry_map_thre;
    DevBuf<uint32_t> ref_bits, qry_bits;     // the score-step column maps as bits + per-word prefixes
    DevBuf<uint16_t> ref_prefix, qry_prefix;
    DevBuf<int8_t> ref_limbs;
    DevBuf<int64_t> ref_n2;
    DevBuf<double> ref_rinv;
    DevBuf<float> ref_f32;
    std::vector<int64_t> h_ref_n2;
    DevBuf<float> reff_data;
    DevBuf<int32_t> reff_indices, reff_indptr;
    DevBuf<int> filter_max;        // filter_csr: longest compacted row
    DevBuf<int> sp_items;          // split path: two chunk lists
    DevBuf<int> sp_nitems;         // split path: their lengths
    DevBuf<int32_t> d_blk_base;    // fine-tune lists: first 32-row block of each label
    DevBuf<uint32_t> d_row_perm;   // fine-tune lists: block position -> position in the label's rows
    DevBuf<int32_t> d_ell_off;     // fine-tune lists: start of each 32-row block in ref_sorted
    uint32_t R32 = 0;              // reference rows with each label's range padded to a multiple of 32
    int pack_shift = 0;            // packed fine-tune row scan (0: not representable, plain scan)
    int pack_scan = 2;             // tuning: packed scan when representable (2: and narrow when representable)
    bool pack_narrow = false;      // the trained reference allows 32-bit run sums
    DevBuf<uint32_t> ref_sorted;       // thre-pool entries of each reference row, by value
    DevBuf<uint32_t> d_ctidx, d_ft_genes, d_ft_idx;
    DevBuf<int32_t> d_gene_thre;
    DevBuf<LabelQ> d_lq_label;
    DevBuf<int> next_cell;
    DevBuf<uint8_t> ft_row_mask;   // rows of the listed cells (learned form's fine-tune)
    int corr_f16 = 0;              // tuning: score-step correlation on FP16 operands (not exact)
    int corr_pair = 0;             // tuning: exact correlation on SM pairs (cta_group::2, 256-row tiles)
    int corr_gm = 1;               // tuning: row bands per group of the correlation's tile order
    int select_warps = 16;         // tuning: score-step selection, 8 or 16 warps per row-staging CTA, 0 / 1 a warp per row
    int host_training = 0;         // tuning: marker medians and pair lists on the host instead of the device
    int pipeline = 0;              // tuning: fine-tune each score block on its own stream while the next is scored
    cudaStream_t ft_s = nullptr;   // the pipelined fine-tune's stream
    std::vector<cudaEvent_t> blk_ev;  // one per score block (+ 1): block scored / fine-tune joined
    DevBuf<uint16_t> ref_f16;      // reference ranks as IEEE half rows [R][Kp]
    bool ref_f16_ready = false;
    DevBuf<int32_t> d_lorder;     // label ids by reference-cell count, longest first (score-step selection)
    DevBuf<int32_t> scan_part;    // tile sums of the filter's exclusive scan
    DevBuf<int32_t> d_lstart;     // first reference column of each label (L + 1 entries)
    DevBuf<uint32_t> ext_min, ext_max;  // per (query, label) score extremes of a score block
    DevBuf<RankItem> rank_overflow;  // rows ranked by the rank kernel's large-buffer tier
    DevBuf<int> rank_n_overflow;
    int limb_w = 0;              // split of the exact limbs (split_limbs), chosen at training
    int limb_base128 = 0;        // tuning: train with the base-128 split
    int corr_wide = 18;          // tuning: 128 x 256 form (8 / 16 epilogue warps, 18 overlapped), 0 128 x 160
    int ft_warps = 8;            // warps per CTA of the persistent fine-tune (8 or 32)
    int ft_heavy = 6;            // candidates from which a cell takes the split path
    size_t score_chunk_bytes = (size_t)1 << 30;  // score-step correlation block (queries x reference)
    DevBuf<int64_t> ft_keys;
    DevBuf<int32_t> ft_ncand;
    // split path state
    DevBuf<int32_t> sp_cells;
    DevBuf<uint8_t> sp_top;
    DevBuf<int> sp_ntop, sp_rounds, sp_times, sp_state, sp_nS, sp_kq, sp_total, sp_off, sp_eqv;
    DevBuf<int64_t> sp_nq;
    DevBuf<double> sp_rq;
    DevBuf<float> sp_scores, sp_nan;
    DevBuf<unsigned long long> sp_rows;
    DevBuf<int32_t> ft_order;
    DevBuf<int> ft_order_n;
    DevBuf<int32_t> d_final, d_rounds;
    DevBuf<unsigned long long> d_round_sum;  // profiling: fine-tune rounds of the listed cells
    DevBuf<float> ft_scratch;

    // learned proposal
    Mlp mlp;
    DevBuf<float> mlp_x;
    DevBuf<uint8_t> mlp_bad, role;
    DevBuf<int32_t> mlp_y, mlp_idx, mlp_yb, prop, plain, route_final;
    DevBuf<float> mlp_xb, prop_conf, mlp_scores;
    DevBuf<int> n_plain;

    // streamed query batches: two sets of CSR buffers (batch i + 1 uploads while batch i runs)
    DevBuf<float> sq_data[2];
    DevBuf<int32_t> sq_indices[2], sq_indptr[2];
    cudaEvent_t sq_up_start[2] = {nullptr, nullptr}, sq_up_done[2] = {nullptr, nullptr};
    cudaEvent_t sq_free[2] = {nullptr, nullptr}, sq_end = nullptr;

    // the autotuner's device copy of a host sample
    DevBuf<float> tn_data;
    DevBuf<int32_t> tn_indices, tn_indptr;

    // per-call query buffers
    DevBuf<float> q_data;
    DevBuf<int32_t> q_indices, q_indptr;
    DevBuf<int8_t> q_limbs;
    DevBuf<int64_t> q_n2;
    DevBuf<double> q_rinv;
    DevBuf<float> q_f32;
    DevBuf<float> scores;
    DevBuf<LabelQ> lq;
    DevBuf<float> label_scores;
    DevBuf<int32_t> first;
    DevBuf<uint8_t> flags;
    DevBuf<float> sel_scratch;
    DevBuf<RankGroup> rank_groups;
    DevBuf<int> status;
    DevBuf<int32_t> counts, offsets;
    DevBuf<float> qf_data;
    DevBuf<int32_t> qf_indices, qf_indptr;

    // fine-tune round buffers
    DevBuf<int32_t> ft_maps;
    DevBuf<RankGroup> ft_rgroups_q, ft_rgroups_r;
    DevBuf<RankItem> ft_items_q, ft_items_r;
    DevBuf<int16_t> ft_qd, ft_rd;
    DevBuf<int64_t> ft_qn, ft_rn;
    DevBuf<double> ft_qr, ft_rr;
    DevBuf<float> ft_qf, ft_rf;
    DevBuf<FtGroup> ft_groups;
    DevBuf<FtCorrItem> ft_corr_items;
    DevBuf<FtSelItem> ft_sel_items;
    DevBuf<LabelQ> ft_lq;
    DevBuf<float> ft_scores, ft_label_scores;
};

namespace {

int pow2_at_least(int v) {
    int n = 1;
    while (n < v) n <<= 1;
    return n;
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// SGR_TRACE=1 prints per-round fine-tune statistics and phase times to stderr (diagnostics only:
// it synchronises after each phase, so traced runs are slower).
bool trace_on() {
    static int on = -1;
    if (on < 0) {
        const char* e = getenv("SGR_TRACE");
        on = (e && *e && *e != '0') ? 1 : 0;
    }
    return on == 1;
}

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct PhaseClock {
    cudaStream_t s;
    bool on;
    double t;
    PhaseClock(cudaStream_t s_) : s(s_), on(trace_on()), t(now_ms()) {}
    double lap() {
        if (!on) return 0;
        cudaStreamSynchronize(s);
        double n = now_ms(), d = n - t;
        t = n;
        return d;
    }
};

template <class F>
sgr_status guarded(sgr_ctx* ctx, F&& f) {
    if (!ctx) return SGR_ERR_INVALID_ARGUMENT;
    ctx->err.clear();
    try {
        if (ctx->device >= 0) SGR_CUDA(cudaSetDevice(ctx->device));
        const uint64_t l0 = launch_count();
        f();
        if (ctx->stream) {
            SGR_CUDA(cudaStreamSynchronize(ctx->stream));
            ctx->prof.collect();
        }
        ctx->prof.acc.launches += launch_count() - l0;
        return SGR_OK;
    } catch (const Error& e) {
        ctx->err = e.what();
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        if (ctx->side) cudaStreamSynchronize(ctx->side);
        if (ctx->copy) cudaStreamSynchronize(ctx->copy);  // no copy may read caller memory after return
        if (ctx->ft_s) cudaStreamSynchronize(ctx->ft_s);
        cudaGetLastError();
        ctx->prof.spans.clear();
        ctx->prof.used = 0;
        ctx->prof.rounds_pending = false;
        return e.code;
    } catch (const std::bad_alloc&) {
        ctx->err = "host allocation failed";
        return SGR_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return SGR_ERR_INVALID_ARGUMENT;
    }
}

void check_csr_shape(const sgr_csr* m, const char* what) {
    if (!m) fail(SGR_ERR_INVALID_ARGUMENT, std::string(what) + ": null matrix");
    if (m->n_rows && (!m->indptr)) fail(SGR_ERR_INVALID_ARGUMENT, std::string(what) + ": null indptr");
}

// Host-side validation of a host CSR (offsets monotone, columns in range).
void validate_host_csr(const sgr_csr* m, const char* what) {
    check_csr_shape(m, what);
    if (m->indptr[0] != 0) fail(SGR_ERR_INVALID_ARGUMENT, std::string(what) + ": indptr[0] != 0");
    for (uint32_t r = 0; r < m->n_rows; ++r)
        if (m->indptr[r + 1] < m->indptr[r])
            fail(SGR_ERR_INVALID_ARGUMENT, std::string(what) + ": indptr decreases at row " + std::to_string(r));
}

void check_status(sgr_ctx* ctx) {
    int st = 0;
    SGR_CUDA(cudaMemcpyAsync(&st, ctx->status.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    SGR_CUDA(cudaStreamSynchronize(ctx->stream));
    if (st & 1) fail(SGR_ERR_INVALID_ARGUMENT, "a CSR column index is out of range");
    if (st & 2) fail(SGR_ERR_INVALID_ARGUMENT, "a CSR value is NaN");
    if (st & 8) fail(SGR_ERR_STATE, "NaN-bearing score list without sort scratch");
    if (st & SGR_TC_TIMEOUT) fail(SGR_ERR_TIMEOUT, "a bounded wait of the tensor-core correlation ran out");
    // bit 4: libstdc++ would have read outside a NaN-bearing list; the result is the bounded one
}

void reset_status(sgr_ctx* ctx) {
    ctx->status.ensure(1);
    SGR_CUDA(cudaMemsetAsync(ctx->status.p, 0, sizeof(int), ctx->stream));
}

// Makes the query CSR device-resident (borrowed when it already is).
struct DevCsr {
    const float* data;
    const int32_t* indices;
    const int32_t* indptr;
    uint32_t n_rows, n_cols;
    int64_t nnz;  // -1 when unknown (device input)
};

// defer_rows (host input): only indptr is copied here and the value / index buffers are sized;
// score_device copies the rows chunk by chunk, overlapped with the scoring of earlier chunks.
DevCsr query_on_device(sgr_ctx* ctx, const sgr_csr* q, bool defer_rows = false) {
    check_csr_shape(q, "query");
    if (ctx->markers_ready && q->n_cols != ctx->mk.qry_colmap.size())
        fail(SGR_ERR_INVALID_ARGUMENT, "query has " + std::to_string(q->n_cols) + " columns, the query gene names given "
                                       "at training " + std::to_string(ctx->mk.qry_colmap.size()));
    if (q->on_device) {
        int32_t nnz = 0;
        if (q->n_rows) {
            SGR_CUDA(cudaMemcpyAsync(&nnz, q->indptr + q->n_rows, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
            SGR_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        return {q->data, q->indices, q->indptr, q->n_rows, q->n_cols, nnz};
    }
    validate_host_csr(q, "query");
    const size_t nnz = (size_t)q->indptr[q->n_rows];
    if (defer_rows) {
        ctx->q_data.ensure(std::max<size_t>(nnz, 1));
        ctx->q_indices.ensure(std::max<size_t>(nnz, 1));
        ctx->q_indptr.upload(q->indptr, (size_t)q->n_rows + 1, ctx->stream);
        return {ctx->q_data.p, ctx->q_indices.p, ctx->q_indptr.p, q->n_rows, q->n_cols, (int64_t)nnz};
    }
    int sp = ctx->prof.begin(ST_H2D, ctx->stream);
    ctx->q_data.upload(q->data, nnz, ctx->stream);
    ctx->q_indices.upload(q->indices, nnz, ctx->stream);
    ctx->q_indptr.upload(q->indptr, (size_t)q->n_rows + 1, ctx->stream);
    ctx->prof.end(sp, ctx->stream);
    return {ctx->q_data.p, ctx->q_indices.p, ctx->q_indptr.p, q->n_rows, q->n_cols, (int64_t)nnz};
}

int sort_cap(int G) { return std::min(pow2_at_least(std::max(G, 32)), 4096); }

// Gather + rank of rows [r0, r0 + n) of a device CSR; `group` (device) holds the outputs of row r0.
void rank_range(sgr_ctx* ctx, const DevCsr& m, const RankGroup* group, int G, int Kp, uint32_t r0, uint32_t n,
                int out_mode, int norm_mode, const uint32_t* map_bits = nullptr, const uint16_t* map_prefix = nullptr) {
    RankLaunch a{};
    a.data = m.data;
    a.indices = m.indices;
    a.indptr = m.indptr;
    a.n_cols = m.n_cols;
    a.items = nullptr;
    a.row0 = r0;
    a.n_items = n;
    a.groups = group;
    a.out_mode = out_mode;
    a.norm_mode = norm_mode;
    a.max_Kp = Kp;
    a.cap = sort_cap(G);
    a.status = ctx->status.p;
    a.overflow = ctx->rank_overflow.ensure(std::max<uint32_t>(n, 1));
    a.n_overflow = ctx->rank_n_overflow.ensure(1);
    a.map_bits = map_bits;
    a.map_prefix = map_prefix;
    launch_rank(a, ctx->stream);
}

// Gather + rank of rows [0, n) of a device CSR over one gene subset.
void rank_rows(sgr_ctx* ctx, const DevCsr& m, const RankGroup& grp, int out_mode, int norm_mode,
               const uint32_t* map_bits = nullptr, const uint16_t* map_prefix = nullptr) {
    ctx->rank_groups.upload(&grp, 1, ctx->stream);
    rank_range(ctx, m, ctx->rank_groups.p, grp.G, grp.Kp, 0, m.n_rows, out_mode, norm_mode, map_bits, map_prefix);
}

// The compact form (bits + per-word prefixes) of an increasing column map, uploaded.
void upload_column_bits(const std::vector<int32_t>& colmap, DevBuf<uint32_t>& bits, DevBuf<uint16_t>& prefix,
                        cudaStream_t s) {
    const size_t n_words = (colmap.size() + 31) / 32;
    std::vector<uint32_t> b(std::max<size_t>(n_words, 1), 0);
    std::vector<uint16_t> p(std::max<size_t>(n_words, 1), 0);
    column_bits(colmap.data(), (uint32_t)colmap.size(), b.data(), p.data());
    bits.upload(b, s);
    prefix.upload(p, s);
}

// The context's copy stream, created on first use.
cudaStream_t copy_stream(sgr_ctx* ctx) {
    if (!ctx->copy) SGR_CUDA(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
    return ctx->copy;
}

// Copies the values and indices of a host query's rows into the device CSR buffers on the copy
// stream, one row chunk at a time (chunk c: rows [starts[c], starts[c + 1])); ctx->up_ev[c] is
// recorded after chunk c.
void copy_row_chunks(sgr_ctx* ctx, const sgr_csr* h, const std::vector<uint32_t>& starts) {
    cudaStream_t cs = copy_stream(ctx);
    const uint32_t n_chunks = (uint32_t)starts.size() - 1;
    while (ctx->up_ev.size() < n_chunks) {
        cudaEvent_t e;
        SGR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->up_ev.push_back(e);
    }
    // the buffers may still be read by work queued earlier on the compute stream
    SGR_CUDA(cudaEventRecord(ctx->up_ev[0], ctx->stream));
    SGR_CUDA(cudaStreamWaitEvent(cs, ctx->up_ev[0], 0));
    const int sp = ctx->prof.begin(ST_H2D, cs);
    for (uint32_t c = 0; c < n_chunks; ++c) {
        const uint32_t r0 = starts[c], r1 = starts[c + 1];
        const size_t b = (size_t)h->indptr[r0], e = (size_t)h->indptr[r1];
        if (e > b) {
            SGR_CUDA(cudaMemcpyAsync(ctx->q_data.p + b, h->data + b, (e - b) * sizeof(float),
                                     cudaMemcpyHostToDevice, cs));
            SGR_CUDA(cudaMemcpyAsync(ctx->q_indices.p + b, h->indices + b, (e - b) * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, cs));
        }
        if (c + 1 == n_chunks) ctx->prof.end(sp, cs);
        SGR_CUDA(cudaEventRecord(ctx->up_ev[c], cs));
    }
}

// Compacts a device CSR to the columns with map >= 0 into (data, indices, indptr) buffers.  Returns
// the longest compacted row (read back with the total, in the same synchronisation).
int32_t filter_csr(sgr_ctx* ctx, const DevCsr& m, const int32_t* map, DevBuf<float>& od, DevBuf<int32_t>& oi,
                   DevBuf<int32_t>& op, const uint8_t* row_mask = nullptr) {
    ctx->counts.ensure(m.n_rows + 1);
    op.ensure((size_t)m.n_rows + 1);
    ctx->filter_max.ensure(1);
    SGR_CUDA(cudaMemsetAsync(ctx->filter_max.p, 0, sizeof(int), ctx->stream));
    launch_filter_count(m.indptr, m.indices, m.n_rows, m.n_cols, map, ctx->counts.p, ctx->stream, row_mask,
                        ctx->filter_max.p);
    int32_t* scan_scratch = ctx->scan_part.ensure(2 * (((size_t)m.n_rows + 4095) / 4096) + 1);
    launch_exclusive_scan(ctx->counts.p, op.p, m.n_rows, scan_scratch, ctx->stream);
    int32_t total = 0, longest = 0;
    SGR_CUDA(cudaMemcpyAsync(&total, op.p + m.n_rows, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    SGR_CUDA(cudaMemcpyAsync(&longest, ctx->filter_max.p, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    SGR_CUDA(cudaStreamSynchronize(ctx->stream));
    od.ensure(std::max<int32_t>(total, 1));
    oi.ensure(std::max<int32_t>(total, 1));
    launch_filter_fill(m.data, m.indptr, m.indices, m.n_rows, m.n_cols, map, op.p, od.p, oi.p, ctx->stream, row_mask);
    return longest;
}

std::vector<int32_t> position_map(const std::vector<int32_t>& colmap, const std::vector<uint32_t>& genes,
                                  uint32_t W) {
    std::vector<int32_t> pos(W, -1);
    for (size_t i = 0; i < genes.size(); ++i) pos[genes[i]] = (int32_t)i;
    std::vector<int32_t> out(colmap.size(), -1);
    for (size_t c = 0; c < colmap.size(); ++c)
        if (colmap[c] >= 0 && (uint32_t)colmap[c] < W) out[c] = pos[colmap[c]];
    return out;
}

void train(sgr_ctx* ctx, const sgr_csr* ref, const int32_t* celltypes, const char* const* label_names,
           uint32_t n_labels, const char* const* ref_genes, const char* const* qry_genes, uint32_t n_qry) {
    if (!ref || ref->on_device) fail(SGR_ERR_INVALID_ARGUMENT, "reference must be a host CSR");
    if (!celltypes || !label_names || !ref_genes || !qry_genes) fail(SGR_ERR_INVALID_ARGUMENT, "null argument");
    validate_host_csr(ref, "reference");
    for (uint32_t r = 0; r < ref->n_rows; ++r)
        for (int32_t i = ref->indptr[r]; i < ref->indptr[r + 1]; ++i)
            if ((uint32_t)ref->indices[i] >= ref->n_cols)
                fail(SGR_ERR_INVALID_ARGUMENT, "reference column index out of range");
    ctx->trained = false;
    ctx->markers_ready = false;
    HostCsr h{ref->n_rows, ref->n_cols, ref->data, ref->indices, ref->indptr};
    Markers& mk = ctx->mk;
    const bool on_device = ctx->device >= 0 && !ctx->host_training;
    if (on_device) prepare_markers(h, celltypes, n_labels, ref_genes, qry_genes, n_qry, mk);
    else train_markers(h, celltypes, n_labels, ref_genes, qry_genes, n_qry, ctx->cores, mk);
    ctx->R = ref->n_rows;
    ctx->ref_cols = ref->n_cols;
    ctx->ref_f16_ready = false;
    if (ctx->device < 0) {  // host-only context: marker training only
        ctx->G = (int)mk.common.size();
        ctx->Kp = round_up(std::max(ctx->G, 1), 128);
        ctx->Wt = (uint32_t)mk.thre.size();
        ctx->markers_ready = true;
        return;
    }

    // regrouped reference CSR
    std::vector<int32_t> indptr(ctx->R + 1, 0);
    for (uint32_t j = 0; j < ctx->R; ++j) {
        uint32_t r = mk.ref_order[j];
        indptr[j + 1] = indptr[j] + (ref->indptr[r + 1] - ref->indptr[r]);
    }
    std::vector<float> data(indptr[ctx->R]);
    std::vector<int32_t> indices(indptr[ctx->R]);
    for (uint32_t j = 0; j < ctx->R; ++j) {
        uint32_t r = mk.ref_order[j];
        std::copy(ref->data + ref->indptr[r], ref->data + ref->indptr[r + 1], data.begin() + indptr[j]);
        std::copy(ref->indices + ref->indptr[r], ref->indices + ref->indptr[r + 1], indices.begin() + indptr[j]);
    }
    cudaStream_t s = ctx->stream;
    ctx->ref_data.upload(data, s);
    ctx->ref_indices.upload(indices, s);
    ctx->ref_indptr.upload(indptr, s);
    // medians and per-pair marker lists on the device
    if (on_device)
        rank_markers_device(ctx->ref_data.p, ctx->ref_indices.p, ctx->ref_indptr.p, ctx->R, ctx->ref_cols,
                            (int64_t)indptr[ctx->R], mk, s);
    ctx->G = (int)mk.common.size();
    ctx->Kp = round_up(std::max(ctx->G, 1), 128);
    ctx->Wt = (uint32_t)mk.thre.size();
    ctx->markers_ready = true;
    if (ctx->G > 8128) fail(SGR_ERR_UNSUPPORTED, "more than 8128 score-step marker genes");
    // the exact limbs' split: the two-accumulator split where it keeps every limb in int8
    ctx->limb_w = ctx->limb_base128 ? 0 : pick_limb_w(ctx->G);
    if (ctx->Wt > 40000) fail(SGR_ERR_UNSUPPORTED, "fine-tune gene pool above 40000 genes");
    {
        const std::vector<int32_t> rmap = position_map(mk.ref_colmap, mk.common, mk.W);
        const std::vector<int32_t> qmap = position_map(mk.qry_colmap, mk.common, mk.W);
        ctx->ref_map_common.upload(rmap, s);
        ctx->qry_map_common.upload(qmap, s);
        upload_column_bits(rmap, ctx->ref_bits, ctx->ref_prefix, s);
        upload_column_bits(qmap, ctx->qry_bits, ctx->qry_prefix, s);
        SGR_CUDA(cudaStreamSynchronize(s));  // the host maps are freed on leaving this block
    }
    ctx->ref_map_thre.upload(position_map(mk.ref_colmap, mk.thre, mk.W), s);
    ctx->qry_map_thre.upload(position_map(mk.qry_colmap, mk.thre, mk.W), s);

    // score-step reference ranks (int8 limb planes), resident for every query batch
    reset_status(ctx);
    ctx->ref_limbs.ensure((size_t)ctx->R * 3 * ctx->Kp);
    ctx->ref_n2.ensure(ctx->R);
    ctx->ref_rinv.ensure(ctx->R);
    ctx->ref_f32.ensure(ctx->R);
    DevCsr rm{ctx->ref_data.p, ctx->ref_indices.p, ctx->ref_indptr.p, ctx->R, ctx->ref_cols, (int64_t)indptr[ctx->R]};
    RankGroup g{ctx->ref_map_common.p, ctx->G, ctx->Kp, ctx->ref_limbs.p, ctx->ref_n2.p, ctx->ref_rinv.p,
                ctx->ref_f32.p, ctx->limb_w};
    rank_rows(ctx, rm, g, RANK_LIMBS, NORM_SEQ, ctx->ref_bits.p, ctx->ref_prefix.p);
    ctx->h_ref_n2.resize(ctx->R);
    SGR_CUDA(cudaMemcpyAsync(ctx->h_ref_n2.data(), ctx->ref_n2.p, ctx->R * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    // fine-tune: reference compacted to the thre pool, each row's entries sorted by value
    filter_csr(ctx, rm, ctx->ref_map_thre.p, ctx->reff_data, ctx->reff_indices, ctx->reff_indptr);
    // 32-row blocks per label: a block is as long as its longest row, rounded up to 4 entries
    std::vector<int32_t> fptr(ctx->R + 1);
    SGR_CUDA(cudaMemcpyAsync(fptr.data(), ctx->reff_indptr.p, (ctx->R + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                             s));
    SGR_CUDA(cudaStreamSynchronize(s));
    const uint32_t L = mk.n_labels;
    std::vector<int32_t> blk_base(L + 1), ell_base(std::max<uint32_t>(ctx->R, 1)), ell_len(std::max<uint32_t>(ctx->R, 1));
    std::vector<int32_t> ell_off{0};
    ctx->R32 = 0;
    // inside each label the rows are laid out longest first, so that a block's rows are of similar
    // length (less padding); row_perm maps a row's block position back to its position in the label
    std::vector<uint32_t> row_perm(std::max<uint32_t>(ctx->R, 1));
    for (uint32_t l = 0; l < L; ++l) {
        const uint32_t start = mk.ctidx[2 * l], len = mk.ctidx[2 * l + 1];
        std::vector<uint32_t> order(len);
        for (uint32_t j = 0; j < len; ++j) order[j] = j;
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
            return fptr[start + x + 1] - fptr[start + x] > fptr[start + y + 1] - fptr[start + y];
        });
        for (uint32_t j = 0; j < len; ++j) row_perm[start + j] = order[j];
        blk_base[l] = (int32_t)ell_off.size() - 1;
        ctx->R32 += (len + 31) & ~31u;
        for (uint32_t b0 = 0; b0 < len; b0 += 32) {
            const uint32_t nb = std::min<uint32_t>(32, len - b0);
            int mx = 0;
            for (uint32_t t = 0; t < nb; ++t) {
                const uint32_t r = start + order[b0 + t];
                mx = std::max(mx, fptr[r + 1] - fptr[r]);
            }
            const int len4 = (mx + 3) & ~3;
            for (uint32_t t = 0; t < nb; ++t) {
                const uint32_t r = start + order[b0 + t];
                ell_base[r] = ell_off.back() + 4 * (int32_t)t;
                ell_len[r] = len4;
            }
            const int64_t next = (int64_t)ell_off.back() + 32ll * len4;
            if (next > INT32_MAX) fail(SGR_ERR_UNSUPPORTED, "fine-tune reference lists exceed 2^31 entries");
            ell_off.push_back((int32_t)next);
        }
    }
    blk_base[L] = (int32_t)ell_off.size() - 1;
    // packed row scan: a run's kept count (<= the longest row) in the high bits, its e-sum
    // (<= longest row x 2 Wt) below bit `shift`
    {
        int64_t max_row = 1;
        for (uint32_t r = 0; r < ctx->R; ++r) max_row = std::max<int64_t>(max_row, fptr[r + 1] - fptr[r]);
        int cbits = 0;
        while ((int64_t(1) << cbits) <= max_row) ++cbits;
        const int shift = 32 - cbits;
        ctx->pack_shift = (shift > 0 && max_row * 2 * (int64_t)std::max<uint32_t>(ctx->Wt, 1) < (int64_t(1) << shift))
                              ? shift : 0;
        // 32-bit run sums: X <= 4 k^2 Wt and sum b^3 <= k^3 for the longest row k
        const int64_t wt = std::max<uint32_t>(ctx->Wt, 1);
        ctx->pack_narrow = ctx->pack_shift > 0 && 4 * max_row * max_row * wt < (int64_t(1) << 32) &&
                           max_row * max_row * max_row < (int64_t(1) << 32);
    }
    ctx->d_row_perm.upload(row_perm, s);
    ctx->d_blk_base.upload(blk_base, s);
    ctx->d_ell_off.upload(ell_off, s);
    DevBuf<int32_t> d_base, d_len;
    d_base.upload(ell_base, s);
    d_len.upload(ell_len, s);
    ctx->ref_sorted.ensure((size_t)std::max<int32_t>(ell_off.back(), 4));
    launch_ref_presort(ctx->reff_data.p, ctx->reff_indices.p, ctx->reff_indptr.p, d_base.p, d_len.p, ctx->R,
                       std::min(pow2_at_least(std::max<int>(ctx->Wt, 32)), 8192), ctx->Wt, ctx->ref_sorted.p, s);
    SGR_CUDA(cudaStreamSynchronize(s));  // the row tables are freed on return
    ctx->d_ctidx.upload(mk.ctidx, s);
    {
        std::vector<int32_t> lstart(mk.n_labels + 1);
        for (uint32_t l = 0; l < mk.n_labels; ++l) lstart[l] = (int32_t)mk.ctidx[2 * l];
        lstart[mk.n_labels] = (int32_t)ctx->R;
        ctx->d_lstart.upload(lstart, s);
    }
    ctx->d_ft_genes.upload(mk.ft_genes.empty() ? std::vector<uint32_t>{0} : mk.ft_genes, s);
    ctx->d_ft_idx.upload(mk.ft_idx, s);
    std::vector<int32_t> gt(mk.n_labels + 1, 0);
    for (uint32_t n = 1; n <= mk.n_labels; ++n) gt[n] = marker_count(n);
    ctx->d_gene_thre.upload(gt, s);
    check_status(ctx);
    ctx->trained = true;
}

// SGR_EXACT_SIMT=1 runs the exact correlation on CUDA cores (FP64) instead of the tensor cores, to
// cross-check the two on a device (diagnostics).
bool exact_simt() {
    static int on = -1;
    if (on < 0) {
        const char* e = getenv("SGR_EXACT_SIMT");
        on = (e && *e && *e != '0') ? 1 : 0;
    }
    return on == 1;
}

// Score-step correlation of nq query rows (LIMBS at A, norms at offset q0) with every reference row.
// Reference ranks as IEEE half rows for the FP16 correlation variant (ranked on first use).
void ensure_ref_f16(sgr_ctx* ctx) {
    if (ctx->ref_f16_ready) return;
    if (ctx->G > 2048) fail(SGR_ERR_UNSUPPORTED, "FP16 correlation variant needs at most 2048 marker genes");
    ctx->ref_f16.ensure((size_t)ctx->R * ctx->Kp);
    DevBuf<int64_t> n2;
    DevBuf<double> rinv;
    DevBuf<float> f32;
    n2.ensure(ctx->R);
    rinv.ensure(ctx->R);
    f32.ensure(ctx->R);
    DevCsr rm{ctx->ref_data.p, ctx->ref_indices.p, ctx->ref_indptr.p, ctx->R, ctx->ref_cols, -1};
    RankGroup g{ctx->ref_map_common.p, ctx->G, ctx->Kp, ctx->ref_f16.p, n2.p, rinv.p, f32.p};
    rank_rows(ctx, rm, g, RANK_F16, NORM_NONE, ctx->ref_bits.p, ctx->ref_prefix.p);
    SGR_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->ref_f16_ready = true;
}

void correlate(sgr_ctx* ctx, bool fp32, const int8_t* A, int nq, uint32_t q0, float* out, int64_t ld,
               LabelExtremes ext = LabelExtremes{}) {
    if (ctx->corr_f16 && !fp32) {
        launch_corr_tc(A, reinterpret_cast<const int8_t*>(ctx->ref_f16.p), nq, (int)ctx->R, ctx->Kp,
                       ctx->q_rinv.p + q0, ctx->ref_rinv.p, ctx->q_n2.p + q0, ctx->ref_n2.p, out, ld, ctx->status.p,
                       ctx->stream, true, ext, false, ctx->corr_gm, 0, ctx->corr_wide);
        return;
    }
    if (fp32 || exact_simt())
        launch_corr_simt(fp32, A, ctx->ref_limbs.p, nq, (int)ctx->R, ctx->G, ctx->Kp, ctx->q_f32.p + q0,
                         ctx->ref_f32.p, ctx->q_rinv.p + q0, ctx->ref_rinv.p, ctx->q_n2.p + q0, ctx->ref_n2.p, out,
                         ld, ctx->limb_w, ctx->stream);
    else
        launch_corr_tc(A, ctx->ref_limbs.p, nq, (int)ctx->R, ctx->Kp, ctx->q_rinv.p + q0, ctx->ref_rinv.p,
                       ctx->q_n2.p + q0, ctx->ref_n2.p, out, ld, ctx->status.p, ctx->stream, false, ext,
                       ctx->corr_pair != 0, ctx->corr_gm, ctx->limb_w, ctx->corr_wide);
}

// A score step in progress: the query's rows are ranked and scored in blocks of `chunk` rows.
struct ScorePlan {
    DevCsr q;
    const sgr_csr* host = nullptr;
    float p = 0.8f, thre = 0.05f;
    uint32_t chunk = 1, n_chunks = 0;  // chunk: the largest block's rows
    std::vector<uint32_t> starts;      // block c: rows [starts[c], starts[c + 1])
    bool fp32 = false, f16 = false, tc_ext = false;
    int rank_out = RANK_LIMBS, rank_norm = NORM_NONE;
    float* scratch = nullptr;
    uint32_t max_len = 1;
    LabelExtremes ext{};
};

// Prepares the score step over the rows of `q`.  host: the caller's host CSR when q's rows are not
// yet on the device (query_on_device with defer_rows); they are copied block by block on the copy
// stream now, and each block is ranked and scored by score_block once its rows have arrived.
ScorePlan score_begin(sgr_ctx* ctx, const DevCsr& q, float p, float thre, const sgr_csr* host) {
    cudaStream_t s = ctx->stream;
    ScorePlan pl;
    pl.q = q;
    pl.host = host;
    pl.p = p;
    pl.thre = thre;
    const uint32_t Q = q.n_rows, R = ctx->R, L = ctx->mk.n_labels;
    pl.fp32 = ctx->mode == SGR_MODE_FP32REF;
    ctx->q_limbs.ensure((size_t)Q * 3 * ctx->Kp);
    ctx->q_n2.ensure(Q);
    ctx->q_rinv.ensure(Q);
    ctx->q_f32.ensure(Q);
    pl.f16 = ctx->corr_f16 && !pl.fp32;
    if (pl.f16) ensure_ref_f16(ctx);
    pl.chunk = (uint32_t)std::max<size_t>(1, std::min<size_t>(Q, ctx->score_chunk_bytes / (4 * (size_t)R)));
    // Blocks of `chunk` rows.  When the rows come from the host, the score step waits on the copy,
    // and only the last block is left to score once the copy ends: that block is cut into halves,
    // quarters, ... down to about 2,048 rows, so that little is left after the last rows arrive.
    std::vector<uint32_t> sizes;
    for (uint32_t r = 0; r < Q; r += pl.chunk) sizes.push_back(std::min(pl.chunk, Q - r));
    if (host && !sizes.empty()) {
        uint32_t last = sizes.back();
        sizes.pop_back();
        while (last > 2048) {
            const uint32_t half = last / 2;
            sizes.push_back(half);
            last -= half;
        }
        sizes.push_back(last);
    }
    pl.starts.assign(1, 0);
    for (uint32_t n : sizes) pl.starts.push_back(pl.starts.back() + n);
    pl.n_chunks = (uint32_t)sizes.size();
    // Rows already on the device are ranked in one launch.  Host rows are ranked block by block as
    // they arrive: one rank group per block, each writing its own rows' limbs and norms.
    const size_t row_bytes = (size_t)(pl.f16 ? 2 : 3) * ctx->Kp;
    const uint32_t n_groups = host ? pl.n_chunks : 1;
    std::vector<RankGroup> groups(n_groups);
    for (uint32_t c = 0; c < n_groups; ++c) {
        const size_t r0 = pl.starts[c];
        groups[c] = RankGroup{ctx->qry_map_common.p, ctx->G,          ctx->Kp,
                              ctx->q_limbs.p + r0 * row_bytes, ctx->q_n2.p + r0, ctx->q_rinv.p + r0,
                              ctx->q_f32.p + r0, ctx->limb_w};
    }
    ctx->rank_groups.upload(groups, s);
    pl.rank_out = pl.f16 ? RANK_F16 : RANK_LIMBS;
    pl.rank_norm = pl.fp32 ? NORM_SEQ : NORM_NONE;
    if (host) {
        copy_row_chunks(ctx, host, pl.starts);
    } else {
        const uint64_t l0 = launch_count();
        const int sp = ctx->prof.begin(ST_RANK, s);
        rank_range(ctx, q, ctx->rank_groups.p, ctx->G, ctx->Kp, 0, Q, pl.rank_out, pl.rank_norm, ctx->qry_bits.p,
                   ctx->qry_prefix.p);
        ctx->prof.end(sp, s);
        ctx->prof.acc.rank_launches += launch_count() - l0;
    }

    std::vector<LabelQ> lq(L);
    bool any_nan_ref = false;
    for (uint32_t l = 0; l < L; ++l) {
        lq[l] = make_lq((int)ctx->mk.ctidx[2 * l], (int)ctx->mk.ctidx[2 * l + 1], p);
        for (uint32_t r = ctx->mk.ctidx[2 * l]; r < ctx->mk.ctidx[2 * l] + ctx->mk.ctidx[2 * l + 1]; ++r)
            if (ctx->h_ref_n2[r] == 0) lq[l].has_nan = 1, any_nan_ref = true;
    }
    ctx->lq.upload(lq, s);
    std::vector<int32_t> lorder(L);
    for (uint32_t l = 0; l < L; ++l) lorder[l] = (int32_t)l;
    std::stable_sort(lorder.begin(), lorder.end(),
                     [&](int32_t x, int32_t y) { return ctx->mk.ctidx[2 * x + 1] > ctx->mk.ctidx[2 * y + 1]; });
    ctx->d_lorder.upload(lorder, s);
    for (uint32_t l = 0; l < L; ++l) pl.max_len = std::max(pl.max_len, ctx->mk.ctidx[2 * l + 1]);
    if (any_nan_ref) pl.scratch = ctx->sel_scratch.ensure((size_t)select_warps_with_scratch() * pl.max_len);
    ctx->label_scores.ensure((size_t)Q * L);
    ctx->first.ensure(Q);
    ctx->flags.ensure((size_t)Q * L);
    ctx->scores.ensure((size_t)pl.chunk * R);
    // the tensor-core correlation also writes each (query, label) list's extremes for the selection
    pl.tc_ext = !pl.fp32 && !exact_simt();
    if (pl.tc_ext) {
        pl.ext.lstart = ctx->d_lstart.p;
        pl.ext.L = (int)L;
        pl.ext.kmin = ctx->ext_min.ensure((size_t)pl.chunk * L);
        pl.ext.kmax = ctx->ext_max.ensure((size_t)pl.chunk * L);
    }
    return pl;
}

// Block c of the score step on the context's stream: rows [starts[c], starts[c + 1]).
void score_block(sgr_ctx* ctx, const ScorePlan& pl, uint32_t c) {
    cudaStream_t s = ctx->stream;
    const uint32_t R = ctx->R, L = ctx->mk.n_labels;
    const uint32_t q0 = pl.starts[c];
    const int nq = (int)(pl.starts[c + 1] - q0);
    int sp = -1;
    if (pl.host) {
        SGR_CUDA(cudaStreamWaitEvent(s, ctx->up_ev[c], 0));
        const uint64_t l0 = launch_count();
        sp = ctx->prof.begin(ST_RANK, s);
        rank_range(ctx, pl.q, ctx->rank_groups.p + c, ctx->G, ctx->Kp, q0, (uint32_t)nq, pl.rank_out, pl.rank_norm,
                   ctx->qry_bits.p, ctx->qry_prefix.p);
        ctx->prof.end(sp, s);
        ctx->prof.acc.rank_launches += launch_count() - l0;
    }
    const uint64_t c0 = launch_count();
    sp = ctx->prof.begin(ST_CORR, s);
    if (pl.tc_ext) {
        SGR_CUDA(cudaMemsetAsync(pl.ext.kmin, 0xff, (size_t)nq * L * sizeof(uint32_t), s));
        SGR_CUDA(cudaMemsetAsync(pl.ext.kmax, 0, (size_t)nq * L * sizeof(uint32_t), s));
    }
    correlate(ctx, pl.fp32, ctx->q_limbs.p + (size_t)q0 * (pl.f16 ? 2 : 3) * ctx->Kp, nq, q0, ctx->scores.p, R, pl.ext);
    ctx->prof.end(sp, s);
    ctx->prof.acc.corr_launches += launch_count() - c0;
    sp = ctx->prof.begin(ST_SELECT, s);
    ctx->prof.acc.select_launches++;
    ctx->prof.acc.select_bytes += 4ull * (uint64_t)nq * R;
    launch_select_first(ctx->scores.p, R, nq, (int)L, ctx->lq.p, pl.p, pl.thre, ctx->q_n2.p + q0,
                        ctx->label_scores.p + (size_t)q0 * L, ctx->first.p + q0, ctx->flags.p + (size_t)q0 * L,
                        pl.scratch, pl.max_len, ctx->status.p, (int)R, ctx->d_lorder.p, s, pl.ext.kmin,
                        pl.ext.kmax, ctx->select_warps);
    ctx->prof.end(sp, s);
}

void score_end(sgr_ctx* ctx, const ScorePlan& pl) {
    const uint32_t Q = pl.q.n_rows;
    ctx->prof.acc.cells += Q;
    ctx->prof.acc.corr_ops += 2ull * Q * ctx->R * (uint64_t)ctx->G;
    ctx->prof.acc.rank_bytes += 8ull * (uint64_t)(pl.q.nnz) + 4ull * (Q + 1) + 3ull * Q * (uint64_t)ctx->Kp;
}

// Score-step device pass over the rows of `q` (see score_begin for `host`).
void score_device(sgr_ctx* ctx, const DevCsr& q, float p, float thre, const sgr_csr* host = nullptr) {
    const ScorePlan pl = score_begin(ctx, q, p, thre, host);
    for (uint32_t c = 0; c < pl.n_chunks; ++c) score_block(ctx, pl, c);
    score_end(ctx, pl);
}

// ---- fine-tune ---------------------------------------------------------------------------------

struct CellState {
    std::vector<uint8_t> top;  // candidate labels in the reference's list order
    int times = 0;
    int rounds = 0;
};

// Genes of one candidate set: union over ordered pairs of the first min(len, gene_thre) entries of
// the pair's fine-tune list, ascending thre ids (src/cusingler.cu:1141-1161).
std::vector<uint32_t> round_genes(const Markers& mk, const std::vector<uint8_t>& labels) {
    const uint32_t L = mk.n_labels;
    const int gene_thre = marker_count(labels.size());
    std::vector<uint32_t> genes;
    for (uint8_t i : labels)
        for (uint8_t j : labels) {
            if (i == j) continue;
            uint32_t pos = mk.ft_idx[(i * L + j) * 2];
            int len = (int)mk.ft_idx[(i * L + j) * 2 + 1];
            if (len > gene_thre) len = gene_thre;
            genes.insert(genes.end(), mk.ft_genes.begin() + pos, mk.ft_genes.begin() + pos + len);
        }
    std::sort(genes.begin(), genes.end());
    genes.erase(std::unique(genes.begin(), genes.end()), genes.end());
    return genes;
}

// One reference fine-tune decision from the candidate scores in list order
// (src/cusingler.cu:1270-1295).
std::vector<uint8_t> decide(const std::vector<uint8_t>& top, const std::vector<float>& sc, float thre) {
    int mn, mx;
    stl::minmax(sc.data(), (int)sc.size(), &mn, &mx);
    const float lo = sc[mn], hi = sc[mx];
    const float t = hi - thre;
    if (std::isnan(hi)) return {top.front()};
    std::vector<uint8_t> res;
    for (size_t i = 0; i < sc.size(); ++i) {
        if (sc[i] <= lo || sc[i] < t) continue;
        if (sc[i] == hi) res.insert(res.begin(), top[i]);
        else res.push_back(top[i]);
    }
    if (res.empty()) res.push_back(top.front());
    return res;
}

struct Group {
    std::vector<uint8_t> labels;  // ascending
    std::vector<uint32_t> genes;  // thre ids, ascending
    std::vector<uint32_t> cells;
};

void finetune_device(sgr_ctx* ctx, const DevCsr& q, const uint8_t* flags, float p, float thre, int times,
                     int32_t* final_labels, int32_t* rounds_out) {
    cudaStream_t s = ctx->stream;
    const Markers& mk = ctx->mk;
    const uint32_t Q = q.n_rows, L = mk.n_labels, Wt = ctx->Wt;
    const bool fp32 = ctx->mode == SGR_MODE_FP32REF;
    const int sp_ft = ctx->prof.begin(ST_FT, s);
    struct EndSpan {
        sgr_ctx* c;
        int id;
        ~EndSpan() {
            if (id >= 0) cudaEventRecord(c->prof.spans[id].b, c->stream);
        }
    } end_ft{ctx, sp_ft};

    // query compacted to the thre pool (once per call)
    filter_csr(ctx, q, ctx->qry_map_thre.p, ctx->qf_data, ctx->qf_indices, ctx->qf_indptr);
    DevCsr qf{ctx->qf_data.p, ctx->qf_indices.p, ctx->qf_indptr.p, Q, std::max<uint32_t>(Wt, 1), -1};
    DevCsr rf{ctx->reff_data.p, ctx->reff_indices.p, ctx->reff_indptr.p, ctx->R, std::max<uint32_t>(Wt, 1), -1};

    std::vector<CellState> st(Q);
    for (uint32_t i = 0; i < Q; ++i) {
        for (uint32_t l = 0; l < L; ++l)
            if (flags[(size_t)i * L + l]) st[i].top.push_back((uint8_t)l);
        if (st[i].top.size() >= 2 && times >= 0) {
            ctx->prof.acc.ft_cells++;
            ctx->prof.acc.ft_candidates += st[i].top.size();
        }
    }

    uint32_t max_label = 1;
    for (uint32_t l = 0; l < L; ++l) max_label = std::max(max_label, mk.ctidx[2 * l + 1]);

    for (;;) {
        // active cells grouped by candidate set
        std::map<std::vector<uint8_t>, uint32_t> gid;
        std::vector<Group> groups;
        for (uint32_t i = 0; i < Q; ++i) {
            CellState& c = st[i];
            if (!(c.top.size() > 1 && (times == 0 || c.times++ < times))) continue;
            std::vector<uint8_t> key = c.top;
            std::sort(key.begin(), key.end());
            auto it = gid.find(key);
            if (it == gid.end()) {
                it = gid.emplace(key, (uint32_t)groups.size()).first;
                groups.push_back(Group{key, round_genes(mk, key), {}});
            }
            groups[it->second].cells.push_back(i);
        }
        if (groups.empty()) break;
        if (trace_on()) {
            size_t cells = 0;
            for (auto& g : groups) cells += g.cells.size();
            fprintf(stderr, "[sgr ft] round: %zu active cells in %zu candidate sets\n", cells, groups.size());
        }
        // sets with fewer than 20 genes keep their first candidate (src/cusingler.cu:1158-1159)
        std::vector<uint32_t> work;
        for (uint32_t gi = 0; gi < groups.size(); ++gi) {
            if (groups[gi].genes.size() < 20) {
                for (uint32_t c : groups[gi].cells) {
                    st[c].top = {st[c].top.front()};
                    st[c].rounds++;
                }
            } else {
                work.push_back(gi);
            }
        }
        // process the remaining groups in batches bounded by device memory
        size_t wi = 0;
        while (wi < work.size()) {
            std::vector<uint32_t> batch;
            size_t bytes = 0;
            const size_t budget = (size_t)4 << 30;
            while (wi < work.size()) {
                const Group& g = groups[work[wi]];
                size_t nref = 0;
                for (uint8_t l : g.labels) nref += mk.ctidx[2 * l + 1];
                const size_t Kp = round_up((int)g.genes.size(), 32);
                const size_t b = (nref + g.cells.size()) * Kp * 2 + g.cells.size() * nref * 4 + (size_t)Wt * 4;
                if (!batch.empty() && bytes + b > budget) break;
                batch.push_back(work[wi++]);
                bytes += b;
            }
            // tables
            PhaseClock pc(s);
            const uint32_t nb = (uint32_t)batch.size();
            std::vector<int32_t> maps((size_t)nb * Wt, -1);
            std::vector<FtGroup> fg(nb);
            std::vector<RankGroup> rgq(nb), rgr(nb);
            std::vector<RankItem> iq, ir;
            std::vector<FtCorrItem> ci;
            std::vector<FtSelItem> si;
            std::vector<LabelQ> lqs;
            int64_t q_rows = 0, r_rows = 0, sc_off = 0, out_off = 0, q_elems = 0, r_elems = 0;
            int maxKp = 32;
            for (uint32_t b = 0; b < nb; ++b) {
                const Group& g = groups[batch[b]];
                const int G = (int)g.genes.size();
                const int Kp = round_up(G, 32);
                maxKp = std::max(maxKp, Kp);
                for (int i = 0; i < G; ++i) maps[(size_t)b * Wt + g.genes[i]] = i;
                FtGroup& f = fg[b];
                f.G = G;
                f.Kp = Kp;
                f.n_cells = (int32_t)g.cells.size();
                f.q_el = q_elems;
                f.r_el = r_elems;
                f.q_row = q_rows;
                f.r_row = r_rows;
                f.s_off = sc_off;
                f.n_labels = (int32_t)g.labels.size();
                f.lq_off = (int32_t)lqs.size();
                f.out_off = out_off;
                int32_t nref = 0;
                for (uint8_t l : g.labels) {
                    const uint32_t st0 = mk.ctidx[2 * l], len = mk.ctidx[2 * l + 1];
                    lqs.push_back(make_lq(nref, (int)len, p));
                    for (uint32_t r = st0; r < st0 + len; ++r) ir.push_back(RankItem{r, b, (uint32_t)nref++, 0});
                }
                f.n_ref = nref;
                for (uint32_t c = 0; c < g.cells.size(); ++c) {
                    iq.push_back(RankItem{g.cells[c], b, c, 0});
                    si.push_back(FtSelItem{b, c});
                }
                const uint32_t qb = 16;
                for (int32_t r = 0; r < nref; ++r)
                    for (uint32_t c0 = 0; c0 < g.cells.size(); c0 += qb)
                        ci.push_back(FtCorrItem{b, (uint32_t)r, c0, std::min<uint32_t>(c0 + qb, g.cells.size())});
                q_elems += (int64_t)g.cells.size() * Kp;
                r_elems += (int64_t)nref * Kp;
                q_rows += g.cells.size();
                r_rows += nref;
                sc_off += (int64_t)g.cells.size() * nref;
                out_off += (int64_t)g.cells.size() * g.labels.size();
            }
            ctx->ft_maps.upload(maps, s);
            ctx->ft_qd.ensure(std::max<int64_t>(q_elems, 1));
            ctx->ft_rd.ensure(std::max<int64_t>(r_elems, 1));
            ctx->ft_qn.ensure(q_rows);
            ctx->ft_rn.ensure(r_rows);
            ctx->ft_qr.ensure(q_rows);
            ctx->ft_rr.ensure(r_rows);
            ctx->ft_qf.ensure(q_rows);
            ctx->ft_rf.ensure(r_rows);
            for (uint32_t b = 0; b < nb; ++b) {
                const FtGroup& f = fg[b];
                const int32_t* map = ctx->ft_maps.p + (size_t)b * Wt;
                rgq[b] = RankGroup{map, f.G, f.Kp, ctx->ft_qd.p + f.q_el, ctx->ft_qn.p + f.q_row,
                                   ctx->ft_qr.p + f.q_row, ctx->ft_qf.p + f.q_row};
                rgr[b] = RankGroup{map, f.G, f.Kp, ctx->ft_rd.p + f.r_el, ctx->ft_rn.p + f.r_row,
                                   ctx->ft_rr.p + f.r_row, ctx->ft_rf.p + f.r_row};
            }
            const double t_host = pc.lap();
            ctx->ft_rgroups_q.upload(rgq, s);
            ctx->ft_rgroups_r.upload(rgr, s);
            ctx->ft_items_q.upload(iq, s);
            ctx->ft_items_r.upload(ir, s);
            RankLaunch a{};
            a.out_mode = RANK_D16;
            a.norm_mode = fp32 ? NORM_TREE128 : NORM_NONE;
            a.max_Kp = maxKp;
            a.cap = std::min(pow2_at_least(maxKp), 4096);
            a.status = ctx->status.p;
            a.data = qf.data;
            a.indices = qf.indices;
            a.indptr = qf.indptr;
            a.n_cols = qf.n_cols;
            a.items = ctx->ft_items_q.p;
            a.n_items = (uint32_t)iq.size();
            a.groups = ctx->ft_rgroups_q.p;
            launch_rank(a, s);
            const double t_rank_q = pc.lap();
            a.data = rf.data;
            a.indices = rf.indices;
            a.indptr = rf.indptr;
            a.n_cols = rf.n_cols;
            a.items = ctx->ft_items_r.p;
            a.n_items = (uint32_t)ir.size();
            a.groups = ctx->ft_rgroups_r.p;
            launch_rank(a, s);
            const double t_rank_r = pc.lap();

            ctx->ft_groups.upload(fg, s);
            ctx->ft_corr_items.upload(ci, s);
            ctx->ft_sel_items.upload(si, s);
            ctx->ft_lq.upload(lqs, s);
            ctx->ft_scores.ensure(std::max<int64_t>(sc_off, 1));
            ctx->ft_label_scores.ensure(std::max<int64_t>(out_off, 1));
            launch_ft_corr(fp32, ctx->ft_groups.p, ctx->ft_corr_items.p, (uint32_t)ci.size(), ctx->ft_qd.p,
                           ctx->ft_rd.p, ctx->ft_qf.p, ctx->ft_rf.p, ctx->ft_qr.p, ctx->ft_rr.p, ctx->ft_qn.p,
                           ctx->ft_rn.p, ctx->ft_scores.p, s);
            const double t_corr = pc.lap();
            float* scratch = ctx->sel_scratch.ensure((size_t)select_warps_with_scratch() * max_label);
            launch_ft_select(ctx->ft_groups.p, ctx->ft_sel_items.p, (uint32_t)si.size(), ctx->ft_lq.p, p,
                             ctx->ft_scores.p, ctx->ft_label_scores.p, scratch, max_label, ctx->status.p, s);
            std::vector<float> ls(out_off);
            SGR_CUDA(cudaMemcpyAsync(ls.data(), ctx->ft_label_scores.p, out_off * sizeof(float),
                                     cudaMemcpyDeviceToHost, s));
            check_status(ctx);
            const double t_sel = pc.lap();
            // decisions, in each cell's own list order
            for (uint32_t b = 0; b < nb; ++b) {
                const Group& g = groups[batch[b]];
                const FtGroup& f = fg[b];
                for (uint32_t c = 0; c < g.cells.size(); ++c) {
                    CellState& cs = st[g.cells[c]];
                    std::vector<float> sc(cs.top.size());
                    for (size_t i = 0; i < cs.top.size(); ++i) {
                        const size_t j = std::lower_bound(g.labels.begin(), g.labels.end(), cs.top[i]) - g.labels.begin();
                        sc[i] = ls[f.out_off + (int64_t)c * f.n_labels + j];
                    }
                    cs.top = decide(cs.top, sc, thre);
                    cs.rounds++;
                }
            }
            if (trace_on())
                fprintf(stderr,
                        "[sgr ft] batch groups=%u cells=%zu ref_rows=%zu corr_items=%zu maxKp=%d | host %.2f "
                        "rank_q %.2f rank_r %.2f corr %.2f select %.2f decide %.2f ms\n",
                        nb, iq.size(), ir.size(), ci.size(), maxKp, t_host, t_rank_q, t_rank_r, t_corr, t_sel,
                        pc.lap());
        }
    }
    for (uint32_t i = 0; i < Q; ++i) {
        final_labels[i] = st[i].top.empty() ? 0 : st[i].top.front();
        if (rounds_out) rounds_out[i] = st[i].rounds;
        ctx->prof.acc.ft_cell_rounds += st[i].rounds;
    }
}

// The context's second stream (its fork / join events and the split path's state buffers), created
// on first use.
cudaStream_t side_stream(sgr_ctx* ctx) {
    if (!ctx->side) {
        SGR_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
        SGR_CUDA(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
        SGR_CUDA(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
        SGR_CUDA(cudaEventCreateWithFlags(&ctx->ev_state[0], cudaEventDisableTiming));
        SGR_CUDA(cudaEventCreateWithFlags(&ctx->ev_state[1], cudaEventDisableTiming));
        SGR_CUDA(cudaMallocHost(reinterpret_cast<void**>(&ctx->h_state), 2 * 1024 * sizeof(int32_t)));
    }
    return ctx->side;
}

// Exact-mode fine-tune: the persistent kernel over a device work queue.  `flags_dev` is the
// Q x L candidate-flag matrix in device memory.
// out_row0: the cells' outputs go to ctx->d_final / d_rounds from this row on (the row of q's first
// cell in a larger query whose blocks are fine-tuned one after another).
void finetune_persistent(sgr_ctx* ctx, const DevCsr& q, const uint8_t* flags_dev, float p, float thre, int times,
                         int32_t* final_labels, int32_t* rounds_out, const int32_t* cell_list = nullptr,
                         const int* n_list = nullptr, uint32_t out_row0 = 0) {
    cudaStream_t s = ctx->stream;
    const Markers& mk = ctx->mk;
    const uint32_t Q = q.n_rows, L = mk.n_labels, Wt = ctx->Wt;
    const int sp_ft = ctx->prof.begin(ST_FT, s);
    const int32_t* listed = cell_list;  // the caller's cells (cell_list is replaced by the queue order)
    const int* n_listed = n_list;
    // thre-pool rows of the cells to fine-tune (all cells, or only the listed ones)
    const uint8_t* row_mask = nullptr;
    if (cell_list) {
        int n = 0;
        SGR_CUDA(cudaMemcpyAsync(&n, n_list, sizeof(int), cudaMemcpyDeviceToHost, s));
        SGR_CUDA(cudaStreamSynchronize(s));
        uint8_t* mask = ctx->ft_row_mask.ensure(std::max<uint32_t>(Q, 1));
        SGR_CUDA(cudaMemsetAsync(mask, 0, Q, s));
        launch_mark_rows(cell_list, n, mask, s);
        row_mask = mask;
    }
    const int32_t longest = filter_csr(ctx, q, ctx->qry_map_thre.p, ctx->qf_data, ctx->qf_indices, ctx->qf_indptr,
                                       row_mask);
    uint32_t max_label = 1;
    std::vector<LabelQ> lq(L);
    for (uint32_t l = 0; l < L; ++l) {
        max_label = std::max(max_label, mk.ctidx[2 * l + 1]);
        lq[l] = make_lq(0, (int)mk.ctidx[2 * l + 1], p);
    }
    ctx->d_lq_label.upload(lq, s);
    // query sort buffer: the longest thre-pool row of this batch (rows beyond 8192 entries take the
    // kernel's counting path)
    const int qmax = std::max(32, longest);
    const int capq = std::min(pow2_at_least(qmax), 8192);
    const int nw = ctx->ft_warps;
    const size_t smem = ft_persistent_smem((int)std::max<uint32_t>(Wt, 1), capq, nw);
    if (smem > 220 * 1024) fail(SGR_ERR_UNSUPPORTED, "fine-tune gene pool too wide for shared memory");
    const int grid = ft_persistent_grid(smem, nw);
    const int64_t per_cta = (int64_t)ctx->R32 + nw * (int64_t)max_label;
    ctx->ft_scratch.ensure((size_t)grid * per_cta);
    ctx->next_cell.ensure(1);
    SGR_CUDA(cudaMemsetAsync(ctx->next_cell.p, 0, sizeof(int), s));
    ctx->d_final.ensure((size_t)out_row0 + Q);
    ctx->d_rounds.ensure((size_t)out_row0 + Q);
    FtPersistentArgs a{};
    a.ref_sorted = ctx->ref_sorted.p;
    a.pack_shift = ctx->pack_scan ? ctx->pack_shift : 0;
    a.narrow = ctx->pack_scan == 2 && ctx->pack_narrow ? 1 : 0;
    a.row_perm = ctx->d_row_perm.p;
    a.blk_base = ctx->d_blk_base.p;
    a.ell_off = ctx->d_ell_off.p;
    a.ctidx = ctx->d_ctidx.p;
    a.ft_genes = ctx->d_ft_genes.p;
    a.ft_idx = ctx->d_ft_idx.p;
    a.gene_thre = ctx->d_gene_thre.p;
    a.lq_label = ctx->d_lq_label.p;
    a.L = (int)L;
    a.Wt = (int)std::max<uint32_t>(Wt, 1);
    a.qf_data = ctx->qf_data.p;
    a.qf_idx = ctx->qf_indices.p;
    a.qf_ptr = ctx->qf_indptr.p;
    a.Q = (int)Q;
    a.flags = flags_dev;
    a.p = p;
    a.thre = thre;
    a.times = times;
    // heaviest cells first (reference rows of their first-round candidates), so that the last cells
    // on the work queue are light ones; cells with many candidates take the split path
    std::vector<int32_t> heavy_cells;
    {
        int n = (int)Q;
        std::vector<int32_t> list;
        if (cell_list) {
            SGR_CUDA(cudaMemcpyAsync(&n, n_list, sizeof(int), cudaMemcpyDeviceToHost, s));
            SGR_CUDA(cudaStreamSynchronize(s));
            list.resize(n);
            if (n) SGR_CUDA(cudaMemcpyAsync(list.data(), cell_list, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        }
        ctx->ft_keys.ensure(std::max(n, 1));
        ctx->ft_ncand.ensure(std::max(n, 1));
        launch_ft_keys(n, cell_list, (int)L, flags_dev, ctx->d_ctidx.p, ctx->ft_keys.p, ctx->ft_ncand.p, s);
        std::vector<int64_t> keys(n);
        std::vector<int32_t> ncand(n);
        if (n) {
            SGR_CUDA(cudaMemcpyAsync(keys.data(), ctx->ft_keys.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
            SGR_CUDA(cudaMemcpyAsync(ncand.data(), ctx->ft_ncand.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        }
        SGR_CUDA(cudaStreamSynchronize(s));
        std::vector<int32_t> order, heavy;
        std::vector<int32_t> idx(n);
        for (int i = 0; i < n; ++i) idx[i] = i;
        std::stable_sort(idx.begin(), idx.end(), [&](int32_t x, int32_t y) { return keys[x] > keys[y]; });
        for (int i : idx) {
            const int32_t c = cell_list ? list[i] : i;
            if (ncand[i] >= ctx->ft_heavy) heavy.push_back(c);
            else order.push_back(c);
            if (ncand[i] >= 2) {  // a cell with two or more candidates runs at least one round
                ctx->prof.acc.ft_cells++;
                ctx->prof.acc.ft_candidates += (uint64_t)ncand[i];
            }
        }
        int n_order = (int)order.size();
        ctx->prof.acc.ft_queue_cells += (uint64_t)n_order;
        ctx->prof.acc.ft_split_cells += heavy.size();
        ctx->ft_order.upload(order.empty() ? std::vector<int32_t>{0} : order, s);
        ctx->ft_order_n.upload(&n_order, 1, s);
        cell_list = ctx->ft_order.p;
        n_list = ctx->ft_order_n.p;
        heavy_cells.swap(heavy);
    }
    a.cell_list = cell_list;
    a.n_list = n_list;
    a.next_cell = ctx->next_cell.p;
    a.final_labels = ctx->d_final.p + out_row0;
    a.rounds = ctx->d_rounds.p + out_row0;
    a.scratch = ctx->ft_scratch.p;
    a.scratch_per_cta = per_cta;
    a.max_rcand = (int)ctx->R32;
    a.max_label = (int)max_label;
    a.capq = capq;
    a.status = ctx->status.p;
    // Heavy cells take the split path on a second stream, concurrently with the work-queue kernel:
    // the two write disjoint cells, and the split rounds fill the SMs that the queue's last cells
    // leave idle.  Its buffers are sized first (a reallocation would synchronise the device).
    cudaStream_t ss = s;
    if (!heavy_cells.empty()) {
        const size_t Hm = std::min<size_t>(1024, heavy_cells.size());
        ctx->sp_cells.ensure(Hm);
        ctx->sp_top.ensure(Hm * 256);
        ctx->sp_ntop.ensure(Hm);
        ctx->sp_rounds.ensure(Hm);
        ctx->sp_times.ensure(Hm);
        ctx->sp_state.ensure(Hm);
        ctx->sp_nS.ensure(Hm);
        ctx->sp_kq.ensure(Hm);
        ctx->sp_total.ensure(Hm);
        ctx->sp_off.ensure(Hm * 257);
        ctx->sp_eqv.ensure(Hm * std::max<uint32_t>(Wt, 1));
        ctx->sp_nq.ensure(Hm);
        ctx->sp_rq.ensure(Hm);
        ctx->sp_scores.ensure(Hm * ctx->R32);
        ctx->sp_nan.ensure(Hm * 16 * max_label);
        ctx->sp_rows.ensure(1);
        ss = side_stream(ctx);
        SGR_CUDA(cudaEventRecord(ctx->ev_fork, s));
        SGR_CUDA(cudaStreamWaitEvent(ss, ctx->ev_fork, 0));
    }
    launch_ft_persistent(a, grid, smem, nw, s);
    // heavy cells: rounds spread over the whole GPU, in batches
    for (size_t h0 = 0; h0 < heavy_cells.size(); h0 += 1024) {
        const int H = (int)std::min<size_t>(1024, heavy_cells.size() - h0);
        cudaStream_t s = ss;  // the split path's stream
        ctx->sp_cells.upload(heavy_cells.data() + h0, H, s);
        ctx->sp_top.ensure((size_t)H * 256);
        ctx->sp_ntop.ensure(H);
        ctx->sp_rounds.ensure(H);
        ctx->sp_times.ensure(H);
        ctx->sp_state.ensure(H);
        ctx->sp_nS.ensure(H);
        ctx->sp_kq.ensure(H);
        ctx->sp_total.ensure(H);
        ctx->sp_off.ensure((size_t)H * 257);
        ctx->sp_eqv.ensure((size_t)H * std::max<uint32_t>(Wt, 1));
        ctx->sp_nq.ensure(H);
        ctx->sp_rq.ensure(H);
        ctx->sp_scores.ensure((size_t)H * ctx->R32);
        ctx->sp_nan.ensure((size_t)H * 16 * max_label);
        SGR_CUDA(cudaMemsetAsync(ctx->sp_state.p, 0, H * sizeof(int), s));
        ctx->sp_rows.ensure(1);
        SGR_CUDA(cudaMemsetAsync(ctx->sp_rows.p, 0, sizeof(unsigned long long), s));
        const int max_chunks = (int)((ctx->R32 + 255) / 256);
        ctx->sp_items.ensure((size_t)2 * H * max_chunks);
        ctx->sp_nitems.ensure(2);
        SGR_CUDA(cudaMemsetAsync(ctx->sp_nitems.p, 0, 2 * sizeof(int), s));
        FtSplit sp{ctx->sp_cells.p, ctx->sp_top.p, ctx->sp_ntop.p, ctx->sp_rounds.p, ctx->sp_times.p,
                   ctx->sp_state.p, ctx->sp_nS.p, ctx->sp_kq.p, ctx->sp_nq.p, ctx->sp_rq.p, ctx->sp_total.p,
                   ctx->sp_off.p, ctx->sp_eqv.p, ctx->sp_scores.p, ctx->sp_nan.p, (int)ctx->R32, ctx->sp_rows.p,
                   ctx->sp_items.p, ctx->sp_nitems.p, H * max_chunks, max_chunks};
        split_round_setup(a);
        launch_split_first(a, sp, H, s);
        // Rounds run kRoundsPerGraph at a time from one CUDA graph (rounds of finished cells do
        // nothing), with one host check of the cells' states per graph launch; a stream that
        // cannot be captured runs the same rounds as plain launches.
        constexpr int kRoundsPerGraph = 4;
        cudaGraphExec_t exec = nullptr;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const uint64_t before = launch_count();
            cudaGraph_t graph = nullptr;
            try {
                for (int r = 0; r < kRoundsPerGraph; ++r) launch_split_round(a, sp, H, r & 1, s);
            } catch (...) {
                cudaStreamEndCapture(s, &graph);
                if (graph) cudaGraphDestroy(graph);
                cudaGetLastError();
                throw;
            }
            if (cudaStreamEndCapture(s, &graph) == cudaSuccess && graph) {
                if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) exec = nullptr;
                cudaGraphDestroy(graph);
            }
            // launches recorded into the graph are counted when the graph runs
            count_launch(before - launch_count());
        }
        cudaGetLastError();
        // Launches are pipelined: launch k + 1 is queued before the cells' states after launch k are
        // read (copied asynchronously into pinned memory), so the device never waits for the host;
        // the launch queued after the last cell finished runs rounds that do nothing.  Each round
        // drops at least one candidate, so L + 2 rounds finish every cell.
        uint32_t rounds_run = 0, rounds_at[2] = {0, 0};
        for (int launched = 0;; ++launched) {
            if (exec) {
                const cudaError_t e = cudaGraphLaunch(exec, s);
                if (e != cudaSuccess) {
                    cudaGraphExecDestroy(exec);
                    SGR_CUDA(e);
                }
                count_launch(2 * kRoundsPerGraph);
                rounds_run += kRoundsPerGraph;
            } else {
                launch_split_round(a, sp, H, (int)(rounds_run & 1), s);
                rounds_run += 1;
            }
            const int cur = launched & 1;
            rounds_at[cur] = rounds_run;
            SGR_CUDA(cudaMemcpyAsync(ctx->h_state + cur * 1024, ctx->sp_state.p, H * sizeof(int),
                                     cudaMemcpyDeviceToHost, s));
            SGR_CUDA(cudaEventRecord(ctx->ev_state[cur], s));
            if (launched == 0) continue;
            const int prev = cur ^ 1;
            SGR_CUDA(cudaEventSynchronize(ctx->ev_state[prev]));
            const int32_t* state = ctx->h_state + prev * 1024;
            bool all = true;
            for (int i = 0; i < H; ++i) all &= state[i] == 2;
            if (all) break;
            if (rounds_at[prev] > L + 3) {
                if (exec) cudaGraphExecDestroy(exec);
                fail(SGR_ERR_STATE, "fine-tune split path did not converge");
            }
        }
        if (exec) cudaGraphExecDestroy(exec);
        unsigned long long rows = 0;
        SGR_CUDA(cudaMemcpyAsync(&rows, ctx->sp_rows.p, sizeof(rows), cudaMemcpyDeviceToHost, s));
        SGR_CUDA(cudaStreamSynchronize(s));
        ctx->prof.acc.ft_split_rounds += rounds_run;
        ctx->prof.acc.ft_split_rows += rows;
    }
    if (ss != s) {  // join the split path's stream
        SGR_CUDA(cudaEventRecord(ctx->ev_join, ss));
        SGR_CUDA(cudaStreamWaitEvent(s, ctx->ev_join, 0));
    }
    ctx->prof.end(sp_ft, s);
    if (!final_labels) {  // caller reads ctx->d_final / d_rounds itself
        // profiling: rounds of the listed cells, added on the device (rounds_sum_begin / _end)
        if (ctx->prof.on && listed && ctx->d_round_sum.p)
            launch_sum_listed(listed, n_listed, ctx->d_rounds.p + out_row0, ctx->d_round_sum.p, s);
        return;
    }
    SGR_CUDA(cudaMemcpyAsync(final_labels, ctx->d_final.p + out_row0, Q * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    std::vector<int32_t> rounds(Q);
    SGR_CUDA(cudaMemcpyAsync(rounds.data(), ctx->d_rounds.p + out_row0, Q * sizeof(int32_t), cudaMemcpyDeviceToHost,
                             s));
    check_status(ctx);
    for (uint32_t i = 0; i < Q; ++i) {
        if (rounds_out) rounds_out[i] = rounds[i];
        ctx->prof.acc.ft_cell_rounds += rounds[i];
    }
}

// Profiling of the learned form: the fine-tune rounds of its listed cells are summed on the device
// over a call and read back with the call's results.
void rounds_sum_begin(sgr_ctx* ctx) {
    if (!ctx->prof.on) return;
    if (!ctx->prof.h_rounds)
        SGR_CUDA(cudaMallocHost(reinterpret_cast<void**>(&ctx->prof.h_rounds), sizeof(unsigned long long)));
    SGR_CUDA(cudaMemsetAsync(ctx->d_round_sum.ensure(1), 0, sizeof(unsigned long long), ctx->stream));
}

void rounds_sum_end(sgr_ctx* ctx) {
    if (!ctx->prof.on) return;
    SGR_CUDA(cudaMemcpyAsync(ctx->prof.h_rounds, ctx->d_round_sum.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             ctx->stream));
    ctx->prof.rounds_pending = true;
}

// The context's fine-tune stream for the pipelined annotation, created on first use.
cudaStream_t ft_stream(sgr_ctx* ctx) {
    if (!ctx->ft_s) SGR_CUDA(cudaStreamCreateWithFlags(&ctx->ft_s, cudaStreamNonBlocking));
    return ctx->ft_s;
}

cudaEvent_t block_event(sgr_ctx* ctx, size_t i) {
    while (ctx->blk_ev.size() <= i) {
        cudaEvent_t e;
        SGR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->blk_ev.push_back(e);
    }
    return ctx->blk_ev[i];
}

// Exact-mode annotation with the fine-tune of each score block on a stream of its own: block c's
// fine-tune runs while block c + 1 is ranked, correlated and selected (and, for a host query, while
// later blocks are still being copied).  A cell's fine-tune reads only its own row, flags and the
// trained reference, so blocks are independent.  learned: the proposal network routes each block's
// cells as sgr_annotate_learned does (row0: the query's first row in a streamed sequence, for the
// hashed check sample).  Results land in host arrays.
void annotate_pipelined(sgr_ctx* ctx, const DevCsr& q, const sgr_csr* host, float p, float thre, int32_t times,
                        bool learned, float min_confidence, float check_fraction, int32_t* first_labels,
                        int32_t* final_labels, float* label_scores, sgr_learned_stats* stats, uint64_t row0) {
    const uint32_t Q = q.n_rows, L = ctx->mk.n_labels;
    cudaStream_t s = ctx->stream, f = ft_stream(ctx);
    if (learned) rounds_sum_begin(ctx);
    ScorePlan pl = score_begin(ctx, q, p, thre, host);
    ctx->d_final.ensure(Q);
    ctx->d_rounds.ensure(Q);
    if (learned) {
        ctx->mlp_x.ensure((size_t)Q * L);
        ctx->mlp_bad.ensure(Q);
        ctx->prop.ensure(Q);
        ctx->prop_conf.ensure(Q);
        ctx->route_final.ensure(Q);
        ctx->plain.ensure(Q);
        ctx->role.ensure(Q);
        ctx->n_plain.ensure(pl.n_chunks);
        SGR_CUDA(cudaMemsetAsync(ctx->n_plain.p, 0, pl.n_chunks * sizeof(int), s));
    }
    const uint32_t per10k = (uint32_t)std::lround(std::min(std::max(check_fraction, 0.f), 1.f) * 10000.f);
    auto finetune_block = [&](uint32_t c) {
        const uint32_t r0 = pl.starts[c], n = pl.starts[c + 1] - r0;
        SGR_CUDA(cudaStreamWaitEvent(f, block_event(ctx, c), 0));
        DevCsr qc{q.data, q.indices, q.indptr + r0, n, q.n_cols, -1};
        ctx->stream = f;
        try {
            finetune_persistent(ctx, qc, ctx->flags.p + (size_t)r0 * L, p, thre, times,
                                learned ? nullptr : final_labels + r0, nullptr, learned ? ctx->plain.p + r0 : nullptr,
                                learned ? ctx->n_plain.p + c : nullptr, r0);
        } catch (...) {
            ctx->stream = s;
            throw;
        }
        ctx->stream = s;
    };
    for (uint32_t c = 0; c < pl.n_chunks; ++c) {
        score_block(ctx, pl, c);
        if (learned) {
            const uint32_t r0 = pl.starts[c], n = pl.starts[c + 1] - r0;
            const int sp = ctx->prof.begin(ST_MLP, s);
            ctx->mlp.features(ctx->label_scores.p + (size_t)r0 * L, (int)n, ctx->mlp_x.p + (size_t)r0 * L,
                              ctx->mlp_bad.p + r0, s);
            ctx->mlp.predict(ctx->mlp_x.p + (size_t)r0 * L, (int)n, ctx->prop.p + r0, ctx->prop_conf.p + r0, s);
            launch_learned_route((int)n, (int)L, ctx->flags.p + (size_t)r0 * L, ctx->mlp_bad.p + r0, ctx->prop.p + r0,
                                 ctx->prop_conf.p + r0, min_confidence, per10k, 0x243F6A8885A308D3ull, row0 + r0,
                                 ctx->route_final.p + r0, ctx->plain.p + r0, ctx->n_plain.p + c, ctx->role.p + r0, s);
            ctx->prof.end(sp, s);
        }
        SGR_CUDA(cudaEventRecord(block_event(ctx, c), s));
        if (c > 0) finetune_block(c - 1);  // runs while block c is on the score stream
    }
    score_end(ctx, pl);
    if (pl.n_chunks) finetune_block(pl.n_chunks - 1);
    // join the fine-tune stream
    cudaEvent_t done = block_event(ctx, pl.n_chunks);
    SGR_CUDA(cudaEventRecord(done, f));
    SGR_CUDA(cudaStreamWaitEvent(s, done, 0));
    SGR_CUDA(cudaMemcpyAsync(first_labels, ctx->first.p, Q * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    if (label_scores)
        SGR_CUDA(cudaMemcpyAsync(label_scores, ctx->label_scores.p, (size_t)Q * L * sizeof(float),
                                 cudaMemcpyDeviceToHost, s));
    if (!learned) {
        check_status(ctx);
        return;
    }
    rounds_sum_end(ctx);
    std::vector<int32_t> rf(Q), ff(Q);
    std::vector<uint8_t> role(Q);
    SGR_CUDA(cudaMemcpyAsync(rf.data(), ctx->route_final.p, Q * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SGR_CUDA(cudaMemcpyAsync(ff.data(), ctx->d_final.p, Q * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SGR_CUDA(cudaMemcpyAsync(role.data(), ctx->role.p, Q, cudaMemcpyDeviceToHost, s));
    check_status(ctx);
    sgr_learned_stats st{};
    st.cells = Q;
    for (uint32_t i = 0; i < Q; ++i) {
        if (role[i] == 0) {
            final_labels[i] = rf[i];
            st.decided++;
        } else {
            final_labels[i] = ff[i];
            st.finetuned++;
            if (role[i] == 2) {
                st.checked++;
                st.check_agree += rf[i] == ff[i];
            }
        }
    }
    if (stats) *stats = st;
}

// Plain form (score step, then the fine-tune) of a query whose rows are on the device, or are copied
// block by block from `host` during the score step.  Results land in host arrays.
void annotate_plain(sgr_ctx* ctx, const DevCsr& q, const sgr_csr* host, float quantile, float finetune_thre,
                    int32_t finetune_times, int32_t* first_labels, int32_t* final_labels, float* label_scores) {
    if (ctx->pipeline && ctx->mode == SGR_MODE_EXACT) {
        annotate_pipelined(ctx, q, host, quantile, finetune_thre, finetune_times, false, 0.f, 0.f, first_labels,
                           final_labels, label_scores, nullptr, 0);
        return;
    }
    score_device(ctx, q, quantile, finetune_thre, host);
    const uint32_t Q = q.n_rows, L = ctx->mk.n_labels;
    cudaStream_t s = ctx->stream;
    SGR_CUDA(cudaMemcpyAsync(first_labels, ctx->first.p, Q * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    if (label_scores)
        SGR_CUDA(cudaMemcpyAsync(label_scores, ctx->label_scores.p, (size_t)Q * L * sizeof(float),
                                 cudaMemcpyDeviceToHost, s));
    if (ctx->mode == SGR_MODE_EXACT) {
        finetune_persistent(ctx, q, ctx->flags.p, quantile, finetune_thre, finetune_times, final_labels, nullptr);
    } else {
        std::vector<uint8_t> fl((size_t)Q * L);
        SGR_CUDA(cudaMemcpyAsync(fl.data(), ctx->flags.p, fl.size(), cudaMemcpyDeviceToHost, s));
        check_status(ctx);
        finetune_device(ctx, q, fl.data(), quantile, finetune_thre, finetune_times, final_labels, nullptr);
    }
}

// Learned form (score step, proposal network, the plain fine-tune for routed cells) of a query whose
// rows are on the device, or are copied block by block from `host` during the score step.
void annotate_learned(sgr_ctx* ctx, const DevCsr& q, const sgr_csr* host, float quantile, float finetune_thre,
                      int32_t finetune_times, float min_confidence, float check_fraction, int32_t* first_labels,
                      int32_t* final_labels, sgr_learned_stats* stats, uint64_t row0 = 0) {
    if (ctx->pipeline) {
        annotate_pipelined(ctx, q, host, quantile, finetune_thre, finetune_times, true, min_confidence, check_fraction,
                           first_labels, final_labels, nullptr, stats, row0);
        return;
    }
    const uint32_t Q = q.n_rows, L = ctx->mk.n_labels;
    cudaStream_t s = ctx->stream;
    rounds_sum_begin(ctx);
    score_device(ctx, q, quantile, finetune_thre, host);
    const int sp = ctx->prof.begin(ST_MLP, s);
    ctx->mlp_x.ensure((size_t)Q * L);
    ctx->mlp_bad.ensure(Q);
    ctx->prop.ensure(Q);
    ctx->prop_conf.ensure(Q);
    ctx->route_final.ensure(Q);
    ctx->plain.ensure(Q);
    ctx->role.ensure(Q);
    ctx->n_plain.ensure(1);
    ctx->mlp.features(ctx->label_scores.p, (int)Q, ctx->mlp_x.p, ctx->mlp_bad.p, s);
    ctx->mlp.predict(ctx->mlp_x.p, (int)Q, ctx->prop.p, ctx->prop_conf.p, s);
    SGR_CUDA(cudaMemsetAsync(ctx->n_plain.p, 0, sizeof(int), s));
    const uint32_t per10k = (uint32_t)std::lround(std::min(std::max(check_fraction, 0.f), 1.f) * 10000.f);
    launch_learned_route((int)Q, (int)L, ctx->flags.p, ctx->mlp_bad.p, ctx->prop.p, ctx->prop_conf.p,
                         min_confidence, per10k, 0x243F6A8885A308D3ull, row0, ctx->route_final.p, ctx->plain.p,
                         ctx->n_plain.p, ctx->role.p, s);
    ctx->prof.end(sp, s);
    finetune_persistent(ctx, q, ctx->flags.p, quantile, finetune_thre, finetune_times, nullptr, nullptr,
                        ctx->plain.p, ctx->n_plain.p);
    rounds_sum_end(ctx);
    std::vector<int32_t> rf(Q), ff(Q);
    std::vector<uint8_t> role(Q);
    SGR_CUDA(cudaMemcpyAsync(first_labels, ctx->first.p, Q * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SGR_CUDA(cudaMemcpyAsync(rf.data(), ctx->route_final.p, Q * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SGR_CUDA(cudaMemcpyAsync(ff.data(), ctx->d_final.p, Q * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SGR_CUDA(cudaMemcpyAsync(role.data(), ctx->role.p, Q, cudaMemcpyDeviceToHost, s));
    check_status(ctx);
    sgr_learned_stats st{};
    st.cells = Q;
    for (uint32_t i = 0; i < Q; ++i) {
        if (role[i] == 0) {
            final_labels[i] = rf[i];
            st.decided++;
        } else {
            final_labels[i] = ff[i];
            st.finetuned++;
            if (role[i] == 2) {
                st.checked++;
                st.check_agree += rf[i] == ff[i];
            }
        }
    }
    if (stats) *stats = st;
}

// Streamed annotation of host query batches: batch i + 1's rows are uploaded on the copy stream into
// the other of two CSR buffer sets while batch i is annotated on the compute stream.  batch_ms[i]
// (may be NULL) receives the time from the start of batch i's upload to its labels on the host.
void annotate_stream(sgr_ctx* ctx, const sgr_csr* batches, uint32_t n_batches, float quantile, float thre,
                     int32_t times, bool learned, float min_confidence, float check_fraction, int32_t* first_labels,
                     int32_t* final_labels, float* batch_ms, sgr_learned_stats* stats) {
    size_t max_nnz = 1, max_rows = 1;
    for (uint32_t b = 0; b < n_batches; ++b) {
        const sgr_csr* m = batches + b;
        check_csr_shape(m, "query batch");
        if (m->on_device) fail(SGR_ERR_INVALID_ARGUMENT, "streamed query batches are host CSRs");
        if (m->n_cols != ctx->mk.qry_colmap.size())
            fail(SGR_ERR_INVALID_ARGUMENT, "a query batch's column count differs from the query gene names given at "
                                           "training");
        validate_host_csr(m, "query batch");
        max_nnz = std::max<size_t>(max_nnz, (size_t)m->indptr[m->n_rows]);
        max_rows = std::max<size_t>(max_rows, (size_t)m->n_rows + 1);
    }
    for (int i = 0; i < 2; ++i) {
        ctx->sq_data[i].ensure(max_nnz);
        ctx->sq_indices[i].ensure(max_nnz);
        ctx->sq_indptr[i].ensure(max_rows);
        if (!ctx->sq_up_start[i]) {
            SGR_CUDA(cudaEventCreate(&ctx->sq_up_start[i]));
            SGR_CUDA(cudaEventCreateWithFlags(&ctx->sq_up_done[i], cudaEventDisableTiming));
            SGR_CUDA(cudaEventCreateWithFlags(&ctx->sq_free[i], cudaEventDisableTiming));
        }
    }
    if (!ctx->sq_end) SGR_CUDA(cudaEventCreate(&ctx->sq_end));
    cudaStream_t s = ctx->stream, cs = copy_stream(ctx);
    // both buffer sets are free once the work queued so far on the compute stream is done
    for (int i = 0; i < 2; ++i) SGR_CUDA(cudaEventRecord(ctx->sq_free[i], s));
    auto upload = [&](uint32_t b) {
        const int k = b & 1;
        const sgr_csr* m = batches + b;
        const size_t nnz = (size_t)m->indptr[m->n_rows];
        SGR_CUDA(cudaStreamWaitEvent(cs, ctx->sq_free[k], 0));
        SGR_CUDA(cudaEventRecord(ctx->sq_up_start[k], cs));
        const int sp = ctx->prof.begin(ST_H2D, cs);
        SGR_CUDA(cudaMemcpyAsync(ctx->sq_indptr[k].p, m->indptr, ((size_t)m->n_rows + 1) * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, cs));
        if (nnz) {
            SGR_CUDA(cudaMemcpyAsync(ctx->sq_data[k].p, m->data, nnz * sizeof(float), cudaMemcpyHostToDevice, cs));
            SGR_CUDA(cudaMemcpyAsync(ctx->sq_indices[k].p, m->indices, nnz * sizeof(int32_t), cudaMemcpyHostToDevice,
                                     cs));
        }
        ctx->prof.end(sp, cs);
        SGR_CUDA(cudaEventRecord(ctx->sq_up_done[k], cs));
    };
    if (stats) *stats = sgr_learned_stats{};
    if (n_batches) upload(0);
    size_t row0 = 0;
    for (uint32_t b = 0; b < n_batches; ++b) {
        const int k = b & 1;
        if (b + 1 < n_batches) upload(b + 1);
        const sgr_csr* m = batches + b;
        SGR_CUDA(cudaStreamWaitEvent(s, ctx->sq_up_done[k], 0));
        DevCsr q{ctx->sq_data[k].p, ctx->sq_indices[k].p, ctx->sq_indptr[k].p, m->n_rows, m->n_cols,
                 (int64_t)m->indptr[m->n_rows]};
        if (m->n_rows) {
            if (learned) {
                sgr_learned_stats st{};
                annotate_learned(ctx, q, nullptr, quantile, thre, times, min_confidence, check_fraction,
                                 first_labels + row0, final_labels + row0, &st, row0);
                if (stats) {
                    stats->cells += st.cells;
                    stats->decided += st.decided;
                    stats->finetuned += st.finetuned;
                    stats->checked += st.checked;
                    stats->check_agree += st.check_agree;
                }
            } else {
                annotate_plain(ctx, q, nullptr, quantile, thre, times, first_labels + row0, final_labels + row0,
                               nullptr);
            }
        }
        SGR_CUDA(cudaEventRecord(ctx->sq_free[k], s));
        SGR_CUDA(cudaEventRecord(ctx->sq_end, s));
        SGR_CUDA(cudaEventSynchronize(ctx->sq_end));
        if (batch_ms) {
            float ms = 0.f;
            SGR_CUDA(cudaEventElapsedTime(&ms, ctx->sq_up_start[k], ctx->sq_end));
            batch_ms[b] = ms;
        }
        row0 += m->n_rows;
    }
}

}  // namespace

extern "C" {

sgr_status sgr_create(int gpuid, int cores, sgr_ctx** out) {
    if (!out) return SGR_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (gpuid == -1) {  // host-only context: marker training and introspection, no device work
        auto* ctx = new sgr_ctx();
        ctx->device = -1;
        ctx->cores = cores > 0 ? cores : 1;
        *out = ctx;
        return SGR_OK;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || gpuid < 0 || gpuid >= n) {
        cudaGetLastError();
        return SGR_ERR_CUDA;
    }
    auto* ctx = new sgr_ctx();
    ctx->device = gpuid;
    ctx->cores = cores > 0 ? cores : 1;
    if (cudaSetDevice(gpuid) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return SGR_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return SGR_OK;
}

sgr_status sgr_destroy(sgr_ctx* ctx) {
    if (!ctx) return SGR_OK;
    if (ctx->device < 0) {
        delete ctx;
        return SGR_OK;
    }
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->side) cudaStreamSynchronize(ctx->side);
    cudaStream_t s = ctx->own_stream, side = ctx->side;
    cudaEvent_t e1 = ctx->ev_fork, e2 = ctx->ev_join, e3 = ctx->ev_state[0], e4 = ctx->ev_state[1];
    int32_t* hs = ctx->h_state;
    cudaStream_t cp = ctx->copy;
    if (cp) cudaStreamSynchronize(cp);
    std::vector<cudaEvent_t> up = ctx->up_ev;
    for (int i = 0; i < 2; ++i)
        for (cudaEvent_t e : {ctx->sq_up_start[i], ctx->sq_up_done[i], ctx->sq_free[i]})
            if (e) up.push_back(e);
    if (ctx->sq_end) up.push_back(ctx->sq_end);
    for (cudaEvent_t e : ctx->blk_ev) up.push_back(e);
    cudaStream_t fts = ctx->ft_s;
    if (fts) cudaStreamSynchronize(fts);
    delete ctx;  // DevBuf destructors free device memory
    if (fts) cudaStreamDestroy(fts);
    if (cp) cudaStreamDestroy(cp);
    for (cudaEvent_t e : up) cudaEventDestroy(e);
    if (s) cudaStreamDestroy(s);
    if (side) cudaStreamDestroy(side);
    if (e1) cudaEventDestroy(e1);
    if (e2) cudaEventDestroy(e2);
    if (e3) cudaEventDestroy(e3);
    if (e4) cudaEventDestroy(e4);
    if (hs) cudaFreeHost(hs);
    return SGR_OK;
}

sgr_status sgr_set_stream(sgr_ctx* ctx, void* stream) {
    if (!ctx || ctx->device < 0) return SGR_ERR_INVALID_ARGUMENT;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return SGR_OK;
}

sgr_status sgr_autotune(sgr_ctx* ctx, const sgr_csr* sample, float quantile, float finetune_thre,
                        int32_t finetune_times, int32_t learned, float min_confidence, float check_fraction,
                        sgr_tuning* out) {
    if (!ctx || !sample || !out) return SGR_ERR_INVALID_ARGUMENT;
    if (ctx->device < 0) return SGR_ERR_STATE;
    // a host sample is copied to the device once, so that the trials time the kernels and not the
    // copy of the sample
    sgr_csr dev_sample = *sample;
    if (!sample->on_device) {
        const sgr_status st0 = guarded(ctx, [&] {
            validate_host_csr(sample, "sample");
            const size_t nnz = (size_t)sample->indptr[sample->n_rows];
            ctx->tn_data.upload(sample->data, nnz, ctx->stream);
            ctx->tn_indices.upload(sample->indices, nnz, ctx->stream);
            ctx->tn_indptr.upload(sample->indptr, (size_t)sample->n_rows + 1, ctx->stream);
        });
        if (st0 != SGR_OK) return st0;
        dev_sample = sgr_csr{sample->n_rows, sample->n_cols, ctx->tn_data.p, ctx->tn_indices.p, ctx->tn_indptr.p, 1};
    }
    sample = &dev_sample;
    const uint32_t Q = sample->n_rows;
    std::vector<int32_t> first(std::max<uint32_t>(Q, 1)), fin(first.size()), first0, fin0;
    sgr_learned_stats st{};
    auto run = [&]() -> sgr_status {
        return learned ? sgr_annotate_learned(ctx, sample, quantile, finetune_thre, finetune_times, min_confidence,
                                              check_fraction, first.data(), fin.data(), &st)
                       : sgr_annotate(ctx, sample, quantile, finetune_thre, finetune_times, first.data(), fin.data(),
                                      nullptr);
    };
    auto run_score = [&]() -> sgr_status {
        return sgr_score_first(ctx, sample, quantile, finetune_thre, first.data(), nullptr, nullptr);
    };
    auto wall = [](auto&& f, sgr_status& stt) {
        const auto t0 = std::chrono::steady_clock::now();
        stt = f();
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    // every knob is restored if a candidate fails or changes a label
    const int keep_w = ctx->ft_warps, keep_h = ctx->ft_heavy, keep_pair = ctx->corr_pair, keep_gm = ctx->corr_gm,
              keep_sw = ctx->select_warps, keep_pipe = ctx->pipeline, keep_wide = ctx->corr_wide;
    const size_t keep_c = ctx->score_chunk_bytes;
    auto restore = [&]() {
        ctx->ft_warps = keep_w;
        ctx->ft_heavy = keep_h;
        ctx->score_chunk_bytes = keep_c;
        ctx->corr_pair = keep_pair;
        ctx->corr_gm = keep_gm;
        ctx->select_warps = keep_sw;
        ctx->pipeline = keep_pipe;
        ctx->corr_wide = keep_wide;
    };
    sgr_tuning best{};
    best.best_ms = 1e300;
    // one untimed pass grows every buffer to the sample's size
    sgr_status stt = run();
    if (stt != SGR_OK) return stt;
    first0 = first;
    fin0 = fin;

    // phase 1: score-step shapes (correlation form and tile order, score block, selection CTA width),
    // each timed on the score step of the sample; first labels must not change.  Forms: 0 the
    // 128 x 160 tiles, 1 their SM-pair form, 8 / 16 the 128 x 256 tiles with 8 / 16 epilogue warps,
    // 18 their overlapped form.
    const bool exact = ctx->mode == SGR_MODE_EXACT;
    const int forms[] = {0, 1, 8, 16, 18}, gms[] = {1, 16}, chunk_mb[] = {256, 1024}, sel_w[] = {0, 1, 16};
    double score_best = 1e300;
    for (int form : forms)
        for (int gm : gms) {
            if (!exact && (form || gm != 1)) continue;  // the FP32-order correlation runs on CUDA cores
            if (form >= 8 && ctx->limb_w == 0) continue;  // the base-128 split has three accumulators
            for (int c : chunk_mb)
                for (int w : sel_w) {
                    ctx->corr_pair = form == 1;
                    ctx->corr_wide = form >= 8 ? form : 0;
                    ctx->corr_gm = gm;
                    ctx->score_chunk_bytes = (size_t)c << 20;
                    ctx->select_warps = w;
                    const double ms = wall(run_score, stt);
                    if (stt != SGR_OK) {
                        restore();
                        return stt;
                    }
                    if (first != first0) {
                        restore();
                        ctx->err = "autotune: score-step shapes disagree on the labels";
                        return SGR_ERR_STATE;
                    }
                    best.score_trials++;
                    if (ms < score_best) {
                        score_best = ms;
                        best.corr_pair = form == 1;
                        best.corr_wide = form >= 8 ? form : 0;
                        best.corr_gm = gm;
                        best.score_chunk_mb = c;
                        best.select_warps = w;
                    }
                }
        }
    ctx->corr_pair = best.corr_pair;
    ctx->corr_wide = best.corr_wide;
    ctx->corr_gm = best.corr_gm;
    ctx->score_chunk_bytes = (size_t)best.score_chunk_mb << 20;
    ctx->select_warps = best.select_warps;
    best.score_best_ms = score_best;

    // phase 2: fine-tune shapes with the chosen score step, timed on the whole annotation; first and
    // final labels must not change
    const int warps[] = {8, 32};
    const int heavy[] = {4, 6, 9, 16, 1 << 30};
    const int pipes[] = {0, 1};
    for (int pipe : pipes)
    for (int w : warps)
        for (int h : heavy) {
            if (pipe && !exact) continue;  // the FP32-order fine-tune is not pipelined
            ctx->pipeline = pipe;
            ctx->ft_warps = w;
            ctx->ft_heavy = h;
            const double ms = wall(run, stt);
            if (stt != SGR_OK) {
                restore();
                return stt;
            }
            if (first != first0 || fin != fin0) {
                restore();
                ctx->err = "autotune: launch shapes disagree on the labels";
                return SGR_ERR_STATE;
            }
            best.trials++;
            best.worst_ms = std::max(best.worst_ms, ms);
            if (ms < best.best_ms) {
                best.best_ms = ms;
                best.ft_warps = w;
                best.ft_heavy = h;
                best.pipeline = pipe;
            }
        }
    ctx->ft_warps = best.ft_warps;
    ctx->ft_heavy = best.ft_heavy;
    ctx->pipeline = best.pipeline;
    *out = best;
    return SGR_OK;
}

sgr_status sgr_set_tuning(sgr_ctx* ctx, int what, int value) {
    if (!ctx) return SGR_ERR_INVALID_ARGUMENT;
    if (what == 0) {
        if (value != 8 && value != 32) return SGR_ERR_INVALID_ARGUMENT;
        ctx->ft_warps = value;
        return SGR_OK;
    }
    if (what == 1) {
        if (value < 2) return SGR_ERR_INVALID_ARGUMENT;
        ctx->ft_heavy = value;
        return SGR_OK;
    }
    if (what == 2) {
        if (value < 1) return SGR_ERR_INVALID_ARGUMENT;
        ctx->score_chunk_bytes = (size_t)value << 20;
        return SGR_OK;
    }
    if (what == 4) {
        if (value != 0 && value != 1) return SGR_ERR_INVALID_ARGUMENT;
        if (value && ctx->mode != SGR_MODE_EXACT) return SGR_ERR_STATE;
        ctx->corr_f16 = value;
        return SGR_OK;
    }
    if (what == 3) {
        if (value < 0 || value > 2) return SGR_ERR_INVALID_ARGUMENT;
        ctx->pack_scan = value;
        return SGR_OK;
    }
    if (what == 5) {
        if (value != 0 && value != 1) return SGR_ERR_INVALID_ARGUMENT;
        ctx->corr_pair = value;
        return SGR_OK;
    }
    if (what == 6) {
        if (value < 1 || value > 4096) return SGR_ERR_INVALID_ARGUMENT;
        ctx->corr_gm = value;
        return SGR_OK;
    }
    if (what == 7) {
        if (value != 0 && value != 1 && value != 8 && value != 16) return SGR_ERR_INVALID_ARGUMENT;
        ctx->select_warps = value;
        return SGR_OK;
    }
    if (what == 8) {
        if (value != 0 && value != 1) return SGR_ERR_INVALID_ARGUMENT;
        ctx->host_training = value;
        return SGR_OK;
    }
    if (what == 9) {
        if (value != 0 && value != 1) return SGR_ERR_INVALID_ARGUMENT;
        ctx->pipeline = value;
        return SGR_OK;
    }
    if (what == 10) {
        if (value != 0 && value != 8 && value != 16 && value != 18) return SGR_ERR_INVALID_ARGUMENT;
        ctx->corr_wide = value;
        return SGR_OK;
    }
    if (what == 11) {
        if (value != 0 && value != 1) return SGR_ERR_INVALID_ARGUMENT;
        ctx->limb_base128 = value;
        return SGR_OK;
    }
    return SGR_ERR_INVALID_ARGUMENT;
}

sgr_status sgr_set_profiling(sgr_ctx* ctx, int on) {
    if (!ctx) return SGR_ERR_INVALID_ARGUMENT;
    ctx->prof.on = on != 0;
    return SGR_OK;
}

sgr_status sgr_reset_timings(sgr_ctx* ctx) {
    if (!ctx) return SGR_ERR_INVALID_ARGUMENT;
    ctx->prof.acc = sgr_timings{};
    return SGR_OK;
}

sgr_status sgr_get_timings(const sgr_ctx* ctx, sgr_timings* out) {
    if (!ctx || !out) return SGR_ERR_INVALID_ARGUMENT;
    *out = ctx->prof.acc;
    return SGR_OK;
}

const char* sgr_last_error(const sgr_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

sgr_status sgr_set_mode(sgr_ctx* ctx, sgr_mode mode) {
    if (!ctx) return SGR_ERR_INVALID_ARGUMENT;
    if (mode != SGR_MODE_EXACT && mode != SGR_MODE_FP32REF) return SGR_ERR_INVALID_ARGUMENT;
    ctx->mode = mode;
    return SGR_OK;
}

sgr_status sgr_train_ref(sgr_ctx* ctx, const sgr_csr* ref, const int32_t* celltypes, const char* const* label_names,
                         uint32_t n_labels, const char* const* ref_genes, const char* const* qry_genes,
                         uint32_t n_qry_genes) {
    return guarded(ctx, [&] { train(ctx, ref, celltypes, label_names, n_labels, ref_genes, qry_genes, n_qry_genes); });
}

sgr_status sgr_score_first(sgr_ctx* ctx, const sgr_csr* qry, float quantile, float finetune_thre,
                           int32_t* first_labels, float* label_scores, uint8_t* flags) {
    return guarded(ctx, [&] {
        if (!ctx->trained) fail(SGR_ERR_STATE, "score before train");
        if (!first_labels) fail(SGR_ERR_INVALID_ARGUMENT, "null first_labels");
        reset_status(ctx);
        DevCsr q = query_on_device(ctx, qry, true);
        if (q.n_rows == 0) return;
        score_device(ctx, q, quantile, finetune_thre, qry->on_device ? nullptr : qry);
        const uint32_t Q = q.n_rows, L = ctx->mk.n_labels;
        cudaStream_t s = ctx->stream;
        SGR_CUDA(cudaMemcpyAsync(first_labels, ctx->first.p, Q * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        if (label_scores)
            SGR_CUDA(cudaMemcpyAsync(label_scores, ctx->label_scores.p, (size_t)Q * L * sizeof(float),
                                     cudaMemcpyDeviceToHost, s));
        if (flags)
            SGR_CUDA(cudaMemcpyAsync(flags, ctx->flags.p, (size_t)Q * L, cudaMemcpyDeviceToHost, s));
        check_status(ctx);
    });
}

sgr_status sgr_finetune(sgr_ctx* ctx, const sgr_csr* qry, const uint8_t* flags, float quantile, float finetune_thre,
                        int32_t finetune_times, int32_t* final_labels, int32_t* rounds) {
    return guarded(ctx, [&] {
        if (!ctx->trained) fail(SGR_ERR_STATE, "finetune before train");
        if (!flags || !final_labels) fail(SGR_ERR_INVALID_ARGUMENT, "null flags or final_labels");
        reset_status(ctx);
        DevCsr q = query_on_device(ctx, qry);
        if (q.n_rows == 0) return;
        if (ctx->mode == SGR_MODE_EXACT) {
            ctx->flags.upload(flags, (size_t)q.n_rows * ctx->mk.n_labels, ctx->stream);
            finetune_persistent(ctx, q, ctx->flags.p, quantile, finetune_thre, finetune_times, final_labels, rounds);
        } else {
            finetune_device(ctx, q, flags, quantile, finetune_thre, finetune_times, final_labels, rounds);
        }
    });
}

sgr_status sgr_annotate(sgr_ctx* ctx, const sgr_csr* qry, float quantile, float finetune_thre, int32_t finetune_times,
                        int32_t* first_labels, int32_t* final_labels, float* label_scores) {
    return guarded(ctx, [&] {
        if (!ctx->trained) fail(SGR_ERR_STATE, "annotate before train");
        if (!first_labels || !final_labels) fail(SGR_ERR_INVALID_ARGUMENT, "null output");
        reset_status(ctx);
        DevCsr q = query_on_device(ctx, qry, true);
        if (q.n_rows == 0) return;
        annotate_plain(ctx, q, qry->on_device ? nullptr : qry, quantile, finetune_thre, finetune_times, first_labels,
                       final_labels, label_scores);
    });
}

sgr_status sgr_get_info(const sgr_ctx* ctx, sgr_info* out) {
    if (!ctx || !out) return SGR_ERR_INVALID_ARGUMENT;
    if (!ctx->markers_ready) return SGR_ERR_STATE;
    out->n_labels = ctx->mk.n_labels;
    out->n_genes = ctx->mk.W;
    out->n_common = (uint32_t)ctx->mk.common.size();
    out->n_thre = (uint32_t)ctx->mk.thre.size();
    out->filter_genes = ctx->mk.filter_genes ? 1 : 0;
    out->ref_rows = (uint32_t)ctx->mk.ref_order.size();
    out->n_pair_genes = ctx->mk.pair_genes.size();
    return SGR_OK;
}

sgr_status sgr_get_u32(const sgr_ctx* ctx, int what, uint32_t* out, uint64_t cap) {
    if (!ctx || !out) return SGR_ERR_INVALID_ARGUMENT;
    if (!ctx->markers_ready) return SGR_ERR_STATE;
    const Markers& m = ctx->mk;
    const std::vector<uint32_t>* v = nullptr;
    switch (what) {
        case 0: v = &m.common; break;
        case 1: v = &m.thre; break;
        case 2: v = &m.pair_genes; break;
        case 3: v = &m.pair_idx; break;
        case 4: v = &m.ft_genes; break;
        case 5: v = &m.ft_idx; break;
        case 6: v = &m.ctidx; break;
        case 7: v = &m.ref_order; break;
        default: return SGR_ERR_INVALID_ARGUMENT;
    }
    if (v->size() > cap) return SGR_ERR_INVALID_ARGUMENT;
    std::copy(v->begin(), v->end(), out);
    return SGR_OK;
}

sgr_status sgr_debug_ranks(sgr_ctx* ctx, const sgr_csr* rows, int which, int32_t* d_out) {
    return guarded(ctx, [&] {
        if (!ctx->trained) fail(SGR_ERR_STATE, "not trained");
        cudaStream_t s = ctx->stream;
        const int G = ctx->G, Kp = ctx->Kp;
        uint32_t n;
        std::vector<int8_t> limbs;
        if (which == 1) {
            n = ctx->R;
            limbs.resize((size_t)n * 3 * Kp);
            SGR_CUDA(cudaMemcpyAsync(limbs.data(), ctx->ref_limbs.p, limbs.size(), cudaMemcpyDeviceToHost, s));
        } else {
            reset_status(ctx);
            DevCsr q = query_on_device(ctx, rows);
            n = q.n_rows;
            ctx->q_limbs.ensure((size_t)n * 3 * Kp);
            ctx->q_n2.ensure(n);
            ctx->q_rinv.ensure(n);
            ctx->q_f32.ensure(n);
            RankGroup g{ctx->qry_map_common.p, G, Kp, ctx->q_limbs.p, ctx->q_n2.p, ctx->q_rinv.p, ctx->q_f32.p,
                        ctx->limb_w};
            rank_rows(ctx, q, g, RANK_LIMBS, NORM_NONE, ctx->qry_bits.p, ctx->qry_prefix.p);
            limbs.resize((size_t)n * 3 * Kp);
            SGR_CUDA(cudaMemcpyAsync(limbs.data(), ctx->q_limbs.p, limbs.size(), cudaMemcpyDeviceToHost, s));
            check_status(ctx);
        }
        SGR_CUDA(cudaStreamSynchronize(s));
        for (uint32_t r = 0; r < n; ++r) {
            const int8_t* row = limbs.data() + (size_t)r * 3 * Kp;
            for (int i = 0; i < G; ++i) {
                const int p0 = row[i], l = row[Kp + i], sm = row[2 * Kp + i], w = ctx->limb_w;
                const int h = w ? p0 / w : p0;
                if ((w && p0 != w * h) || sm != h + l) fail(SGR_ERR_STATE, "limb planes disagree");
                d_out[(size_t)r * G + i] = limb_mult(w) * p0 + sm;
            }
        }
    });
}

sgr_status sgr_debug_scores(sgr_ctx* ctx, const sgr_csr* qry, float* out) {
    return guarded(ctx, [&] {
        if (!ctx->trained) fail(SGR_ERR_STATE, "not trained");
        reset_status(ctx);
        DevCsr q = query_on_device(ctx, qry);
        const uint32_t Q = q.n_rows, R = ctx->R;
        const bool fp32 = ctx->mode == SGR_MODE_FP32REF;
        cudaStream_t s = ctx->stream;
        ctx->q_limbs.ensure((size_t)Q * 3 * ctx->Kp);
        ctx->q_n2.ensure(Q);
        ctx->q_rinv.ensure(Q);
        ctx->q_f32.ensure(Q);
        const bool f16 = ctx->corr_f16 && !fp32;
        if (f16) ensure_ref_f16(ctx);
        RankGroup g{ctx->qry_map_common.p, ctx->G, ctx->Kp, ctx->q_limbs.p, ctx->q_n2.p, ctx->q_rinv.p, ctx->q_f32.p,
                    ctx->limb_w};
        rank_rows(ctx, q, g, f16 ? RANK_F16 : RANK_LIMBS, fp32 ? NORM_SEQ : NORM_NONE, ctx->qry_bits.p,
                  ctx->qry_prefix.p);
        DevBuf<float> sc;
        sc.ensure((size_t)Q * R);
        correlate(ctx, fp32, ctx->q_limbs.p, (int)Q, 0, sc.p, R);
        SGR_CUDA(cudaMemcpyAsync(out, sc.p, (size_t)Q * R * sizeof(float), cudaMemcpyDeviceToHost, s));
        check_status(ctx);
    });
}

// ---- learned proposal --------------------------------------------------------------------------

sgr_status sgr_mlp_train(sgr_ctx* ctx, const float* label_scores, const int32_t* targets, uint32_t n,
                         const sgr_mlp_config* cfg, float* final_loss) {
    return guarded(ctx, [&] {
        if (ctx->device < 0) fail(SGR_ERR_STATE, "host-only context");
        if (!ctx->markers_ready) fail(SGR_ERR_STATE, "train the reference first (the label count)");
        if (!label_scores || !targets || !cfg || n == 0) fail(SGR_ERR_INVALID_ARGUMENT, "empty training set");
        const int L = (int)ctx->mk.n_labels;
        cudaStream_t s = ctx->stream;
        Mlp& m = ctx->mlp;
        m.init(L, cfg->hidden ? (int)cfg->hidden : 256, cfg->seed, s);
        ctx->mlp_scores.upload(label_scores, (size_t)n * L, s);
        ctx->mlp_x.ensure((size_t)n * L);
        ctx->mlp_bad.ensure(n);
        m.features(ctx->mlp_scores.p, (int)n, ctx->mlp_x.p, ctx->mlp_bad.p, s);
        std::vector<uint8_t> bad(n);
        SGR_CUDA(cudaMemcpyAsync(bad.data(), ctx->mlp_bad.p, n, cudaMemcpyDeviceToHost, s));
        SGR_CUDA(cudaStreamSynchronize(s));
        std::vector<int32_t> good;
        for (uint32_t i = 0; i < n; ++i) {
            if (targets[i] < 0 || targets[i] >= L) fail(SGR_ERR_INVALID_ARGUMENT, "target label out of range");
            if (!bad[i]) good.push_back((int32_t)i);
        }
        if (good.empty()) fail(SGR_ERR_INVALID_ARGUMENT, "no training row without NaN scores");
        ctx->mlp_y.upload(targets, n, s);
        const int B = (int)std::max<uint32_t>(1, std::min<uint32_t>(cfg->batch ? cfg->batch : 4096, (uint32_t)good.size()));
        ctx->mlp_xb.ensure((size_t)B * L);
        ctx->mlp_yb.ensure(B);
        ctx->mlp_idx.ensure(good.size());
        std::mt19937_64 rng(cfg->seed ^ 0x5DEECE66Dull);
        float last = 0.f;
        const int epochs = cfg->epochs ? (int)cfg->epochs : 20;
        for (int e = 0; e < epochs; ++e) {
            std::shuffle(good.begin(), good.end(), rng);
            ctx->mlp_idx.upload(good, s);
            for (size_t b0 = 0; b0 < good.size(); b0 += B) {
                const int nb = (int)std::min<size_t>(B, good.size() - b0);
                m.gather(ctx->mlp_x.p, ctx->mlp_y.p, ctx->mlp_idx.p + b0, nb, ctx->mlp_xb.p, ctx->mlp_yb.p, s);
                m.forward(ctx->mlp_xb.p, nb, s);
                m.backward(ctx->mlp_xb.p, ctx->mlp_yb.p, nb, s);
                m.adamw(cfg->lr, cfg->beta1, cfg->beta2, cfg->eps, cfg->weight_decay, s);
                if (e == epochs - 1 && b0 + B >= good.size()) {
                    std::vector<float> rl(nb);
                    SGR_CUDA(cudaMemcpyAsync(rl.data(), m.row_loss.p, nb * sizeof(float), cudaMemcpyDeviceToHost, s));
                    SGR_CUDA(cudaStreamSynchronize(s));
                    double t = 0;
                    for (float x : rl) t += x;
                    last = (float)(t / nb);
                }
            }
        }
        if (final_loss) *final_loss = last;
    });
}

sgr_status sgr_mlp_predict(sgr_ctx* ctx, const float* label_scores, uint32_t n, int32_t* labels, float* confidence) {
    return guarded(ctx, [&] {
        if (!ctx->mlp.ready) fail(SGR_ERR_STATE, "no trained proposal network");
        const int L = ctx->mlp.L;
        cudaStream_t s = ctx->stream;
        ctx->mlp_scores.upload(label_scores, (size_t)n * L, s);
        ctx->mlp_x.ensure((size_t)n * L);
        ctx->mlp_bad.ensure(n);
        ctx->prop.ensure(n);
        ctx->prop_conf.ensure(n);
        ctx->mlp.features(ctx->mlp_scores.p, (int)n, ctx->mlp_x.p, ctx->mlp_bad.p, s);
        ctx->mlp.predict(ctx->mlp_x.p, (int)n, ctx->prop.p, ctx->prop_conf.p, s);
        SGR_CUDA(cudaMemcpyAsync(labels, ctx->prop.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        SGR_CUDA(cudaMemcpyAsync(confidence, ctx->prop_conf.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    });
}

sgr_status sgr_mlp_params(sgr_ctx* ctx, float* out, uint64_t cap, uint32_t* n_labels, uint32_t* hidden,
                          uint64_t* n_params) {
    return guarded(ctx, [&] {
        if (!ctx->mlp.ready) fail(SGR_ERR_STATE, "no proposal network");
        if (n_labels) *n_labels = (uint32_t)ctx->mlp.L;
        if (hidden) *hidden = (uint32_t)ctx->mlp.H;
        if (n_params) *n_params = ctx->mlp.n_params;
        if (out) {
            if (cap < ctx->mlp.n_params) fail(SGR_ERR_INVALID_ARGUMENT, "parameter buffer too small");
            SGR_CUDA(cudaMemcpyAsync(out, ctx->mlp.w.p, ctx->mlp.n_params * sizeof(float), cudaMemcpyDeviceToHost,
                                     ctx->stream));
        }
    });
}

sgr_status sgr_mlp_load(sgr_ctx* ctx, const float* params, uint32_t n_labels, uint32_t hidden) {
    return guarded(ctx, [&] {
        if (ctx->device < 0) fail(SGR_ERR_STATE, "host-only context");
        if (!params || n_labels == 0 || hidden == 0) fail(SGR_ERR_INVALID_ARGUMENT, "bad parameters");
        ctx->mlp.init((int)n_labels, (int)hidden, 0, ctx->stream);
        ctx->mlp.set_params(params, ctx->stream);
    });
}

sgr_status sgr_mlp_debug_grads(sgr_ctx* ctx, const float* features, const int32_t* targets, uint32_t n, float* grads,
                               float* loss) {
    return guarded(ctx, [&] {
        if (!ctx->mlp.ready) fail(SGR_ERR_STATE, "no proposal network");
        Mlp& m = ctx->mlp;
        cudaStream_t s = ctx->stream;
        ctx->mlp_xb.upload(features, (size_t)n * m.L, s);
        ctx->mlp_yb.upload(targets, n, s);
        m.forward(ctx->mlp_xb.p, (int)n, s);
        m.backward(ctx->mlp_xb.p, ctx->mlp_yb.p, (int)n, s);
        std::vector<float> rl(n);
        SGR_CUDA(cudaMemcpyAsync(grads, m.g.p, m.n_params * sizeof(float), cudaMemcpyDeviceToHost, s));
        SGR_CUDA(cudaMemcpyAsync(rl.data(), m.row_loss.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
        SGR_CUDA(cudaStreamSynchronize(s));
        double t = 0;
        for (float x : rl) t += x;
        if (loss) *loss = (float)(t / n);
    });
}

sgr_status sgr_annotate_learned(sgr_ctx* ctx, const sgr_csr* qry, float quantile, float finetune_thre,
                                int32_t finetune_times, float min_confidence, float check_fraction,
                                int32_t* first_labels, int32_t* final_labels, sgr_learned_stats* stats) {
    return guarded(ctx, [&] {
        if (!ctx->trained) fail(SGR_ERR_STATE, "annotate before train");
        if (ctx->mode != SGR_MODE_EXACT) fail(SGR_ERR_STATE, "the learned form runs in exact mode");
        if (!ctx->mlp.ready || ctx->mlp.L != (int)ctx->mk.n_labels) fail(SGR_ERR_STATE, "no proposal network");
        if (!first_labels || !final_labels) fail(SGR_ERR_INVALID_ARGUMENT, "null output");
        reset_status(ctx);
        DevCsr q = query_on_device(ctx, qry, true);
        if (stats) *stats = sgr_learned_stats{};
        if (q.n_rows == 0) return;
        annotate_learned(ctx, q, qry->on_device ? nullptr : qry, quantile, finetune_thre, finetune_times,
                         min_confidence, check_fraction, first_labels, final_labels, stats);
    });
}

sgr_status sgr_annotate_stream(sgr_ctx* ctx, const sgr_csr* batches, uint32_t n_batches, float quantile,
                               float finetune_thre, int32_t finetune_times, int32_t learned, float min_confidence,
                               float check_fraction, int32_t* first_labels, int32_t* final_labels, float* batch_ms,
                               sgr_learned_stats* stats) {
    return guarded(ctx, [&] {
        if (!ctx->trained) fail(SGR_ERR_STATE, "annotate before train");
        if (n_batches && !batches) fail(SGR_ERR_INVALID_ARGUMENT, "null batch array");
        if (!first_labels || !final_labels) fail(SGR_ERR_INVALID_ARGUMENT, "null output");
        if (learned) {
            if (ctx->mode != SGR_MODE_EXACT) fail(SGR_ERR_STATE, "the learned form runs in exact mode");
            if (!ctx->mlp.ready || ctx->mlp.L != (int)ctx->mk.n_labels) fail(SGR_ERR_STATE, "no proposal network");
        }
        reset_status(ctx);
        annotate_stream(ctx, batches, n_batches, quantile, finetune_thre, finetune_times, learned != 0,
                        min_confidence, check_fraction, first_labels, final_labels, batch_ms, stats);
    });
}

void sgr_debug_stl_sort(float* v, int32_t n) {
    int oob = 0;
    stl::sort(v, n, &oob);
}

void sgr_debug_stl_minmax(const float* v, int32_t n, int32_t* mn, int32_t* mx) {
    int a = 0, b = 0;
    stl::minmax(v, n, &a, &b);
    *mn = a;
    *mx = b;
}

}  // extern "C"
