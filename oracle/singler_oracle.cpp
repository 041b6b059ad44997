// TEST INFRASTRUCTURE ONLY -- the oracle.
//
// A CPU restatement of the reference SingleR annotation path of STOmics/cusingler, used by tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.  The product
// (cusingler_b200/) never links, loads or calls this file.
//
// Every function below cites the reference file:line whose behaviour it restates.  Where the
// reference has undefined behaviour (an empty label, label codes >= the number of label names,
// more common genes than genes), this oracle returns an error instead; the product does the same.
//
// Two arithmetic modes for the correlation:
//   mode 0 "fp32ref": the reference's own FP32 operation order.  Score step: one sequential fused
//          multiply-add chain over genes per (query, ref) pair (src/cusingler.cu:918-945, nvcc
//          contracts `s += x*y` into an fma).  Fine-tune: 128 contiguous gene chunks, each an fma
//          chain, then a stride-doubling pairwise tree (src/cusingler.cu:803-856).
//   mode 1 "exact": numerator sum(d_q * d_r) in int64 over doubled centred ranks
//          d = 2*rank - (G+1), squared norms n = sum(d*d) in int64, and
//          score = float((double(N) * (1/sqrt(double(n_q)))) * (1/sqrt(double(n_r)))).
//
// Parity pins: the host stages (gene sets, codes, pair lists, percentile) are checked against the
// reference's own io.cpp / percentile() compiled from its sources (oracle/ref_harness.cpp); the
// fp32ref scores and labels against the reference module run on a B200 (tests/golden/).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <numeric>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

struct CsrF {
    std::vector<float> data;
    std::vector<int> indices;
    std::vector<int> indptr;
};

struct CsrCode {  // marker-filtered CSR with per-row value codes (InputData, src/types.h:21-42)
    std::vector<uint16_t> data;
    std::vector<int> indices;
    std::vector<int> indptr;
};

struct Ctx {
    int cores = 1;
    std::string err;

    uint32_t ref_h = 0, ref_w = 0, qry_h = 0, qry_w = 0;
    CsrF ref, qry;
    std::vector<std::string> label_names;
    std::vector<uint8_t> codes;  // per ref cell, narrowed to 8 bits (src/io.cpp:813, src/io.h:73)
    std::vector<std::string> ref_genes, qry_genes;

    bool filter_genes = false;
    std::map<uint32_t, uint32_t> ref_gene_index, qry_gene_index;

    std::vector<uint32_t> ctidx;  // (start, len) per label in the regrouped reference
    std::vector<uint32_t> ctids;  // original row id per regrouped row
    std::vector<uint32_t> order;  // kept copy of ctids for tests

    std::vector<uint32_t> train_idxs, train_values;
    std::set<uint32_t> common, thre;

    CsrCode ref_s, qry_s;  // score step, columns = common genes
    uint32_t G = 0;
    std::vector<uint32_t> ft_ctdiff, ft_ctdidx;
    CsrCode ref_f, qry_f;  // fine-tune, columns = thre genes
    uint32_t Wt = 0;

    std::vector<float> label_scores;  // Q x L
    std::vector<float> flags;         // Q x L (the reference's float `labels`, src/types.h:34)
    std::vector<int> first;
    // Decision margins per query cell (for near-tie checks of arithmetic-order label flips): the
    // smallest distance, over every keep / drop / argmax comparison the cell's labels went
    // through, between a score and the value it was compared with.  margin_first covers the score
    // step, margin_final the score step and every fine-tune round.
    std::vector<float> margin_first, margin_final;
    bool trained = false, scored = false;
};

template <class F>
void parallel_for(int cores, size_t n, F f) {
    if (cores <= 1 || n < 2) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    int nt = std::min<size_t>(cores, n);
    std::vector<std::thread> th;
    std::atomic<size_t> next{0};
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&]() {
            for (;;) {
                size_t i = next.fetch_add(1);
                if (i >= n) break;
                f(i);
            }
        });
    for (auto& t : th) t.join();
}

// src/io.cpp:306-349 (findIntersectionGenes).  Gene-name sets are compared by size only, so an
// equal-size intersection keeps the column order as given.
bool find_intersection(Ctx& c) {
    std::set<std::string> a(c.ref_genes.begin(), c.ref_genes.end());
    std::set<std::string> b(c.qry_genes.begin(), c.qry_genes.end());
    std::set<std::string> both;
    std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::inserter(both, both.begin()));
    if (a.size() == b.size() && a.size() == both.size()) {
        c.filter_genes = false;
        return true;
    }
    if (both.empty()) {
        c.err = "no intersection genes between reference and query";
        return false;
    }
    c.filter_genes = true;
    uint32_t k = 0;
    for (uint32_t i = 0; i < c.ref_genes.size(); ++i)
        if (both.count(c.ref_genes[i])) c.ref_gene_index[i] = k++;
    k = 0;
    for (uint32_t i = 0; i < c.qry_genes.size(); ++i)
        if (both.count(c.qry_genes[i])) c.qry_gene_index[i] = k++;
    return true;
}

// src/io.cpp:616-636 (groupbyCelltypes): label-major, stable in original row order.
bool group_by_label(Ctx& c) {
    size_t L = c.label_names.size();
    std::vector<std::vector<uint32_t>> by(L);
    for (size_t i = 0; i < c.codes.size(); ++i) {
        if (c.codes[i] >= L) {
            c.err = "reference label code out of range of the label names";
            return false;
        }
        by[c.codes[i]].push_back(i);
    }
    uint32_t start = 0;
    for (auto& v : by) {
        if (v.empty()) {
            c.err = "a label has no reference cells";
            return false;
        }
        c.ctidx.push_back(start);
        c.ctidx.push_back(v.size());
        start += v.size();
        c.ctids.insert(c.ctids.end(), v.begin(), v.end());
    }
    return true;
}

// src/io.cpp:657-684 (resort).
void resort(Ctx& c) {
    CsrF out;
    out.indptr.push_back(0);
    for (uint32_t j = 0; j < c.ctids.size(); ++j) {
        uint32_t row = c.ctids[j];
        int a = c.ref.indptr[row], b = c.ref.indptr[row + 1];
        out.indptr.push_back(out.indptr.back() + b - a);
        out.indices.insert(out.indices.end(), c.ref.indices.begin() + a, c.ref.indices.begin() + b);
        out.data.insert(out.data.end(), c.ref.data.begin() + a, c.ref.data.begin() + b);
    }
    c.ref = std::move(out);
    c.order = c.ctids;
    c.ctids.clear();
}

// src/io.cpp:687-711 (removeCols).
void remove_cols(CsrF& m, const std::map<uint32_t, uint32_t>& cols) {
    CsrF out;
    out.indptr.push_back(0);
    for (size_t j = 0; j + 1 < m.indptr.size(); ++j) {
        for (int i = m.indptr[j]; i < m.indptr[j + 1]; ++i) {
            auto it = cols.find(m.indices[i]);
            if (it == cols.end()) continue;
            out.indices.push_back(it->second);
            out.data.push_back(m.data[i]);
        }
        out.indptr.push_back(out.data.size());
    }
    m = std::move(out);
}

// src/io.cpp:141-262 (trainData).
bool train_markers(Ctx& c) {
    const uint32_t W = c.ref_w;  // not reduced by removeCols (src/io.cpp:362-367)
    const size_t L = c.ctidx.size() / 2;
    std::vector<std::vector<float>> med(L, std::vector<float>(W, 0.f));
    for (size_t ct = 0; ct < L; ++ct) {
        uint32_t pos = c.ctidx[2 * ct], len = c.ctidx[2 * ct + 1];
        std::vector<std::vector<float>> cols(W);
        for (uint32_t r = pos; r < pos + len; ++r)
            for (int i = c.ref.indptr[r]; i < c.ref.indptr[r + 1]; ++i)
                cols[c.ref.indices[i]].push_back(c.ref.data[i]);
        parallel_for(c.cores, W, [&](size_t g) {
            auto& v = cols[g];
            v.resize(len, 0.f);
            float m;
            if (v.size() % 2 == 0) {
                std::sort(v.begin(), v.end());
                m = (v[v.size() / 2] + v[v.size() / 2 - 1]) / 2;
            } else {
                std::nth_element(v.begin(), v.begin() + v.size() / 2, v.end());
                m = v[v.size() / 2];
            }
            med[ct][g] = m;
        });
    }
    size_t n_common = (size_t)std::round(500 * std::pow(2 / 3.0, std::log2((double)c.label_names.size())));
    size_t n_thre = (size_t)std::round(500 * std::pow(2 / 3.0, std::log2(2.0)));
    if (n_common > W) {
        // the reference reads past the end of its diff list here (src/io.cpp:254-256)
        c.err = "more common genes per label pair than genes";
        return false;
    }
    // Ordered label pairs in ascending (k1, k2), diagonal padded with (0, 0).
    std::vector<std::vector<uint32_t>> pair_pos(L * L);
    std::vector<std::vector<uint32_t>> pair_common(L * L);
    parallel_for(c.cores, L * L, [&](size_t p) {
        size_t k1 = p / L, k2 = p % L;
        if (k1 == k2) return;
        std::vector<std::pair<int, uint32_t>> diff(W);
        for (uint32_t i = 0; i < W; ++i)
            diff[i] = {int(std::round((med[k1][i] - med[k2][i]) * 1e6)), W - i - 1};
        std::sort(diff.begin(), diff.end(), std::greater<std::pair<int, uint32_t>>());
        auto& pos = pair_pos[p];
        for (uint32_t i = 0; i < diff.size() && diff[i].first > 0; ++i) pos.push_back(W - diff[i].second - 1);
        auto& com = pair_common[p];
        for (size_t i = 0; i < n_common; ++i) com.push_back(W - diff[i].second - 1);
    });
    uint32_t start = 0;
    for (size_t p = 0; p < L * L; ++p) {
        if (p / L == p % L) {
            c.train_idxs.push_back(0);
            c.train_idxs.push_back(0);
            continue;
        }
        auto& pos = pair_pos[p];
        for (size_t i = 0; i < pos.size(); ++i) {
            c.train_values.push_back(pos[i]);
            if (i < n_thre) c.thre.insert(pos[i]);
        }
        c.train_idxs.push_back(start);
        c.train_idxs.push_back(pos.size());
        start += pos.size();
        for (auto g : pair_common[p]) c.common.insert(g);
    }
    return true;
}

// src/io.cpp:470-523 (csrFilter): keep the columns in `cols` (remapped to their rank in the set)
// and replace each stored value by its 1-based rank among the row's distinct kept values.
void csr_filter(const CsrF& m, const std::set<uint32_t>& cols, CsrCode& out) {
    std::unordered_map<uint32_t, uint32_t> idx;
    uint32_t k = 0;
    for (auto g : cols) idx[g] = k++;
    out.data.clear();
    out.indices.clear();
    out.indptr.assign(1, 0);
    for (size_t j = 0; j + 1 < m.indptr.size(); ++j) {
        std::set<float> uniq;
        for (int i = m.indptr[j]; i < m.indptr[j + 1]; ++i)
            if (idx.count(m.indices[i])) uniq.insert(m.data[i]);
        std::unordered_map<float, uint16_t> code;
        uint16_t n = 0;
        for (float v : uniq) code[v] = ++n;
        for (int i = m.indptr[j]; i < m.indptr[j + 1]; ++i) {
            auto it = idx.find(m.indices[i]);
            if (it == idx.end()) continue;
            out.indices.push_back(it->second);
            out.data.push_back(code[m.data[i]]);
        }
        out.indptr.push_back(out.data.size());
    }
}

// Tie-averaged rank of each entry of a dense code row: 1 + #less + (#equal - 1) / 2, computed by a
// code histogram and a running start as src/cusingler.cu:745-801 (rankdata_bin3) does; every rank
// kernel of the reference (rankdata, rankdata_batch, src/cusingler.cu:158-179, 601-625) yields the
// same half-integers.
void rank_codes(const uint16_t* codes, uint32_t n, float* out) {
    uint16_t mx = 0;
    for (uint32_t i = 0; i < n; ++i) mx = std::max(mx, codes[i]);
    std::vector<int> bins(mx + 1, 0);
    for (uint32_t i = 0; i < n; ++i) bins[codes[i]]++;
    std::vector<float> rk(mx + 1);
    int start = 0;
    for (int i = 0; i <= mx; ++i) {
        rk[i] = start + (bins[i] + 1) * 0.5;
        start += bins[i];
    }
    for (uint32_t i = 0; i < n; ++i) out[i] = rk[codes[i]];
}

void dense_codes(const CsrCode& m, uint32_t row, uint32_t width, uint16_t* out) {
    std::fill(out, out + width, 0);
    for (int i = m.indptr[row]; i < m.indptr[row + 1]; ++i) out[m.indices[i]] = m.data[i];
}

// src/cusingler.cu:947-978 (percentile): sort a copy, float index grid i*step with
// step = 1/(len-1), lower_bound, linear interpolation in float.
float percentile(std::vector<float> arr, int len, float p) {
    if (len <= 1) return arr.front();
    std::sort(arr.begin(), arr.begin() + len);
    std::vector<float> index;
    float step = 1.0 / (len - 1);
    for (int i = 0; i < len; ++i) index.push_back(i * step);
    if (p <= index.front()) return arr[0];
    if (index.back() <= p) return arr[len - 1];
    auto it = std::lower_bound(index.begin(), index.end(), p);
    float prev_i = *(it - 1);
    float prev_v = arr.at(it - index.begin() - 1);
    float next_v = arr.at(it - index.begin());
    return (p - prev_i) * (next_v - prev_v) / step + prev_v;
}

// Centred ranks x = rank - (G+1)/2 of one dense code row (exact half-integers in float) and the
// doubled integer form d = 2x.
struct RankRow {
    std::vector<float> x;
    std::vector<int32_t> d;
};

void make_rank_row(const uint16_t* codes, uint32_t G, RankRow& rr) {
    rr.x.resize(G);
    rr.d.resize(G);
    rank_codes(codes, G, rr.x.data());
    float mean = (G + 1) / 2.0;
    for (uint32_t i = 0; i < G; ++i) {
        float x = rr.x[i] - mean;
        rr.x[i] = x;
        rr.d[i] = (int32_t)(2 * x);
    }
}

// src/cusingler.cu:918-945 (spearman, score step): fma chain over genes in order.
float spearman_seq(const float* x, const float* y, uint32_t G) {
    float sxy = 0, sxx = 0, syy = 0;
    for (uint32_t i = 0; i < G; ++i) {
        sxy = std::fmaf(x[i], y[i], sxy);
        sxx = std::fmaf(x[i], x[i], sxx);
        syy = std::fmaf(y[i], y[i], syy);
    }
    float div = std::sqrt(sxx * syy);
    return div != 0 ? sxy / div : NAN;
}

// src/cusingler.cu:803-856 (spearman_reduce, fine-tune): 128 contiguous chunks of ceil(G/128)
// genes, fma chain per chunk, then pairwise tree with stride 1, 2, ..., 64.
float spearman_tree(const float* x, const float* y, uint32_t G) {
    float pxy[128], pxx[128], pyy[128];
    uint32_t step = (G + 127) / 128;
    for (int t = 0; t < 128; ++t) {
        float a = 0, b = 0, c = 0;
        for (uint32_t i = t * step; i < (t + 1) * step; ++i) {
            if (i < G) {
                a = std::fmaf(x[i], y[i], a);
                b = std::fmaf(x[i], x[i], b);
                c = std::fmaf(y[i], y[i], c);
            }
        }
        pxy[t] = a;
        pxx[t] = b;
        pyy[t] = c;
    }
    for (int s = 1; s < 128; s *= 2)
        for (int t = 0; t < 128; t += 2 * s) {
            pxy[t] += pxy[t + s];
            pxx[t] += pxx[t + s];
            pyy[t] += pyy[t + s];
        }
    float div = std::sqrt(pxx[0] * pyy[0]);
    return div != 0 ? pxy[0] / div : NAN;
}

int64_t sumsq(const int32_t* d, uint32_t G) {
    int64_t s = 0;
    for (uint32_t i = 0; i < G; ++i) s += (int64_t)d[i] * d[i];
    return s;
}

float exact_score(const int32_t* a, const int32_t* b, uint32_t G, int64_t na, int64_t nb) {
    if (na == 0 || nb == 0) return NAN;
    int64_t n = 0;
    for (uint32_t i = 0; i < G; ++i) n += (int64_t)a[i] * b[i];
    double ra = 1.0 / std::sqrt((double)na), rb = 1.0 / std::sqrt((double)nb);
    return (float)(((double)n * ra) * rb);
}

bool train(Ctx& c) {
    if (!find_intersection(c)) return false;
    // loadRefData (src/io.cpp:351-370)
    if (!group_by_label(c)) return false;
    resort(c);
    if (c.filter_genes) remove_cols(c.ref, c.ref_gene_index);
    if (!train_markers(c)) return false;
    // loadQryData (src/io.cpp:525-538)
    if (c.filter_genes) remove_cols(c.qry, c.qry_gene_index);
    // generateDenseMatrix(0) (src/io.cpp:714-784): common genes for the score step
    csr_filter(c.ref, c.common, c.ref_s);
    csr_filter(c.qry, c.common, c.qry_s);
    c.G = c.common.size();
    // generateDenseMatrix(1): thre genes, pair lists remapped to compact thre indices
    std::map<uint32_t, uint32_t> tmap;
    uint32_t k = 0;
    for (auto g : c.thre) tmap[g] = k++;
    size_t start = 0;
    for (size_t i = 0; i < c.train_idxs.size(); i += 2) {
        uint32_t pos = c.train_idxs[i], len = c.train_idxs[i + 1];
        if (pos == 0 && len == 0) {
            c.ft_ctdidx.push_back(0);
            c.ft_ctdidx.push_back(0);
            continue;
        }
        for (uint32_t j = pos; j < pos + len; ++j) {
            auto it = tmap.find(c.train_values[j]);
            if (it == tmap.end()) continue;
            c.ft_ctdiff.push_back(it->second);
        }
        c.ft_ctdidx.push_back(start);
        c.ft_ctdidx.push_back(c.ft_ctdiff.size() - start);
        start = c.ft_ctdiff.size();
    }
    csr_filter(c.ref, c.thre, c.ref_f);
    csr_filter(c.qry, c.thre, c.qry_f);
    c.Wt = c.thre.size();
    c.trained = true;
    return true;
}

// libstdc++'s std::minmax_element as the reference calls it (src/cusingler.cu:1123, 1270):
// first minimum, last maximum, with its pairwise comparison order (matters for NaN).
std::pair<int, int> minmax_idx(const float* v, int n) {
    auto e = std::minmax_element(v, v + n);
    return {int(e.first - v), int(e.second - v)};
}

// Smallest distance between a score of `v` and the thresholds it is compared with: the maximum
// (argmax), the minimum (the fine-tune's `<= min` drop, when `with_min`) and `t` (the keep bound);
// NaN scores are skipped.  A label decision can only change under score perturbations of at least
// half this margin.
float decision_margin(const float* v, int n, int mn, int mx, float t, bool with_min) {
    float m = std::numeric_limits<float>::infinity();
    for (int i = 0; i < n; ++i) {
        if (std::isnan(v[i])) continue;
        m = std::min(m, std::fabs(v[i] - t));
        if (i != mx && !std::isnan(v[mx])) m = std::min(m, v[mx] - v[i]);
        if (with_min && i != mn && !std::isnan(v[mn])) m = std::min(m, v[i] - v[mn]);
    }
    return m;
}

// src/cusingler.cu:986-1136 (get_label) without slicing: every ref row in one pass.
bool score(Ctx& c, float q, float thre, int mode, int* first_out, float* scores_out, float* flags_out,
           float* raw_out) {
    const uint32_t G = c.G, R = c.ref_h, Q = c.qry_h, L = c.label_names.size();
    std::vector<RankRow> ref_rank(R);
    std::vector<int64_t> ref_n(R);
    parallel_for(c.cores, R, [&](size_t r) {
        std::vector<uint16_t> codes(G);
        dense_codes(c.ref_s, r, G, codes.data());
        make_rank_row(codes.data(), G, ref_rank[r]);
        ref_n[r] = sumsq(ref_rank[r].d.data(), G);
    });
    c.label_scores.assign((size_t)Q * L, 0.f);
    c.flags.assign((size_t)Q * L, 0.f);
    c.first.assign(Q, 0);
    c.margin_first.assign(Q, std::numeric_limits<float>::infinity());
    parallel_for(c.cores, Q, [&](size_t qi) {
        std::vector<uint16_t> codes(G);
        dense_codes(c.qry_s, qi, G, codes.data());
        RankRow qr;
        make_rank_row(codes.data(), G, qr);
        int64_t qn = sumsq(qr.d.data(), G);
        std::vector<float> s(R);
        for (uint32_t r = 0; r < R; ++r)
            s[r] = mode == 0 ? spearman_seq(qr.x.data(), ref_rank[r].x.data(), G)
                             : exact_score(qr.d.data(), ref_rank[r].d.data(), G, qn, ref_n[r]);
        if (raw_out) std::copy(s.begin(), s.end(), raw_out + qi * (size_t)R);
        float* ls = &c.label_scores[qi * L];
        for (uint32_t l = 0; l < L; ++l) {
            uint32_t st = c.ctidx[2 * l], len = c.ctidx[2 * l + 1];
            std::vector<float> tmp(s.begin() + st, s.begin() + st + len);
            ls[l] = percentile(tmp, len, q);
        }
        auto mm = minmax_idx(ls, L);
        c.first[qi] = mm.second;
        float t = ls[mm.second] - thre;
        for (uint32_t l = 0; l < L; ++l)
            if (ls[l] >= t) c.flags[qi * L + l] = 1;
        c.margin_first[qi] = decision_margin(ls, (int)L, mm.first, mm.second, t, false);
    });
    if (first_out) std::copy(c.first.begin(), c.first.end(), first_out);
    if (scores_out) std::copy(c.label_scores.begin(), c.label_scores.end(), scores_out);
    if (flags_out) std::copy(c.flags.begin(), c.flags.end(), flags_out);
    c.scored = true;
    return true;
}

// src/cusingler.cu:1138-1296 (finetune_round).
std::vector<uint32_t> finetune_round(const Ctx& c, uint32_t cell, const std::vector<uint32_t>& top, float q,
                                     float thre, int mode, float* margin) {
    const uint32_t L = c.label_names.size();
    std::set<uint32_t> uniq;
    int gene_thre = std::round(500 * std::pow(2 / 3.0, std::log2((double)top.size())));
    for (auto i : top)
        for (auto j : top) {
            if (i == j) continue;
            int pos = c.ft_ctdidx[(i * L + j) * 2];
            int len = c.ft_ctdidx[(i * L + j) * 2 + 1];
            if (len > gene_thre) len = gene_thre;
            uniq.insert(c.ft_ctdiff.begin() + pos, c.ft_ctdiff.begin() + pos + len);
        }
    if (uniq.size() < 20) return {top.front()};
    std::vector<uint32_t> genes(uniq.begin(), uniq.end());
    const uint32_t G = genes.size();
    std::vector<uint16_t> full(c.Wt), sub(G);
    dense_codes(c.qry_f, cell, c.Wt, full.data());
    for (uint32_t i = 0; i < G; ++i) sub[i] = full[genes[i]];
    RankRow qr;
    make_rank_row(sub.data(), G, qr);
    int64_t qn = sumsq(qr.d.data(), G);
    std::vector<float> scores;
    RankRow rr;
    for (auto lab : top) {
        uint32_t st = c.ctidx[2 * lab], len = c.ctidx[2 * lab + 1];
        std::vector<float> tmp(len);
        for (uint32_t r = st; r < st + len; ++r) {
            dense_codes(c.ref_f, r, c.Wt, full.data());
            for (uint32_t i = 0; i < G; ++i) sub[i] = full[genes[i]];
            make_rank_row(sub.data(), G, rr);
            tmp[r - st] = mode == 0 ? spearman_tree(qr.x.data(), rr.x.data(), G)
                                    : exact_score(qr.d.data(), rr.d.data(), G, qn, sumsq(rr.d.data(), G));
        }
        scores.push_back(percentile(tmp, len, q));
    }
    auto mm = minmax_idx(scores.data(), scores.size());
    float mn = scores[mm.first], mx = scores[mm.second];
    float t = mx - thre;
    if (std::isnan(mx)) return {top.front()};
    *margin = std::min(*margin, decision_margin(scores.data(), (int)scores.size(), mm.first, mm.second, t, true));
    std::vector<uint32_t> res;
    for (uint32_t i = 0; i < scores.size(); ++i) {
        if (scores[i] <= mn || scores[i] < t) continue;
        if (scores[i] == mx)
            res.insert(res.begin(), top[i]);
        else
            res.push_back(top[i]);
    }
    if (res.empty()) res.push_back(top.front());
    return res;
}

// src/cusingler.cu:1297-1333 (cufinetune).
bool finetune(Ctx& c, float q, float thre, int times, int mode, int* final_out, int* rounds_out) {
    const uint32_t L = c.label_names.size();
    c.margin_final.assign(c.qry_h, std::numeric_limits<float>::infinity());
    parallel_for(c.cores, c.qry_h, [&](size_t i) {
        std::vector<uint32_t> top;
        for (uint32_t l = 0; l < L; ++l)
            if (c.flags.at(i * L + l) != 0) top.push_back(l);
        int t = 0, rounds = 0;
        float margin = i < c.margin_first.size() ? c.margin_first[i] : std::numeric_limits<float>::infinity();
        while (top.size() > 1 && (times == 0 || t++ < times)) {
            top = finetune_round(c, i, top, q, thre, mode, &margin);
            rounds++;
        }
        c.margin_final[i] = margin;
        final_out[i] = top.empty() ? 0 : (int)top.front();
        if (rounds_out) rounds_out[i] = rounds;
    });
    return true;
}

}  // namespace

extern "C" {

void* or_create(int cores) {
    auto* c = new Ctx();
    c->cores = cores < 1 ? 1 : cores;
    return c;
}

void or_destroy(void* h) { delete static_cast<Ctx*>(h); }

const char* or_error(void* h) { return static_cast<Ctx*>(h)->err.c_str(); }

// src/io.cpp:792-821 (PyDataParser::prepareData).
int or_load(void* h, uint32_t ref_h, uint32_t ref_w, const float* rd, const int* ri, const int* rp, uint32_t qry_h,
            uint32_t qry_w, const float* qd, const int* qi, const int* qp, const char** label_names,
            uint32_t n_labels, const int* celltypes, const char** ref_genes, const char** qry_genes) {
    Ctx& c = *static_cast<Ctx*>(h);
    c.ref_h = ref_h;
    c.ref_w = ref_w;
    c.qry_h = qry_h;
    c.qry_w = qry_w;
    c.ref.indptr.assign(rp, rp + ref_h + 1);
    c.ref.data.assign(rd, rd + rp[ref_h]);
    c.ref.indices.assign(ri, ri + rp[ref_h]);
    c.qry.indptr.assign(qp, qp + qry_h + 1);
    c.qry.data.assign(qd, qd + qp[qry_h]);
    c.qry.indices.assign(qi, qi + qp[qry_h]);
    for (uint32_t i = 0; i < n_labels; ++i) c.label_names.emplace_back(label_names[i]);
    c.codes.resize(ref_h);
    for (uint32_t i = 0; i < ref_h; ++i) c.codes[i] = (uint8_t)celltypes[i];
    for (uint32_t i = 0; i < ref_w; ++i) c.ref_genes.emplace_back(ref_genes[i]);
    for (uint32_t i = 0; i < qry_w; ++i) c.qry_genes.emplace_back(qry_genes[i]);
    return 0;
}

int or_train(void* h) { return train(*static_cast<Ctx*>(h)) ? 0 : 1; }

uint32_t or_count(void* h, int what) {
    Ctx& c = *static_cast<Ctx*>(h);
    switch (what) {
        case 0: return c.common.size();
        case 1: return c.thre.size();
        case 2: return c.train_values.size();
        case 3: return c.ft_ctdiff.size();
        case 4: return c.filter_genes ? 1 : 0;
        case 5: return c.qry_s.data.size();
        case 6: return c.ref_s.data.size();
    }
    return 0;
}

// what: 0 common genes, 1 thre genes, 2 train values (pair lists), 3 train idxs, 4 fine-tune
// ctdiff, 5 fine-tune ctdidx, 6 ctidx, 7 regrouped-row order
void or_get_u32(void* h, int what, uint32_t* out) {
    Ctx& c = *static_cast<Ctx*>(h);
    switch (what) {
        case 0: std::copy(c.common.begin(), c.common.end(), out); break;
        case 1: std::copy(c.thre.begin(), c.thre.end(), out); break;
        case 2: std::copy(c.train_values.begin(), c.train_values.end(), out); break;
        case 3: std::copy(c.train_idxs.begin(), c.train_idxs.end(), out); break;
        case 4: std::copy(c.ft_ctdiff.begin(), c.ft_ctdiff.end(), out); break;
        case 5: std::copy(c.ft_ctdidx.begin(), c.ft_ctdidx.end(), out); break;
        case 6: std::copy(c.ctidx.begin(), c.ctidx.end(), out); break;
        case 7: std::copy(c.order.begin(), c.order.end(), out); break;
    }
}

// Score-step ranks of one row as doubled centred integers d = 2*rank - (G+1).
// which: 0 ref (regrouped order), 1 query.
void or_rank_row(void* h, int which, uint32_t row, int32_t* out) {
    Ctx& c = *static_cast<Ctx*>(h);
    std::vector<uint16_t> codes(c.G);
    dense_codes(which == 0 ? c.ref_s : c.qry_s, row, c.G, codes.data());
    RankRow rr;
    make_rank_row(codes.data(), c.G, rr);
    std::copy(rr.d.begin(), rr.d.end(), out);
}

// Score-step codes in CSR form (for bit-exact checks of the gather).
void or_codes(void* h, int which, uint16_t* data, int* indices, int* indptr) {
    Ctx& c = *static_cast<Ctx*>(h);
    const CsrCode& m = which == 0 ? c.ref_s : c.qry_s;
    std::copy(m.data.begin(), m.data.end(), data);
    std::copy(m.indices.begin(), m.indices.end(), indices);
    std::copy(m.indptr.begin(), m.indptr.end(), indptr);
}

int or_score(void* h, float quantile, float thre, int mode, int* first, float* label_scores, float* flags,
             float* raw) {
    Ctx& c = *static_cast<Ctx*>(h);
    if (!c.trained) return 1;
    return score(c, quantile, thre, mode, first, label_scores, flags, raw) ? 0 : 1;
}

int or_finetune(void* h, float quantile, float thre, int times, int mode, int* final_labels, int* rounds) {
    Ctx& c = *static_cast<Ctx*>(h);
    if (!c.scored) return 1;
    return finetune(c, quantile, thre, times, mode, final_labels, rounds) ? 0 : 1;
}

// Decision margins of the last score (which 0) or fine-tune (which 1) call, one per query cell.
void or_margins(void* h, int which, float* out) {
    Ctx& c = *static_cast<Ctx*>(h);
    const std::vector<float>& m = which == 0 ? c.margin_first : c.margin_final;
    std::copy(m.begin(), m.end(), out);
}

// Overrides the first-round flags (Q x L) so that fine-tune can be checked on its own.
void or_set_flags(void* h, const float* flags) {
    Ctx& c = *static_cast<Ctx*>(h);
    c.flags.assign(flags, flags + (size_t)c.qry_h * c.label_names.size());
    c.scored = true;
}

float or_percentile(const float* arr, int len, float p) {
    std::vector<float> v(arr, arr + len);
    return percentile(v, len, p);
}

void or_minmax(const float* v, int n, int* mn, int* mx) {
    auto r = minmax_idx(v, n);
    *mn = r.first;
    *mx = r.second;
}

void or_sort(float* v, int n) { std::sort(v, v + n); }

}  // extern "C"
