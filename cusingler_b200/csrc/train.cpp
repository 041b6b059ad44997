// Host marker training: the reference's DataParser stages that decide the gene sets
// (src/io.cpp:141-262, 306-349, 616-684, 714-757 of STOmics/cusingler), rewritten for speed but
// with the same results: medians come from the stored values plus a count of implicit zeros
// instead of a dense per-gene column, and label pairs are ranked in parallel.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>

#include "sgr_internal.h"

namespace sgr {

int marker_count(size_t n) { return (int)std::round(500 * std::pow(2 / 3.0, std::log2((double)n))); }

namespace {

template <class F>
void run_parallel(int cores, size_t n, F f) {
    int nt = (int)std::min<size_t>(std::max(cores, 1), n);
    if (nt <= 1) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&] {
            for (size_t i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto& t : th) t.join();
}

// Gene-name intersection (src/io.cpp:306-349).  Equal-size name sets keep the columns as they are;
// otherwise each side keeps its own columns whose name is shared, renumbered in its own order.
void intersect_genes(const HostCsr& ref, const char* const* ref_genes, const char* const* qry_genes,
                     uint32_t n_qry, Markers& m) {
    std::set<std::string> a, b;
    for (uint32_t i = 0; i < ref.n_cols; ++i) a.insert(ref_genes[i]);
    for (uint32_t i = 0; i < n_qry; ++i) b.insert(qry_genes[i]);
    std::set<std::string> both;
    std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::inserter(both, both.begin()));
    m.ref_colmap.assign(ref.n_cols, -1);
    m.qry_colmap.assign(n_qry, -1);
    if (a.size() == b.size() && a.size() == both.size()) {
        m.filter_genes = false;
        for (uint32_t i = 0; i < ref.n_cols; ++i) m.ref_colmap[i] = (int32_t)i;
        for (uint32_t i = 0; i < n_qry; ++i) m.qry_colmap[i] = i < ref.n_cols ? (int32_t)i : -1;
        return;
    }
    if (both.empty()) fail(SGR_ERR_NO_INTERSECTION, "no gene name is shared by reference and query");
    m.filter_genes = true;
    int32_t k = 0;
    for (uint32_t i = 0; i < ref.n_cols; ++i)
        if (both.count(ref_genes[i])) m.ref_colmap[i] = k++;
    k = 0;
    for (uint32_t i = 0; i < n_qry; ++i)
        if (both.count(qry_genes[i])) m.qry_colmap[i] = k++;
}

// Median of `len` values: the stored ones in `v` (modified: sorted) plus len - v.size() zeros,
// with the reference's even/odd rule (src/io.cpp:143-164).
float median_with_zeros(std::vector<float>& v, uint32_t len) {
    if (v.empty()) return 0.f;
    std::sort(v.begin(), v.end());
    const uint32_t nz = len - (uint32_t)v.size();
    const uint32_t p0 = (uint32_t)(std::lower_bound(v.begin(), v.end(), 0.f) - v.begin());
    auto at = [&](uint32_t t) -> float {
        if (t < p0) return v[t];
        if (t < p0 + nz) return 0.f;
        return v[t - nz];
    };
    if (len % 2 == 0) return (at(len / 2) + at(len / 2 - 1)) / 2;
    return at(len / 2);
}

struct PairLists {
    std::vector<uint32_t> positive;  // diff > 0, by (diff desc, gene asc)
    std::vector<uint32_t> top;       // first n_common of the full order
};

// One ordered label pair (src/io.cpp:228-257): rounded scaled median differences, ranked by
// difference descending with ties to the smaller gene.
void rank_pair(const std::vector<float>& m1, const std::vector<float>& m2, size_t n_common, PairLists& out) {
    const uint32_t W = (uint32_t)m1.size();
    std::vector<std::pair<int, uint32_t>> pos, neg;  // (-diff, gene) for an ascending sort
    std::vector<uint32_t> zero;
    for (uint32_t g = 0; g < W; ++g) {
        float df = m1[g] - m2[g];
        int d = int(std::round(df * 1e6));
        if (d > 0) pos.push_back({-d, g});
        else if (d == 0) zero.push_back(g);
        else neg.push_back({-d, g});
    }
    std::sort(pos.begin(), pos.end());
    out.positive.resize(pos.size());
    for (size_t i = 0; i < pos.size(); ++i) out.positive[i] = pos[i].second;
    out.top.clear();
    for (size_t i = 0; i < pos.size() && out.top.size() < n_common; ++i) out.top.push_back(pos[i].second);
    for (size_t i = 0; i < zero.size() && out.top.size() < n_common; ++i) out.top.push_back(zero[i]);
    if (out.top.size() < n_common) {
        size_t need = n_common - out.top.size();
        std::partial_sort(neg.begin(), neg.begin() + std::min(need, neg.size()), neg.end());
        for (size_t i = 0; i < need && i < neg.size(); ++i) out.top.push_back(neg[i].second);
    }
}

}  // namespace

void prepare_markers(const HostCsr& ref, const int32_t* celltypes, uint32_t n_labels,
                     const char* const* ref_genes, const char* const* qry_genes, uint32_t n_qry_genes, Markers& m) {
    m = Markers();
    m.n_labels = n_labels;
    m.W = ref.n_cols;
    if (n_labels == 0) fail(SGR_ERR_INVALID_ARGUMENT, "no label names");
    if (n_labels > 256) fail(SGR_ERR_UNSUPPORTED, "more than 256 labels (codes are 8-bit)");
    intersect_genes(ref, ref_genes, qry_genes, n_qry_genes, m);

    // Regroup reference rows by label, stable (src/io.cpp:616-684); codes narrowed to 8 bits.
    std::vector<std::vector<uint32_t>> by(n_labels);
    for (uint32_t i = 0; i < ref.n_rows; ++i) {
        uint32_t code = (uint8_t)celltypes[i];
        if (code >= n_labels)
            fail(SGR_ERR_INVALID_ARGUMENT, "reference cell " + std::to_string(i) + " has label code " +
                                               std::to_string(code) + " >= number of label names");
        by[code].push_back(i);
    }
    uint32_t start = 0;
    for (uint32_t l = 0; l < n_labels; ++l) {
        if (by[l].empty()) fail(SGR_ERR_EMPTY_LABEL, "label " + std::to_string(l) + " has no reference cell");
        m.ctidx.push_back(start);
        m.ctidx.push_back((uint32_t)by[l].size());
        start += (uint32_t)by[l].size();
        m.ref_order.insert(m.ref_order.end(), by[l].begin(), by[l].end());
    }
    if ((size_t)marker_count(n_labels) > m.W) fail(SGR_ERR_UNSUPPORTED, "more marker genes per label pair than genes");
}

void finish_markers(Markers& m, const uint8_t* in_common, const uint8_t* in_thre) {
    const uint32_t W = m.W, L = m.n_labels;
    m.common.clear();
    m.thre.clear();
    std::vector<int32_t> thre_id(W, -1);
    for (uint32_t g = 0; g < W; ++g) {
        if (in_common[g]) m.common.push_back(g);
        if (in_thre[g]) {
            thre_id[g] = (int32_t)m.thre.size();
            m.thre.push_back(g);
        }
    }
    // Pair lists restricted to the thre pool, in thre-compact ids (src/io.cpp:722-757).
    m.ft_genes.clear();
    m.ft_idx.clear();
    uint32_t fstart = 0;
    for (size_t p = 0; p < (size_t)L * L; ++p) {
        uint32_t pos = m.pair_idx[2 * p], len = m.pair_idx[2 * p + 1];
        if (pos == 0 && len == 0) {
            m.ft_idx.push_back(0);
            m.ft_idx.push_back(0);
            continue;
        }
        for (uint32_t j = pos; j < pos + len; ++j) {
            int32_t t = thre_id[m.pair_genes[j]];
            if (t >= 0) m.ft_genes.push_back((uint32_t)t);
        }
        m.ft_idx.push_back(fstart);
        m.ft_idx.push_back((uint32_t)m.ft_genes.size() - fstart);
        fstart = (uint32_t)m.ft_genes.size();
    }
}

void rank_markers_host(const HostCsr& ref, int cores, Markers& m) {
    const uint32_t n_labels = m.n_labels;
    std::vector<std::vector<uint32_t>> by(n_labels);
    for (uint32_t l = 0; l < n_labels; ++l)
        by[l].assign(m.ref_order.begin() + m.ctidx[2 * l], m.ref_order.begin() + m.ctidx[2 * l] + m.ctidx[2 * l + 1]);

    // Per-label medians over every gene id (implicit zeros included).
    const uint32_t W = m.W;
    std::vector<std::vector<float>> med(n_labels);
    run_parallel(cores, n_labels, [&](size_t l) {
        std::vector<uint32_t> cnt(W + 1, 0);
        for (uint32_t r : by[l])
            for (int32_t i = ref.indptr[r]; i < ref.indptr[r + 1]; ++i) {
                int32_t g = m.ref_colmap[ref.indices[i]];
                if (g >= 0) cnt[g + 1]++;
            }
        for (uint32_t g = 0; g < W; ++g) cnt[g + 1] += cnt[g];
        std::vector<float> vals(cnt[W]);
        std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
        for (uint32_t r : by[l])
            for (int32_t i = ref.indptr[r]; i < ref.indptr[r + 1]; ++i) {
                int32_t g = m.ref_colmap[ref.indices[i]];
                if (g >= 0) vals[fill[g]++] = ref.data[i];
            }
        med[l].assign(W, 0.f);
        std::vector<float> v;
        const uint32_t len = (uint32_t)by[l].size();
        for (uint32_t g = 0; g < W; ++g) {
            v.assign(vals.begin() + cnt[g], vals.begin() + cnt[g + 1]);
            med[l][g] = median_with_zeros(v, len);
        }
    });

    const size_t n_common = (size_t)marker_count(n_labels);
    const size_t n_thre = (size_t)marker_count(2);
    std::vector<PairLists> pl((size_t)n_labels * n_labels);
    run_parallel(cores, pl.size(), [&](size_t p) {
        size_t a = p / n_labels, b = p % n_labels;
        if (a != b) rank_pair(med[a], med[b], n_common, pl[p]);
    });
    std::vector<uint8_t> in_common(W, 0), in_thre(W, 0);
    uint32_t off = 0;
    m.pair_genes.clear();
    m.pair_idx.clear();
    for (size_t p = 0; p < pl.size(); ++p) {
        if (p / n_labels == p % n_labels) {
            m.pair_idx.push_back(0);
            m.pair_idx.push_back(0);
            continue;
        }
        const auto& pos = pl[p].positive;
        m.pair_genes.insert(m.pair_genes.end(), pos.begin(), pos.end());
        for (size_t i = 0; i < pos.size() && i < n_thre; ++i) in_thre[pos[i]] = 1;
        for (uint32_t g : pl[p].top) in_common[g] = 1;
        m.pair_idx.push_back(off);
        m.pair_idx.push_back((uint32_t)pos.size());
        off += (uint32_t)pos.size();
    }
    finish_markers(m, in_common.data(), in_thre.data());
}

void train_markers(const HostCsr& ref, const int32_t* celltypes, uint32_t n_labels,
                   const char* const* ref_genes, const char* const* qry_genes, uint32_t n_qry_genes,
                   int cores, Markers& m) {
    prepare_markers(ref, celltypes, n_labels, ref_genes, qry_genes, n_qry_genes, m);
    rank_markers_host(ref, cores, m);
}

}  // namespace sgr
