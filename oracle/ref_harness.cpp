// TEST INFRASTRUCTURE ONLY.
//
// Links the reference's own host code (src/io.cpp and the host function percentile() of
// src/cusingler.cu, compiled from the reference sources by oracle/Makefile into oracle/_ref/) and
// exposes its host stages through a C ABI, so that the oracle's restatement can be checked
// against the reference itself on the CPU: gene intersection, label regrouping, marker training
// (src/io.cpp:141-262), the marker-column CSR filter with per-row value codes (src/io.cpp:470-523)
// and the percentile (src/cusingler.cu:947-978).  No CUDA call is made.

#include <map>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>
#include <mutex>
#include <thread>

#define private public
#include "io.h"
#undef private

float percentile(std::vector<float> arr, int len, float p);  // src/cusingler.cu:947

namespace {
struct Harness {
    PyDataParser* dp = nullptr;
    std::vector<uint32_t> common, thre, train_idxs, train_values, ctidx;
    std::vector<uint16_t> s_ref_data, s_qry_data;
    std::vector<int> s_ref_indices, s_ref_indptr, s_qry_indices, s_qry_indptr;
    std::vector<uint32_t> ft_ctdiff, ft_ctdidx;
    std::vector<uint16_t> f_ref_data, f_qry_data;
    std::vector<int> f_ref_indices, f_ref_indptr, f_qry_indices, f_qry_indptr;
    uint64_t max_uniq_s = 0, max_uniq_f = 0;
};
}  // namespace

extern "C" {

void* ref_create(int cores) {
    auto* h = new Harness();
    h->dp = new PyDataParser(cores);
    return h;
}

void ref_destroy(void* p) {
    auto* h = static_cast<Harness*>(p);
    delete h->dp;
    delete h;
}

// Runs prepareData .. preprocess, then generateDenseMatrix(0) and (1), keeping their outputs.
// The caller must make sure the gene sets intersect (the reference calls exit() otherwise).
int ref_run(void* p, uint32_t ref_h, uint32_t ref_w, const float* rd, const int* ri, const int* rp, uint32_t qry_h,
            uint32_t qry_w, const float* qd, const int* qi, const int* qp, const char** label_names,
            uint32_t n_labels, const int* celltypes, const char** ref_genes, const char** qry_genes) {
    auto* h = static_cast<Harness*>(p);
    std::vector<float> ref_data(rd, rd + rp[ref_h]), qry_data(qd, qd + qp[qry_h]);
    std::vector<int> ref_indices(ri, ri + rp[ref_h]), ref_indptr(rp, rp + ref_h + 1);
    std::vector<int> qry_indices(qi, qi + qp[qry_h]), qry_indptr(qp, qp + qry_h + 1);
    std::vector<std::string> codes, cellnames, rg, qg;
    for (uint32_t i = 0; i < n_labels; ++i) codes.emplace_back(label_names[i]);
    std::vector<int> ct(celltypes, celltypes + ref_h);
    for (uint32_t i = 0; i < qry_h; ++i) cellnames.push_back(std::to_string(i));
    for (uint32_t i = 0; i < ref_w; ++i) rg.emplace_back(ref_genes[i]);
    for (uint32_t i = 0; i < qry_w; ++i) qg.emplace_back(qry_genes[i]);
    auto* dp = h->dp;
    dp->prepareData(ref_h, ref_w, ref_data, ref_indices, ref_indptr, qry_h, qry_w, qry_data, qry_indices, qry_indptr,
                    codes, ct, cellnames, rg, qg);
    dp->findIntersectionGenes();
    dp->loadRefData();
    dp->trainData();
    dp->loadQryData();
    dp->preprocess();
    h->common.assign(dp->common_genes.begin(), dp->common_genes.end());
    h->thre.assign(dp->thre_genes.begin(), dp->thre_genes.end());
    h->train_idxs = dp->ref_train_idxs;
    h->train_values = dp->ref_train_values;
    h->ctidx = dp->raw_data.ctidx;
    dp->generateDenseMatrix(0, h->max_uniq_s);
    h->s_ref_data = dp->raw_data.ref_data;
    h->s_ref_indices = dp->raw_data.ref_indices;
    h->s_ref_indptr = dp->raw_data.ref_indptr;
    h->s_qry_data = dp->raw_data.qry_data;
    h->s_qry_indices = dp->raw_data.qry_indices;
    h->s_qry_indptr = dp->raw_data.qry_indptr;
    dp->generateDenseMatrix(1, h->max_uniq_f);
    h->ft_ctdiff = dp->raw_data.ctdiff;
    h->ft_ctdidx = dp->raw_data.ctdidx;
    h->f_ref_data = dp->raw_data.ref_data;
    h->f_ref_indices = dp->raw_data.ref_indices;
    h->f_ref_indptr = dp->raw_data.ref_indptr;
    h->f_qry_data = dp->raw_data.qry_data;
    h->f_qry_indices = dp->raw_data.qry_indices;
    h->f_qry_indptr = dp->raw_data.qry_indptr;
    return 0;
}

// Sizes: 0 common, 1 thre, 2 train_values, 3 train_idxs, 4 ft ctdiff, 5 ft ctdidx, 6 ctidx,
// 7 score-step ref nnz, 8 score-step qry nnz, 9 fine-tune ref nnz, 10 fine-tune qry nnz,
// 11 max_uniq_gene (score), 12 max_uniq_gene (fine-tune)
uint64_t ref_count(void* p, int what) {
    auto* h = static_cast<Harness*>(p);
    switch (what) {
        case 0: return h->common.size();
        case 1: return h->thre.size();
        case 2: return h->train_values.size();
        case 3: return h->train_idxs.size();
        case 4: return h->ft_ctdiff.size();
        case 5: return h->ft_ctdidx.size();
        case 6: return h->ctidx.size();
        case 7: return h->s_ref_data.size();
        case 8: return h->s_qry_data.size();
        case 9: return h->f_ref_data.size();
        case 10: return h->f_qry_data.size();
        case 11: return h->max_uniq_s;
        case 12: return h->max_uniq_f;
    }
    return 0;
}

void ref_get_u32(void* p, int what, uint32_t* out) {
    auto* h = static_cast<Harness*>(p);
    const std::vector<uint32_t>* v = nullptr;
    switch (what) {
        case 0: v = &h->common; break;
        case 1: v = &h->thre; break;
        case 2: v = &h->train_values; break;
        case 3: v = &h->train_idxs; break;
        case 4: v = &h->ft_ctdiff; break;
        case 5: v = &h->ft_ctdidx; break;
        case 6: v = &h->ctidx; break;
    }
    if (v) std::copy(v->begin(), v->end(), out);
}

// stage 0: score step (common genes), 1: fine-tune (thre genes); which 0 ref, 1 query
void ref_codes(void* p, int stage, int which, uint16_t* data, int* indices, int* indptr) {
    auto* h = static_cast<Harness*>(p);
    const std::vector<uint16_t>& d = stage == 0 ? (which == 0 ? h->s_ref_data : h->s_qry_data)
                                                : (which == 0 ? h->f_ref_data : h->f_qry_data);
    const std::vector<int>& ix = stage == 0 ? (which == 0 ? h->s_ref_indices : h->s_qry_indices)
                                            : (which == 0 ? h->f_ref_indices : h->f_qry_indices);
    const std::vector<int>& ip = stage == 0 ? (which == 0 ? h->s_ref_indptr : h->s_qry_indptr)
                                            : (which == 0 ? h->f_ref_indptr : h->f_qry_indptr);
    std::copy(d.begin(), d.end(), data);
    std::copy(ix.begin(), ix.end(), indices);
    std::copy(ip.begin(), ip.end(), indptr);
}

float ref_percentile(const float* arr, int len, float p) {
    std::vector<float> v(arr, arr + len);
    return percentile(v, len, p);
}

}  // extern "C"
