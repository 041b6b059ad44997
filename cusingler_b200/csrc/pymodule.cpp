// Drop-in pybind11 module `cusingler` with the reference's `run` signature
// (src/main.cpp:32-52, 68-88 of STOmics/cusingler): train on the reference CSR, score, fine-tune,
// return [[cell, firstLabel, finalLabel], ...] in query order (src/pipeline.cpp:158-164).
//
// Differences from the reference, all on the error path or in the input conversion:
// * errors raise RuntimeError (the reference calls exit(), which ends the interpreter);
// * numeric arrays are taken as numpy buffers without an element-wise copy (lists still work);
// * label names, cell names and gene names may be str or bytes (h5py yields bytes).

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "sgr.h"

namespace py = pybind11;
using namespace pybind11::literals;

namespace {

using farr = py::array_t<float, py::array::c_style | py::array::forcecast>;
using iarr = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;

std::vector<std::string> to_strings(const py::handle& h) {
    std::vector<std::string> out;
    for (auto item : py::iter(h)) {
        if (py::isinstance<py::bytes>(item)) out.push_back(item.cast<std::string>());
        else out.push_back(py::str(item).cast<std::string>());
    }
    return out;
}

std::vector<const char*> cptrs(const std::vector<std::string>& v) {
    std::vector<const char*> p;
    for (auto& s : v) p.push_back(s.c_str());
    return p;
}

struct Ctx {
    sgr_ctx* c = nullptr;
    ~Ctx() { sgr_destroy(c); }
    void check(sgr_status st, const char* what) {
        if (st != SGR_OK) throw std::runtime_error(std::string(what) + ": " + sgr_last_error(c));
    }
};

sgr_csr make_csr(uint32_t h, uint32_t w, const farr& d, const iarr& i, const iarr& p, const char* what) {
    if ((size_t)p.size() != (size_t)h + 1) throw std::invalid_argument(std::string(what) + ": indptr length != height + 1");
    int64_t nnz = p.at(h);
    if (d.size() < nnz || i.size() < nnz) throw std::invalid_argument(std::string(what) + ": data/indices shorter than indptr[-1]");
    return sgr_csr{h, w, d.data(), i.data(), p.data(), 0};
}

py::list run(int cores, int gpuid, uint32_t ref_height, uint32_t ref_width, farr ref_data, iarr ref_indices,
             iarr ref_indptr, uint32_t qry_height, uint32_t qry_width, farr qry_data, iarr qry_indices,
             iarr qry_indptr, py::object codes, iarr celltypes, py::object cellnames, py::object ref_geneidx,
             py::object qry_geneidx, float quantile, float finetune_thre, int finetune_times) {
    auto label_names = to_strings(codes);
    auto cells = to_strings(cellnames);
    auto rg = to_strings(ref_geneidx);
    auto qg = to_strings(qry_geneidx);
    if (rg.size() != ref_width || qg.size() != qry_width)
        throw std::invalid_argument("gene name count differs from the matrix width");
    if ((size_t)celltypes.size() != ref_height) throw std::invalid_argument("celltype length != ref_height");
    if (cells.size() != qry_height) throw std::invalid_argument("cellnames length != qry_height");
    sgr_csr ref = make_csr(ref_height, ref_width, ref_data, ref_indices, ref_indptr, "reference");
    sgr_csr qry = make_csr(qry_height, qry_width, qry_data, qry_indices, qry_indptr, "query");
    auto ln = cptrs(label_names), rgp = cptrs(rg), qgp = cptrs(qg);
    std::vector<int32_t> first(qry_height), fin(qry_height);
    {
        py::gil_scoped_release nogil;
        Ctx c;
        if (sgr_create(gpuid, cores, &c.c) != SGR_OK) throw std::runtime_error("cannot initialise GPU " + std::to_string(gpuid));
        c.check(sgr_train_ref(c.c, &ref, celltypes.data(), ln.data(), (uint32_t)ln.size(), rgp.data(), qgp.data(),
                              (uint32_t)qgp.size()),
                "train");
        // `quantile` is a percent, divided in float as src/main.cpp:47 does
        c.check(sgr_annotate(c.c, &qry, quantile / 100, finetune_thre, finetune_times, first.data(), fin.data(), nullptr),
                "annotate");
    }
    py::list res;
    for (uint32_t i = 0; i < qry_height; ++i) {
        py::list row;
        row.append(cells[i]);
        row.append(label_names.at(first[i]));
        row.append(label_names.at(fin[i]));
        res.append(row);
    }
    return res;
}

}  // namespace

PYBIND11_MODULE(cusingler, m) {
    m.doc() = "SingleR cell annotation on a B200 (drop-in for the cusingler module)";
    m.def("run", &run,
          "Annotate query cells against a labelled reference; returns [[cell, firstLabel, finalLabel], ...].",
          "cores"_a, "gpuid"_a, "ref_height"_a, "ref_width"_a, "ref_data"_a, "ref_indices"_a, "ref_indptr"_a,
          "qry_height"_a, "qry_width"_a, "qry_data"_a, "qry_indices"_a, "qry_indptr"_a, "codes"_a, "celltype"_a,
          "cellnames"_a, "ref_geneidx"_a, "qry_geneidx"_a, "quantile"_a = 80, "finetune_thre"_a = 0.05,
          "finetune_times"_a = 0);
#ifdef VERSION_INFO
    m.attr("__version__") = VERSION_INFO;
#else
    m.attr("__version__") = "dev";
#endif
}
