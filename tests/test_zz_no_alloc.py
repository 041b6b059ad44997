"""The allocation-free label selection (sgr_select_labels_noalloc) against sgr_score_first.

It serves callers that cannot allocate device memory (their framework owns the GPU's memory, or
they are recording a CUDA graph): it works on device buffers the caller passes and keeps its only
temporary space in a fixed array inside the library.  This file is collected last so that a run
stopping at the first failure has already run every other test; it also passes on its own in a
fresh process.
"""

import numpy as np
import pytest

from cusingler_b200 import abi, synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _case(kind, constant_rows=False):
    prob = H.problem(kind)
    ref, qry = prob.ref, prob.qry
    if constant_rows:
        # empty reference rows make NaN-bearing score lists (the path that uses the fixed scratch)
        ptr = ref.indptr.copy()
        cut = {0, 1, 40}
        rows = [(ref.indices[ptr[i]:ptr[i + 1]], ref.data[ptr[i]:ptr[i + 1]]) if i not in cut else
                (np.zeros(0, np.int32), np.zeros(0, np.float32)) for i in range(ref.n_rows)]
        ind = np.concatenate([r[0] for r in rows]).astype(np.int32)
        dat = np.concatenate([r[1] for r in rows]).astype(np.float32)
        ip = np.zeros(ref.n_rows + 1, np.int32)
        ip[1:] = np.cumsum([len(r[0]) for r in rows])
        ref = synth.CSR(ref.n_rows, ref.n_cols, dat, ind, ip, ref.labels)
        prob = O.Problem(ref, qry, prob.label_names, prob.celltypes, prob.ref_genes, prob.qry_genes)
    a = abi.Annotator(gpuid=0, mode=abi.MODE_EXACT)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    return a, prob


@pytest.mark.parametrize("kind,constant_rows", [("tiny", False), ("tiny", True), ("small", False)])
def test_noalloc_matches_score_first(kind, constant_rows):
    import torch

    a, prob = _case(kind, constant_rows)
    first, scores, flags = a.score_first(prob.qry)
    raw = a.debug_scores(prob.qry)                # Q x R correlations, the same the score step uses
    ranges = a.u32(6)                             # (start, len) of each label's reference columns
    Q, R = raw.shape
    L = len(prob.label_names)
    dev = torch.device("cuda", 0)
    d_scores = torch.from_numpy(raw).to(dev)
    for call in range(2):                         # two calls in a row share the fixed scratch
        d_ls = torch.full((Q, L), -7.0, dtype=torch.float32, device=dev)
        d_first = torch.full((Q,), -1, dtype=torch.int32, device=dev)
        d_flags = torch.full((Q, L), 9, dtype=torch.uint8, device=dev)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        st = abi.select_labels_noalloc(d_scores.data_ptr(), R, Q, ranges, 0.8, 0.05, d_ls.data_ptr(),
                                       d_first.data_ptr(), d_flags.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream)
        assert st == 0
        torch.cuda.synchronize()
        if call == 1:  # (the first call may load the library's module that holds the fixed array)
            assert torch.cuda.mem_get_info(0)[0] == free_before  # the call allocated no device memory
        ls = d_ls.cpu().numpy()
        assert H.ulp_diff(ls, scores).max() == 0, call
        assert np.array_equal(d_first.cpu().numpy(), first), call
        assert np.array_equal(d_flags.cpu().numpy(), flags), call
        if not constant_rows:  # and the oracle's exact-mode labels directly
            res = H.oracle_run(kind, 1)
            assert H.ulp_diff(ls, res["scores"]).max() == 0 and np.array_equal(d_first.cpu().numpy(), res["first"])


def test_noalloc_rejects_oversized_and_bad_ranges():
    # validated on the host before any device work
    big = np.array([0, 200000], np.uint32)
    assert abi.select_labels_noalloc(1, 200000, 1, big, 0.8, 0.05, 1, 1, None) == 6   # UNSUPPORTED
    bad = np.array([0, 10, 10, 10], np.uint32)
    assert abi.select_labels_noalloc(1, 15, 1, bad, 0.8, 0.05, 1, 1, None) == 1       # out of range
    empty = np.array([0, 0], np.uint32)
    assert abi.select_labels_noalloc(1, 15, 1, empty, 0.8, 0.05, 1, 1, None) == 5     # EMPTY_LABEL
