"""Parity on the mid-size shape (20,000 reference cells x 25,000 genes, 30 labels, ~6 % nonzero,
about 1,070 score-step marker genes) with 2,000 query cells, through the C ABI against the oracle.

* exact mode: first labels, label scores and final labels bit-exact with the oracle's exact formula;
* fp32ref mode: the same, bit-exact with the oracle's restatement of the reference's FP32 order;
* exact vs the reference's FP32 order: every first or final label that differs is a near-tie (one of
  its decisions compared two values less than 1e-5 apart in the FP32-order run).
"""

import numpy as np
import pytest

from cusingler_b200 import abi, synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _mid_problem(n_qry=2000):
    wl = synth.WORKLOADS["mid"]
    world = synth.make_world(wl, 0)
    ref = synth.generate(world, wl.n_ref, 0)
    qry = synth.generate(world, n_qry, 1)
    genes = synth.names("G", ref.n_cols)
    return O.Problem(ref, qry, synth.names("CT", wl.n_labels), ref.labels, genes, genes)


def _oracle(prob, mode):
    orc = O.Oracle(prob)
    orc.train()
    first, scores, _, _ = orc.score(mode=mode)
    m_first = orc.margins(0)
    final, rounds = orc.finetune(mode=mode)
    return dict(first=first, scores=scores, final=final, rounds=rounds, m_first=m_first, m_final=orc.margins(1))


def test_mid_shape_labels_match_oracle():
    prob = _mid_problem()
    fp = _oracle(prob, O.MODE_FP32REF)
    ex = _oracle(prob, O.MODE_EXACT)
    for mode, want in ((abi.MODE_EXACT, ex), (abi.MODE_FP32REF, fp)):
        a = abi.Annotator(gpuid=0, mode=mode)
        a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
        first, final, scores = a.annotate(prob.qry, with_scores=True)
        assert H.ulp_diff(scores, want["scores"]).max() == 0, mode
        assert np.array_equal(first, want["first"]), mode
        assert np.array_equal(final, want["final"]), mode
        if mode == abi.MODE_EXACT:
            assert np.nanmax(np.abs(scores.astype(np.float64) - fp["scores"])) < H.NEAR_TIE
            assert len(H.unexplained_flips(first, fp["first"], fp["m_first"])) == 0
            assert len(H.unexplained_flips(final, fp["final"], fp["m_final"])) == 0
        a.close()
