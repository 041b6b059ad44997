"""Product host marker training (C ABI, host-only context) against the oracle, and its errors."""

import numpy as np
import pytest

from cusingler_b200 import abi, synth
from tests import helpers as H


def _train(prob):
    a = abi.Annotator(gpuid=-1, cores=4)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    return a


@pytest.mark.parametrize("kind", ["tiny", "families", "small"])
def test_markers_match_oracle(kind):
    prob = H.problem(kind)
    a = _train(prob)
    orc = H.O.Oracle(prob)
    orc.train()
    for what, fn in [(0, orc.common), (1, orc.thre), (2, orc.train_values), (3, orc.train_idxs),
                     (4, orc.ft_ctdiff), (5, orc.ft_ctdidx), (6, orc.ctidx), (7, orc.ref_order)]:
        assert np.array_equal(a.u32(what), fn()), what
    inf = a.info()
    assert inf.n_labels == len(prob.label_names) and inf.filter_genes == 0


def test_markers_gene_filter_matches_oracle():
    ref, qry, L = H.dataset("tiny")
    rg = synth.names("G", ref.n_cols)
    qg = synth.names("G", qry.n_cols)
    rng = np.random.default_rng(7)
    for i in rng.choice(len(rg), 200, replace=False):
        rg[i] = f"R{i}"
    prob = H.O.Problem(ref, qry, synth.names("CT", L), ref.labels, rg, qg)
    a = _train(prob)
    orc = H.O.Oracle(prob)
    orc.train()
    assert a.info().filter_genes == 1
    for what, fn in [(0, orc.common), (1, orc.thre), (2, orc.train_values), (4, orc.ft_ctdiff)]:
        assert np.array_equal(a.u32(what), fn()), what


def test_errors():
    ref, qry, L = H.dataset("tiny")
    names = synth.names("CT", L)
    rg = synth.names("G", ref.n_cols)
    a = abi.Annotator(gpuid=-1)
    # a label name without reference cells (the reference would read an empty vector's front())
    with pytest.raises(abi.SgrError) as e:
        a.train(ref, ref.labels, names + ["EMPTY"], rg, rg)
    assert e.value.status == 5
    # a code beyond the label names (out of bounds in the reference's groupby)
    codes = ref.labels.copy()
    codes[3] = L + 2
    with pytest.raises(abi.SgrError) as e:
        a.train(ref, codes, names, rg, rg)
    assert e.value.status == 1
    # no shared gene name (the reference calls exit(-1))
    with pytest.raises(abi.SgrError) as e:
        a.train(ref, ref.labels, names, rg, [f"X{i}" for i in range(ref.n_cols)])
    assert e.value.status == 4
    # device stages on a host-only context
    a.train(ref, ref.labels, names, rg, rg)
    with pytest.raises(abi.SgrError) as e:
        a.score_first(qry)
    assert e.value.status == 7


def test_codes_are_narrowed_to_8_bits():
    """Codes pass through uint8 as src/io.cpp:813 copies them (256 + l is label l)."""
    prob = H.problem("tiny")
    a = _train(prob)
    b = abi.Annotator(gpuid=-1)
    b.train(prob.ref, prob.celltypes + 256, prob.label_names, prob.ref_genes, prob.qry_genes)
    assert np.array_equal(a.u32(0), b.u32(0))
