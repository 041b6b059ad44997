"""Marker training on the device (per-label medians, per-pair marker lists, gene sets) against the
oracle, whose host stages are pinned to the reference's own io.cpp: every list sgr_get_u32 returns is
identical, on the seeded workloads, on values with negatives and stored zeros, on pairs with fewer
positive-difference genes than the marker count (zero and negative genes fill the score-step set),
and on pair lists longer than a CTA's shared-memory sort."""

import numpy as np
import pytest

from cusingler_b200 import abi, synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu

WHATS = [(0, "common"), (1, "thre"), (2, "train_values"), (3, "train_idxs"), (4, "ft_ctdiff"), (5, "ft_ctdidx"),
         (6, "ctidx"), (7, "ref_order")]


def _check(prob):
    a = abi.Annotator(gpuid=0)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    orc = O.Oracle(prob)
    orc.train()
    for what, name in WHATS:
        assert np.array_equal(a.u32(what), getattr(orc, name)()), name
    # the host restatement gives the same lists
    h = abi.Annotator(gpuid=0)
    h.set_tuning(8, 1)
    h.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    for what, name in WHATS:
        assert np.array_equal(a.u32(what), h.u32(what)), name
    return a


def _dense_problem(X, labels, n_labels, seed=0):
    """A problem from a dense reference matrix (zeros stay implicit unless `X` holds -0.0 markers)."""
    rows, cols = np.nonzero(X)
    ref = synth.CSR(X.shape[0], X.shape[1], X[rows, cols].astype(np.float32), cols.astype(np.int32),
                    np.concatenate([[0], np.cumsum(np.count_nonzero(X, axis=1))]).astype(np.int32),
                    np.asarray(labels, np.int32))
    qry = ref.rows(0, min(8, ref.n_rows))
    genes = synth.names("G", X.shape[1])
    return O.Problem(ref, qry, synth.names("CT", n_labels), ref.labels, genes, genes)


@pytest.mark.parametrize("kind", ["tiny", "families", "small"])
def test_device_training_matches_oracle(kind):
    _check(H.problem(kind))


def test_device_training_gene_filter():
    ref, qry, L = H.dataset("tiny")
    rg = synth.names("G", ref.n_cols)
    qg = synth.names("G", qry.n_cols)
    for i in np.random.default_rng(7).choice(len(rg), 200, replace=False):
        rg[i] = f"R{i}"
    a = _check(O.Problem(ref, qry, synth.names("CT", L), ref.labels, rg, qg))
    assert a.info().filter_genes == 1


def test_negative_values_stored_zeros_and_odd_even_labels():
    """Values of both signs and explicitly stored zeros; labels of 1, 2, 3 and many cells."""
    rng = np.random.default_rng(11)
    labels = np.concatenate([[0], [1, 1], [2, 2, 2], rng.integers(3, 6, 200)])
    X = rng.normal(0, 1, (labels.size, 400)).astype(np.float32)
    X[rng.random(X.shape) < 0.6] = 0
    X[:, :40] += labels[:, None].astype(np.float32)  # a label signal on the first genes
    prob = _dense_problem(X, labels, 6)
    # stored zeros: re-add some zero entries to the CSR
    ref = prob.ref
    keep_zero = rng.random(ref.data.size) < 0.1
    ref.data[keep_zero] = 0.0
    _check(prob)


def test_pairs_with_few_positive_genes():
    """60 labels on 50 genes with dense values: most pairs have fewer than the 46 marker genes per
    pair with a positive difference, so zero- and negative-difference genes complete the set."""
    rng = np.random.default_rng(5)
    labels = np.repeat(np.arange(60), 5)
    X = (rng.gamma(2.0, 1.0, (labels.size, 50)) + labels[:, None] % 7).astype(np.float32)
    _check(_dense_problem(X, labels, 60))


def test_pair_lists_longer_than_shared_memory():
    """Two labels over 10,000 genes where one label is higher on nearly every gene: the pair list
    (about 10,000 genes) is sorted in the global scratch path."""
    rng = np.random.default_rng(3)
    labels = np.repeat([0, 1], 40)
    X = (rng.gamma(2.0, 1.0, (labels.size, 10000)) + 3.0 * (labels[:, None] == 0)).astype(np.float32)
    _check(_dense_problem(X, labels, 2))
