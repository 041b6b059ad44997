"""The oracle checked against the reference's own host code, compiled from its sources into
oracle/_ref (gene intersection, label regrouping, marker training, the marker-column filter with
per-row value codes, and percentile()).  Skipped where oracle/_ref was not built (it needs the
reference sources, which only the build container has)."""

import numpy as np
import pytest

from cusingler_b200 import synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.skipif(O.ref_lib() is None, reason="oracle/_ref not built")


def _compare_host(prob):
    orc = O.Oracle(prob)
    orc.train()
    ref = O.RefHost(prob)
    for what, fn in [(0, orc.common), (1, orc.thre), (2, orc.train_values), (3, orc.train_idxs),
                     (4, orc.ft_ctdiff), (5, orc.ft_ctdidx), (6, orc.ctidx)]:
        assert np.array_equal(fn(), ref.u32(what)), what
    for which in (0, 1):
        a = orc.codes(which)
        b = ref.codes(0, which)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("kind", ["tiny", "families", "small"])
def test_host_stages_match_reference(kind):
    _compare_host(H.problem(kind))


def test_gene_filter_path_matches_reference():
    """Different gene name sets: intersection, removeCols, original ref width kept (io.cpp:362)."""
    ref, qry, L = H.dataset("tiny")
    rg = synth.names("G", ref.n_cols)
    qg = synth.names("G", qry.n_cols)
    rng = np.random.default_rng(1)
    # drop ~10 % of names on each side by renaming them
    for i in rng.choice(len(rg), len(rg) // 10, replace=False):
        rg[i] = f"R{i}"
    for i in rng.choice(len(qg), len(qg) // 10, replace=False):
        qg[i] = f"Q{i}"
    prob = O.Problem(ref, qry, synth.names("CT", L), ref.labels, rg, qg)
    orc = O.Oracle(prob)
    orc.train()
    assert orc.filter_genes()
    _compare_host(prob)


def test_percentile_matches_reference():
    rng = np.random.default_rng(0)
    for _ in range(3000):
        n = int(rng.integers(1, 400))
        v = rng.uniform(-1, 1, n).astype(np.float32)
        if rng.random() < 0.3:
            v = np.round(v * 8) / 8
        for p in (0.8, 0.5, 0.0, 1.0, 0.999, 0.01):
            assert O.percentile(v, p) == O.ref_percentile(v, p) or (
                np.isnan(O.percentile(v, p)) and np.isnan(O.ref_percentile(v, p)))


def test_percentile_known_answers():
    # values computed by the reference's percentile() (src/cusingler.cu:947) on the CPU
    assert O.ref_percentile([0.1, 0.5, 0.3, 0.9, 0.7], 0.8) == np.float32(0.74000001)
    assert O.ref_percentile([0.1, 0.2, 0.3, 0.4], 0.8) == np.float32(0.340000004)
    assert O.percentile([0.1, 0.5, 0.3, 0.9, 0.7], 0.8) == np.float32(0.74000001)
