"""Golden labels produced by the reference's own module (compiled from its sources for sm_100a and
run on a B200 by tests/golden/make_golden.py): the oracle must reproduce them exactly (CPU), and
the device path must too in fp32ref mode, and in exact mode except at documented near-ties."""

import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
META = json.load(open(os.path.join(HERE, "golden.json")))


def _load(name):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    ref, qry, L, rg, qg, run_kw = mg.build_case(name)
    assert mg.checksum(ref, qry, rg, qg) == META[name]["checksum"], "generator drifted from the fixture"
    g = np.load(os.path.join(HERE, f"{name}.npz"))
    kw = META[name]["run_kwargs"]
    names = [f"CT{i}" for i in range(L)]
    return O.Problem(ref, qry, names, ref.labels, rg, qg), kw, g["first"], g["final"]


def _fp32_margins(prob, kw):
    """The oracle's FP32-order decision margins of every query cell (score step; whole path)."""
    orc = O.Oracle(prob)
    orc.train()
    q = float(np.float32(kw["quantile"]) / np.float32(100))
    orc.score(quantile=q, thre=kw["finetune_thre"], mode=O.MODE_FP32REF)
    m0 = orc.margins(0)
    orc.finetune(quantile=q, thre=kw["finetune_thre"], times=kw["finetune_times"], mode=O.MODE_FP32REF)
    return m0, orc.margins(1)


CASES = sorted(META)


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_labels(name):
    prob, kw, first, final = _load(name)
    orc = O.Oracle(prob)
    orc.train()
    q = np.float32(kw["quantile"]) / np.float32(100)
    f, _, _, _ = orc.score(quantile=float(q), thre=kw["finetune_thre"], mode=O.MODE_FP32REF)
    fin, _ = orc.finetune(quantile=float(q), thre=kw["finetune_thre"], times=kw["finetune_times"],
                          mode=O.MODE_FP32REF)
    assert np.array_equal(f, first)
    assert np.array_equal(fin, final)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_reproduces_reference_labels(name):
    from cusingler_b200 import abi
    prob, kw, first, final = _load(name)
    q = float(np.float32(kw["quantile"]) / np.float32(100))
    for mode in (abi.MODE_FP32REF, abi.MODE_EXACT):
        a = abi.Annotator(gpuid=0, mode=mode)
        a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
        f, fin = a.annotate(prob.qry, quantile=q, thre=kw["finetune_thre"], times=kw["finetune_times"])
        if mode == abi.MODE_FP32REF:
            assert np.array_equal(f, first) and np.array_equal(fin, final)
        else:
            # exact scores differ from the reference's FP32 sums by < 1e-5; a label may only differ
            # where one of its decisions compared two values within that distance (a near-tie)
            from tests import helpers as H
            m_first, m_final = _fp32_margins(prob, kw)
            assert len(H.unexplained_flips(f, first, m_first)) == 0
            assert len(H.unexplained_flips(fin, final, m_final)) == 0
