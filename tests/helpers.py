"""Shared test helpers: seeded problems in the reference's `run` layout, oracle and product runs."""

from __future__ import annotations

import functools

import numpy as np

from cusingler_b200 import synth
from oracle import oracle as O


@functools.lru_cache(maxsize=None)
def dataset(kind: str):
    """(ref, qry, n_labels) for a named small case."""
    if kind == "small":  # the 1,900 x 800 x 15,000-gene, 13-label workload
        w, ref, qry = synth.make_dataset("small", workers=1)
        return ref, qry, 13
    if kind == "tiny":
        w, ref, qry = synth.custom_dataset(600, 160, 3000, 7, 0.08, seed=3)
        return ref, qry, 7
    if kind == "families":
        w, ref, qry = synth.custom_dataset(900, 200, 4000, 10, 0.07, block=(20, 40, 3.0, 4.0),
                                           families=(2, 5, (6, 10), 1.5), seed=5)
        return ref, qry, 10
    raise KeyError(kind)


def problem(kind: str) -> O.Problem:
    ref, qry, L = dataset(kind)
    return O.Problem(ref, qry, synth.names("CT", L), ref.labels, synth.names("G", ref.n_cols),
                     synth.names("G", qry.n_cols))


@functools.lru_cache(maxsize=None)
def oracle_run(kind: str, mode: int, times: int = 0):
    """Oracle first labels, label scores, flags, raw scores, final labels and rounds."""
    orc = O.Oracle(problem(kind))
    orc.train()
    first, scores, flags, raw = orc.score(mode=mode, raw=True)
    margin_first = orc.margins(0)
    final, rounds = orc.finetune(mode=mode, times=times)
    return dict(first=first, scores=scores, flags=flags, raw=raw, final=final, rounds=rounds, oracle=orc,
                margin_first=margin_first, margin_final=orc.margins(1))


NEAR_TIE = 1e-5  # exact and FP32-order scores differ by less than this (tested per score)


def unexplained_flips(labels, ref_labels, margins, tol=NEAR_TIE):
    """Cells whose label differs from `ref_labels` although the oracle's decision margin there is
    at least `tol` (a flip that arithmetic order cannot explain).  Empty when every difference is a
    near-tie."""
    diff = np.nonzero(np.asarray(labels) != np.asarray(ref_labels))[0]
    return diff[~(np.asarray(margins)[diff] < tol)]


def ulp_diff(a, b):
    """Distance in float32 ulps (NaN == NaN counts as 0)."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, np.int64(-2**31) - ia, ia)
    ib = np.where(ib < 0, np.int64(-2**31) - ib, ib)
    d = np.abs(ia - ib)
    both_nan = np.isnan(a) & np.isnan(b)
    return np.where(both_nan, 0, d)
