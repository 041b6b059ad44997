"""TEST INFRASTRUCTURE ONLY: ctypes access to the oracle (liboracle.so) and to the reference's own
host code (oracle/_ref/libref_host.so).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs import this
module, as the checker.  The product package never does.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_host.so")
REF_MODULE_DIR = os.path.join(HERE, "_ref")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C")

MODE_FP32REF = 0
MODE_EXACT = 1


def build(ref: bool = False, ref_src: str | None = None) -> None:
    """Compile the oracle (and, with ref=True, oracle/_ref from the reference sources in ref_src)."""
    targets = ["all"] + (["ref"] if ref else [])
    extra = [f"REF={ref_src}"] if ref and ref_src else []
    subprocess.run(["make", "-s", "-C", HERE] + targets + extra, check=True)


def _strs(xs):
    arr = (C.c_char_p * len(xs))()
    arr[:] = [s.encode() for s in xs]
    return arr


def _load(path, protos):
    lib = C.CDLL(path)
    for name, (res, args) in protos.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        load_args = [C.c_void_p, C.c_uint32, C.c_uint32, _f32p, _i32p, _i32p, C.c_uint32, C.c_uint32, _f32p,
                     _i32p, _i32p, C.c_void_p, C.c_uint32, _i32p, C.c_void_p, C.c_void_p]
        _lib = _load(LIB, {
            "or_create": (C.c_void_p, [C.c_int]),
            "or_destroy": (None, [C.c_void_p]),
            "or_error": (C.c_char_p, [C.c_void_p]),
            "or_load": (C.c_int, load_args),
            "or_train": (C.c_int, [C.c_void_p]),
            "or_count": (C.c_uint32, [C.c_void_p, C.c_int]),
            "or_get_u32": (None, [C.c_void_p, C.c_int, _u32p]),
            "or_rank_row": (None, [C.c_void_p, C.c_int, C.c_uint32, _i32p]),
            "or_codes": (None, [C.c_void_p, C.c_int, _u16p, _i32p, _i32p]),
            "or_score": (C.c_int, [C.c_void_p, C.c_float, C.c_float, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
            "or_finetune": (C.c_int, [C.c_void_p, C.c_float, C.c_float, C.c_int, C.c_int, _i32p, C.c_void_p]),
            "or_set_flags": (None, [C.c_void_p, _f32p]),
            "or_margins": (None, [C.c_void_p, C.c_int, _f32p]),
            "or_percentile": (C.c_float, [_f32p, C.c_int, C.c_float]),
            "or_minmax": (None, [_f32p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "or_sort": (None, [_f32p, C.c_int]),
        })
    return _lib


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            return None
        run_args = [C.c_void_p, C.c_uint32, C.c_uint32, _f32p, _i32p, _i32p, C.c_uint32, C.c_uint32, _f32p,
                    _i32p, _i32p, C.c_void_p, C.c_uint32, _i32p, C.c_void_p, C.c_void_p]
        _ref = _load(REF_LIB, {
            "ref_create": (C.c_void_p, [C.c_int]),
            "ref_destroy": (None, [C.c_void_p]),
            "ref_run": (C.c_int, run_args),
            "ref_count": (C.c_uint64, [C.c_void_p, C.c_int]),
            "ref_get_u32": (None, [C.c_void_p, C.c_int, _u32p]),
            "ref_codes": (None, [C.c_void_p, C.c_int, C.c_int, _u16p, _i32p, _i32p]),
            "ref_percentile": (C.c_float, [_f32p, C.c_int, C.c_float]),
        })
    return _ref


def _csr_args(m):
    return (np.ascontiguousarray(m.data, np.float32), np.ascontiguousarray(m.indices, np.int32),
            np.ascontiguousarray(m.indptr, np.int32))


class Problem:
    """Inputs in the reference's `run` layout (src/main.cpp:32-52)."""

    def __init__(self, ref, qry, label_names, celltypes, ref_genes, qry_genes):
        self.ref, self.qry = ref, qry
        self.label_names = list(label_names)
        self.celltypes = np.ascontiguousarray(celltypes, np.int32)
        self.ref_genes, self.qry_genes = list(ref_genes), list(qry_genes)

    def load_args(self):
        rd, ri, rp = _csr_args(self.ref)
        qd, qi, qp = _csr_args(self.qry)
        self._keep = (_strs(self.label_names), _strs(self.ref_genes), _strs(self.qry_genes))
        return (self.ref.n_rows, self.ref.n_cols, rd, ri, rp, self.qry.n_rows, self.qry.n_cols, qd, qi, qp,
                C.cast(self._keep[0], C.c_void_p), len(self.label_names), self.celltypes,
                C.cast(self._keep[1], C.c_void_p), C.cast(self._keep[2], C.c_void_p))


class Oracle:
    def __init__(self, problem: Problem, cores: int = 0):
        self.L = lib()
        self.p = problem
        self.h = self.L.or_create(cores or os.cpu_count() or 1)
        self.L.or_load(self.h, *problem.load_args())

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_destroy(self.h)
            self.h = None

    def error(self) -> str:
        return self.L.or_error(self.h).decode()

    def train(self) -> None:
        if self.L.or_train(self.h) != 0:
            raise RuntimeError(self.error())

    def u32(self, what: int, count_what: int | None = None, n: int | None = None) -> np.ndarray:
        if n is None:
            n = self.L.or_count(self.h, count_what)
        out = np.zeros(n, np.uint32)
        if n:
            self.L.or_get_u32(self.h, what, out)
        return out

    @property
    def n_labels(self):
        return len(self.p.label_names)

    def common(self):
        return self.u32(0, 0)

    def thre(self):
        return self.u32(1, 1)

    def train_values(self):
        return self.u32(2, 2)

    def train_idxs(self):
        return self.u32(3, n=2 * self.n_labels ** 2)

    def ft_ctdiff(self):
        return self.u32(4, 3)

    def ft_ctdidx(self):
        return self.u32(5, n=2 * self.n_labels ** 2)

    def ctidx(self):
        return self.u32(6, n=2 * self.n_labels)

    def ref_order(self):
        return self.u32(7, n=self.p.ref.n_rows)

    def filter_genes(self) -> bool:
        return bool(self.L.or_count(self.h, 4))

    def rank_row(self, which: int, row: int) -> np.ndarray:
        G = len(self.common())
        out = np.zeros(G, np.int32)
        self.L.or_rank_row(self.h, which, row, out)
        return out

    def codes(self, which: int):
        nnz = self.L.or_count(self.h, 6 if which == 0 else 5)
        rows = self.p.ref.n_rows if which == 0 else self.p.qry.n_rows
        d = np.zeros(nnz, np.uint16)
        i = np.zeros(nnz, np.int32)
        p = np.zeros(rows + 1, np.int32)
        self.L.or_codes(self.h, which, d, i, p)
        return d, i, p

    def score(self, quantile=0.8, thre=0.05, mode=MODE_FP32REF, raw=False):
        Q, L, R = self.p.qry.n_rows, self.n_labels, self.p.ref.n_rows
        first = np.zeros(Q, np.int32)
        scores = np.zeros((Q, L), np.float32)
        flags = np.zeros((Q, L), np.float32)
        raw_arr = np.zeros((Q, R), np.float32) if raw else None
        rc = self.L.or_score(self.h, quantile, thre, mode, first.ctypes.data, scores.ctypes.data,
                             flags.ctypes.data, raw_arr.ctypes.data if raw else None)
        if rc:
            raise RuntimeError(self.error())
        return first, scores, flags, raw_arr

    def margins(self, which: int) -> np.ndarray:
        """Per query cell, the smallest distance between a label score and a value it was compared
        with (the maximum, the minimum, the keep bound) in the last score (which 0) or fine-tune
        (which 1, every round and the score step) call.  A label that differs between the exact and
        the FP32-order arithmetic with a margin below the score difference of the two (< 1e-5) is a
        near-tie."""
        out = np.zeros(self.p.qry.n_rows, np.float32)
        self.L.or_margins(self.h, which, out)
        return out

    def set_flags(self, flags):
        self.L.or_set_flags(self.h, np.ascontiguousarray(flags, np.float32))

    def finetune(self, quantile=0.8, thre=0.05, times=0, mode=MODE_FP32REF):
        Q = self.p.qry.n_rows
        final = np.zeros(Q, np.int32)
        rounds = np.zeros(Q, np.int32)
        rc = self.L.or_finetune(self.h, quantile, thre, times, mode, final, rounds.ctypes.data)
        if rc:
            raise RuntimeError(self.error())
        return final, rounds


class RefHost:
    """The reference's own io.cpp host stages (compiled from its sources into oracle/_ref)."""

    def __init__(self, problem: Problem, cores: int = 0):
        self.L = ref_lib()
        if self.L is None:
            raise FileNotFoundError(REF_LIB)
        self.p = problem
        self.h = self.L.ref_create(cores or os.cpu_count() or 1)
        self.L.ref_run(self.h, *problem.load_args())

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def count(self, what):
        return int(self.L.ref_count(self.h, what))

    def u32(self, what):
        n = self.count(what)
        out = np.zeros(n, np.uint32)
        if n:
            self.L.ref_get_u32(self.h, what, out)
        return out

    def codes(self, stage, which):
        nnz = self.count(7 + 2 * stage + which)
        rows = self.p.ref.n_rows if which == 0 else self.p.qry.n_rows
        d = np.zeros(nnz, np.uint16)
        i = np.zeros(nnz, np.int32)
        p = np.zeros(rows + 1, np.int32)
        self.L.ref_codes(self.h, stage, which, d, i, p)
        return d, i, p


def percentile(arr, p):
    a = np.ascontiguousarray(arr, np.float32)
    return float(lib().or_percentile(a, len(a), p))


def ref_percentile(arr, p):
    a = np.ascontiguousarray(arr, np.float32)
    return float(ref_lib().ref_percentile(a, len(a), p))


def minmax(v):
    a = np.ascontiguousarray(v, np.float32)
    mn, mx = C.c_int(), C.c_int()
    lib().or_minmax(a, len(a), C.byref(mn), C.byref(mx))
    return mn.value, mx.value


def std_sort(v):
    a = np.array(v, np.float32)
    lib().or_sort(a, len(a))
    return a
