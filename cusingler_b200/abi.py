"""ctypes binding of the C ABI in include/sgr.h (libsgr.so).

This is the package's Python API over the native library: every call goes through the C ABI, and
importing it fails loudly when the library is missing (there is no CPU fallback).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsgr.so")

SGR_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "OUT_OF_MEMORY", 4: "NO_INTERSECTION",
    5: "EMPTY_LABEL", 6: "UNSUPPORTED", 7: "STATE", 8: "TIMEOUT",
}
MODE_EXACT = 0
MODE_FP32REF = 1

# Every symbol include/sgr.h declares.
SYMBOLS = [
    "sgr_create", "sgr_destroy", "sgr_last_error", "sgr_set_mode", "sgr_train_ref", "sgr_score_first",
    "sgr_finetune", "sgr_annotate", "sgr_get_info", "sgr_get_u32", "sgr_debug_ranks", "sgr_debug_scores",
    "sgr_debug_stl_sort", "sgr_debug_stl_minmax", "sgr_set_stream", "sgr_set_profiling", "sgr_reset_timings",
    "sgr_get_timings", "sgr_select_labels_noalloc", "sgr_mlp_train", "sgr_mlp_predict", "sgr_mlp_params",
    "sgr_mlp_load", "sgr_mlp_debug_grads", "sgr_annotate_learned", "sgr_set_tuning", "sgr_autotune",
    "sgr_annotate_stream",
]


class SgrCsr(C.Structure):
    _fields_ = [("n_rows", C.c_uint32), ("n_cols", C.c_uint32), ("data", C.c_void_p),
                ("indices", C.c_void_p), ("indptr", C.c_void_p), ("on_device", C.c_int32)]


class SgrInfo(C.Structure):
    _fields_ = [("n_labels", C.c_uint32), ("n_genes", C.c_uint32), ("n_common", C.c_uint32),
                ("n_thre", C.c_uint32), ("filter_genes", C.c_uint32), ("ref_rows", C.c_uint32),
                ("n_pair_genes", C.c_uint64)]


class SgrTimings(C.Structure):
    _fields_ = [("h2d_ms", C.c_double), ("rank_ms", C.c_double), ("corr_ms", C.c_double),
                ("select_ms", C.c_double), ("finetune_ms", C.c_double), ("total_ms", C.c_double),
                ("launches", C.c_uint64), ("corr_launches", C.c_uint64), ("rank_launches", C.c_uint64),
                ("rank_bytes", C.c_uint64), ("corr_ops", C.c_uint64), ("cells", C.c_uint64),
                ("ft_cell_rounds", C.c_uint64), ("mlp_ms", C.c_double), ("select_launches", C.c_uint64),
                ("select_bytes", C.c_uint64), ("ft_queue_cells", C.c_uint64), ("ft_split_cells", C.c_uint64),
                ("ft_split_rounds", C.c_uint64), ("ft_split_rows", C.c_uint64), ("ft_cells", C.c_uint64),
                ("ft_candidates", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SgrTuning(C.Structure):
    _fields_ = [("ft_warps", C.c_int32), ("ft_heavy", C.c_int32), ("score_chunk_mb", C.c_int32),
                ("trials", C.c_int32), ("best_ms", C.c_double), ("worst_ms", C.c_double),
                ("corr_pair", C.c_int32), ("corr_gm", C.c_int32), ("select_warps", C.c_int32),
                ("score_trials", C.c_int32), ("score_best_ms", C.c_double), ("pipeline", C.c_int32),
                ("corr_wide", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SgrMlpConfig(C.Structure):
    _fields_ = [("hidden", C.c_uint32), ("epochs", C.c_uint32), ("batch", C.c_uint32), ("lr", C.c_float),
                ("weight_decay", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("seed", C.c_uint64)]


class SgrLearnedStats(C.Structure):
    _fields_ = [("cells", C.c_uint64), ("decided", C.c_uint64), ("finetuned", C.c_uint64),
                ("checked", C.c_uint64), ("check_agree", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SgrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib():
    """Load libsgr.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m cusingler_b200.build` (or "
                              "__graft_entry__.build()) to compile the CUDA library")
        L = C.CDLL(LIB_PATH)
        vp, u32, i32, f32 = C.c_void_p, C.c_uint32, C.c_int32, C.c_float
        sig = {
            "sgr_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(vp)]),
            "sgr_destroy": (C.c_int, [vp]),
            "sgr_last_error": (C.c_char_p, [vp]),
            "sgr_set_mode": (C.c_int, [vp, C.c_int]),
            "sgr_train_ref": (C.c_int, [vp, C.POINTER(SgrCsr), vp, vp, u32, vp, vp, u32]),
            "sgr_score_first": (C.c_int, [vp, C.POINTER(SgrCsr), f32, f32, vp, vp, vp]),
            "sgr_finetune": (C.c_int, [vp, C.POINTER(SgrCsr), vp, f32, f32, i32, vp, vp]),
            "sgr_annotate": (C.c_int, [vp, C.POINTER(SgrCsr), f32, f32, i32, vp, vp, vp]),
            "sgr_get_info": (C.c_int, [vp, C.POINTER(SgrInfo)]),
            "sgr_get_u32": (C.c_int, [vp, C.c_int, vp, C.c_uint64]),
            "sgr_debug_ranks": (C.c_int, [vp, C.POINTER(SgrCsr), C.c_int, vp]),
            "sgr_debug_scores": (C.c_int, [vp, C.POINTER(SgrCsr), vp]),
            "sgr_debug_stl_sort": (None, [vp, i32]),
            "sgr_debug_stl_minmax": (None, [vp, i32, C.POINTER(i32), C.POINTER(i32)]),
            "sgr_set_stream": (C.c_int, [vp, vp]),
            "sgr_set_profiling": (C.c_int, [vp, C.c_int]),
            "sgr_set_tuning": (C.c_int, [vp, C.c_int, C.c_int]),
            "sgr_autotune": (C.c_int, [vp, C.POINTER(SgrCsr), f32, f32, i32, i32, f32, f32, C.POINTER(SgrTuning)]),
            "sgr_reset_timings": (C.c_int, [vp]),
            "sgr_get_timings": (C.c_int, [vp, C.POINTER(SgrTimings)]),
            "sgr_select_labels_noalloc": (C.c_int, [vp, C.c_int64, u32, vp, u32, f32, f32, vp, vp, vp, vp]),
            "sgr_annotate_stream": (C.c_int, [vp, vp, u32, f32, f32, i32, i32, f32, f32, vp, vp, vp,
                                              C.POINTER(SgrLearnedStats)]),
            "sgr_mlp_train": (C.c_int, [vp, vp, vp, u32, C.POINTER(SgrMlpConfig), C.POINTER(f32)]),
            "sgr_mlp_predict": (C.c_int, [vp, vp, u32, vp, vp]),
            "sgr_mlp_params": (C.c_int, [vp, vp, C.c_uint64, C.POINTER(u32), C.POINTER(u32), C.POINTER(C.c_uint64)]),
            "sgr_mlp_load": (C.c_int, [vp, vp, u32, u32]),
            "sgr_mlp_debug_grads": (C.c_int, [vp, vp, vp, u32, vp, C.POINTER(f32)]),
            "sgr_annotate_learned": (C.c_int, [vp, C.POINTER(SgrCsr), f32, f32, C.c_int32, f32, f32, vp, vp,
                                               C.POINTER(SgrLearnedStats)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _strs(xs):
    arr = (C.c_char_p * len(xs))()
    arr[:] = [s.encode() if isinstance(s, str) else bytes(s) for s in xs]
    return arr


def host_csr(n_rows, n_cols, data, indices, indptr):
    """Keep-alive tuple (struct, arrays) of a host CSR in the library's layout."""
    d = np.ascontiguousarray(data, np.float32)
    i = np.ascontiguousarray(indices, np.int32)
    p = np.ascontiguousarray(indptr, np.int32)
    return SgrCsr(n_rows, n_cols, d.ctypes.data, i.ctypes.data, p.ctypes.data, 0), (d, i, p)


def device_csr(n_rows, n_cols, data_ptr, indices_ptr, indptr_ptr):
    """A CSR already in device memory (raw pointers, e.g. torch tensors' data_ptr())."""
    return SgrCsr(n_rows, n_cols, data_ptr, indices_ptr, indptr_ptr, 1)


class Annotator:
    """One GPU context: train on a labelled reference once, then annotate query batches."""

    def __init__(self, gpuid: int = 0, cores: int = 0, mode: int = MODE_EXACT):
        self.L = lib()
        self.h = C.c_void_p()
        st = self.L.sgr_create(gpuid, cores or os.cpu_count() or 1, C.byref(self.h))
        if st != SGR_OK:
            raise SgrError(st, f"cannot create a context on GPU {gpuid}")
        self.set_mode(mode)
        self.n_labels = 0

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.sgr_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        self.close()

    def _check(self, st):
        if st != SGR_OK:
            raise SgrError(st, self.L.sgr_last_error(self.h).decode())

    def set_mode(self, mode: int):
        self._check(self.L.sgr_set_mode(self.h, mode))

    def train(self, ref, celltypes, label_names, ref_genes, qry_genes):
        """`ref`: an object with n_rows, n_cols, data, indices, indptr (host arrays)."""
        csr, keep = host_csr(ref.n_rows, ref.n_cols, ref.data, ref.indices, ref.indptr)
        ct = np.ascontiguousarray(celltypes, np.int32)
        ln, rg, qg = _strs(label_names), _strs(ref_genes), _strs(qry_genes)
        self._check(self.L.sgr_train_ref(self.h, C.byref(csr), ct.ctypes.data, C.cast(ln, C.c_void_p),
                                         len(label_names), C.cast(rg, C.c_void_p), C.cast(qg, C.c_void_p),
                                         len(qry_genes)))
        self.n_labels = len(label_names)
        return self

    def _csr(self, q):
        if isinstance(q, SgrCsr):
            return q, None
        return host_csr(q.n_rows, q.n_cols, q.data, q.indices, q.indptr)

    def score_first(self, qry, quantile=0.8, thre=0.05):
        csr, keep = self._csr(qry)
        Q, L = csr.n_rows, self.n_labels
        first = np.zeros(Q, np.int32)
        scores = np.zeros((Q, L), np.float32)
        flags = np.zeros((Q, L), np.uint8)
        self._check(self.L.sgr_score_first(self.h, C.byref(csr), quantile, thre, first.ctypes.data,
                                           scores.ctypes.data, flags.ctypes.data))
        return first, scores, flags

    def finetune(self, qry, flags, quantile=0.8, thre=0.05, times=0):
        csr, keep = self._csr(qry)
        Q = csr.n_rows
        fl = np.ascontiguousarray(flags, np.uint8)
        final = np.zeros(Q, np.int32)
        rounds = np.zeros(Q, np.int32)
        self._check(self.L.sgr_finetune(self.h, C.byref(csr), fl.ctypes.data, quantile, thre, times,
                                        final.ctypes.data, rounds.ctypes.data))
        return final, rounds

    def annotate(self, qry, quantile=0.8, thre=0.05, times=0, with_scores=False):
        csr, keep = self._csr(qry)
        Q, L = csr.n_rows, self.n_labels
        first = np.zeros(Q, np.int32)
        final = np.zeros(Q, np.int32)
        scores = np.zeros((Q, L), np.float32) if with_scores else None
        self._check(self.L.sgr_annotate(self.h, C.byref(csr), quantile, thre, times, first.ctypes.data,
                                        final.ctypes.data, _ptr(scores)))
        return (first, final, scores) if with_scores else (first, final)

    # ---- learned proposal ----------------------------------------------------------------------
    def mlp_train(self, label_scores, targets, epochs=20, batch=4096, lr=1e-3, weight_decay=0.01, hidden=256,
                  seed=0):
        x = np.ascontiguousarray(label_scores, np.float32)
        y = np.ascontiguousarray(targets, np.int32)
        cfg = SgrMlpConfig(hidden, epochs, batch, lr, weight_decay, 0.9, 0.999, 1e-8, seed)
        loss = C.c_float()
        self._check(self.L.sgr_mlp_train(self.h, x.ctypes.data, y.ctypes.data, len(y), C.byref(cfg), C.byref(loss)))
        return loss.value

    def mlp_predict(self, label_scores):
        x = np.ascontiguousarray(label_scores, np.float32)
        n = x.shape[0]
        lab = np.zeros(n, np.int32)
        conf = np.zeros(n, np.float32)
        self._check(self.L.sgr_mlp_predict(self.h, x.ctypes.data, n, lab.ctypes.data, conf.ctypes.data))
        return lab, conf

    def mlp_params(self):
        L, H, n = C.c_uint32(), C.c_uint32(), C.c_uint64()
        self._check(self.L.sgr_mlp_params(self.h, None, 0, C.byref(L), C.byref(H), C.byref(n)))
        out = np.zeros(n.value, np.float32)
        self._check(self.L.sgr_mlp_params(self.h, out.ctypes.data, out.size, None, None, None))
        return out, L.value, H.value

    def mlp_load(self, params, n_labels, hidden):
        p = np.ascontiguousarray(params, np.float32)
        self._check(self.L.sgr_mlp_load(self.h, p.ctypes.data, n_labels, hidden))

    def mlp_debug_grads(self, features, targets):
        x = np.ascontiguousarray(features, np.float32)
        y = np.ascontiguousarray(targets, np.int32)
        params, L, H = self.mlp_params()
        g = np.zeros_like(params)
        loss = C.c_float()
        self._check(self.L.sgr_mlp_debug_grads(self.h, x.ctypes.data, y.ctypes.data, len(y), g.ctypes.data,
                                               C.byref(loss)))
        return g, loss.value

    def annotate_learned(self, qry, quantile=0.8, thre=0.05, times=0, min_confidence=0.98, check_fraction=0.01):
        csr, keep = self._csr(qry)
        Q = csr.n_rows
        first = np.zeros(Q, np.int32)
        final = np.zeros(Q, np.int32)
        st = SgrLearnedStats()
        self._check(self.L.sgr_annotate_learned(self.h, C.byref(csr), quantile, thre, times, min_confidence,
                                                check_fraction, first.ctypes.data, final.ctypes.data, C.byref(st)))
        return first, final, st.as_dict()

    def annotate_stream(self, batches, quantile=0.8, thre=0.05, times=0, learned=False, min_confidence=0.98,
                        check_fraction=0.01):
        """Annotate a sequence of host CSR batches (objects with n_rows, n_cols, data, indices, indptr,
        or SgrCsr views of page-locked memory); batch i + 1 uploads while batch i runs.  Returns
        (first, final, batch_ms, stats): labels of all rows in batch order, per-batch latency from
        upload start to labels on the host, and the learned form's routing counts."""
        views, keep = [], []
        for b in batches:
            c, k = self._csr(b)
            views.append(c)
            keep.append(k)
        arr = (SgrCsr * max(1, len(views)))(*views)
        n = sum(v.n_rows for v in views)
        first = np.zeros(n, np.int32)
        final = np.zeros(n, np.int32)
        ms = np.zeros(len(views), np.float32)
        st = SgrLearnedStats()
        self._check(self.L.sgr_annotate_stream(self.h, C.cast(arr, C.c_void_p), len(views), quantile, thre, times,
                                               1 if learned else 0, min_confidence, check_fraction,
                                               first.ctypes.data, final.ctypes.data, ms.ctypes.data, C.byref(st)))
        return first, final, ms, st.as_dict()

    def set_stream(self, stream_ptr):
        """Run on a caller's CUDA stream (e.g. torch.cuda.current_stream().cuda_stream); None = own."""
        self._check(self.L.sgr_set_stream(self.h, stream_ptr))

    def autotune(self, sample, learned=False, quantile=0.8, thre=0.05, times=0, min_confidence=0.98,
                 check_fraction=0.01) -> dict:
        """Time every launch-shape candidate on `sample` and keep the fastest (see sgr_autotune)."""
        csr, keep = self._csr(sample)
        out = SgrTuning()
        self._check(self.L.sgr_autotune(self.h, C.byref(csr), quantile, thre, times, 1 if learned else 0,
                                        min_confidence, check_fraction, C.byref(out)))
        return out.as_dict()

    def set_tuning(self, what: int, value: int):
        self._check(self.L.sgr_set_tuning(self.h, what, value))

    def set_profiling(self, on: bool = True):
        self._check(self.L.sgr_set_profiling(self.h, 1 if on else 0))

    def reset_timings(self):
        self._check(self.L.sgr_reset_timings(self.h))

    def timings(self) -> dict:
        t = SgrTimings()
        self._check(self.L.sgr_get_timings(self.h, C.byref(t)))
        return t.as_dict()

    def info(self) -> SgrInfo:
        out = SgrInfo()
        self._check(self.L.sgr_get_info(self.h, C.byref(out)))
        return out

    def u32(self, what: int) -> np.ndarray:
        inf = self.info()
        L = inf.n_labels
        n = {0: inf.n_common, 1: inf.n_thre, 2: inf.n_pair_genes, 3: 2 * L * L, 5: 2 * L * L, 6: 2 * L,
             7: inf.ref_rows}.get(what)
        if what == 4:
            idx = self.u32(5)
            n = int(idx[-2] + idx[-1]) if len(idx) else 0
            n = max(n, int(max((idx[0::2] + idx[1::2]).max(initial=0), 0)))
        out = np.zeros(max(int(n), 1), np.uint32)
        self._check(self.L.sgr_get_u32(self.h, what, out.ctypes.data, out.size))
        return out[:int(n)]

    def debug_ranks(self, rows=None):
        inf = self.info()
        if rows is None:
            out = np.zeros((inf.ref_rows, inf.n_common), np.int32)
            self._check(self.L.sgr_debug_ranks(self.h, None, 1, out.ctypes.data))
            return out
        csr, keep = self._csr(rows)
        out = np.zeros((csr.n_rows, inf.n_common), np.int32)
        self._check(self.L.sgr_debug_ranks(self.h, C.byref(csr), 0, out.ctypes.data))
        return out

    def debug_scores(self, qry):
        inf = self.info()
        csr, keep = self._csr(qry)
        out = np.zeros((csr.n_rows, inf.ref_rows), np.float32)
        self._check(self.L.sgr_debug_scores(self.h, C.byref(csr), out.ctypes.data))
        return out


def select_labels_noalloc(d_scores, ld, n_rows, label_ranges, quantile, thre, d_label_scores, d_first, d_flags,
                          stream=None):
    """Allocation-free label selection on device buffers the caller owns (raw device pointers).

    For callers that cannot allocate device memory (a framework that owns the GPU's memory, a
    CUDA graph being recorded): the library uses a fixed 4 MiB device array of its own instead.
    Returns the status code (0 = OK)."""
    r = np.ascontiguousarray(label_ranges, np.uint32)
    return lib().sgr_select_labels_noalloc(d_scores, ld, n_rows, r.ctypes.data, len(r) // 2, quantile, thre,
                                           d_label_scores, d_first, d_flags, stream)


def stl_sort(v):
    a = np.array(v, np.float32)
    lib().sgr_debug_stl_sort(a.ctypes.data, len(a))
    return a


def stl_minmax(v):
    a = np.ascontiguousarray(v, np.float32)
    mn, mx = C.c_int32(), C.c_int32()
    lib().sgr_debug_stl_minmax(a.ctypes.data, len(a), C.byref(mn), C.byref(mx))
    return mn.value, mx.value
