"""libsgr.so loads (no GPU needed) and exports every function include/sgr.h declares."""

import ctypes
import os
import re

from cusingler_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "sgr.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sgr_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header_symbols():
    lib = ctypes.CDLL(abi.LIB_PATH)
    names = declared()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
    assert set(abi.SYMBOLS) <= set(names)


def test_dropin_module_imports():
    from cusingler import cusingler
    assert hasattr(cusingler, "run")
    assert cusingler.__version__
    doc = cusingler.run.__doc__
    for arg in ("cores", "gpuid", "ref_height", "qry_indptr", "codes", "celltype", "cellnames",
                "ref_geneidx", "qry_geneidx", "quantile", "finetune_thre", "finetune_times"):
        assert arg in doc
