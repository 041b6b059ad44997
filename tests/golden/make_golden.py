"""Generate golden first/final labels by running the reference's own module on a GPU.

The reference's pybind11 module is compiled from its sources for sm_100a by `make -C oracle ref`
(oracle/_ref/cusingler*.so).  This script runs its `cusingler.run(...)` on seeded synthetic cases
and writes, per case, the reference's first and final labels together with the generator
parameters and a checksum of the inputs (the inputs are regenerated by the tests, not stored).

Run on a machine with a GPU, from the repository root:
    python tests/golden/make_golden.py [out_dir]        (default: tests/golden)
"""

from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cusingler_b200 import synth  # noqa: E402

# name -> (generator kwargs, gene-name edit, extra run kwargs, row edits)
CASES = {
    "tiny": (dict(n_ref=600, n_qry=160, n_genes=3000, n_labels=7, density=0.08, seed=3), None, {}, None),
    "families": (dict(n_ref=900, n_qry=200, n_genes=4000, n_labels=10, density=0.07, block=(20, 40, 3.0, 4.0),
                      families=(2, 5, (6, 10), 1.5), seed=5), None, {}, None),
    "small": (None, None, {}, None),
    "tiny_times1": (dict(n_ref=600, n_qry=160, n_genes=3000, n_labels=7, density=0.08, seed=3), None,
                    {"finetune_times": 1}, None),
    "tiny_q60": (dict(n_ref=600, n_qry=160, n_genes=3000, n_labels=7, density=0.08, seed=3), None,
                 {"quantile": 60, "finetune_thre": 0.1}, None),
    "genefilter": (dict(n_ref=700, n_qry=150, n_genes=3500, n_labels=8, density=0.08, seed=11), "rename", {}, None),
    "constant_rows": (dict(n_ref=600, n_qry=160, n_genes=3000, n_labels=7, density=0.08, seed=3), None, {},
                      "empty"),
}


def build_case(name):
    kw, genes_edit, run_kw, rows_edit = CASES[name]
    if kw is None:
        w, ref, qry = synth.make_dataset("small", workers=1)
        L = 13
    else:
        w, ref, qry = synth.custom_dataset(workers=1, **kw)
        L = kw["n_labels"]
    ref_genes = synth.names("G", ref.n_cols)
    qry_genes = synth.names("G", qry.n_cols)
    if genes_edit == "rename":
        for i in range(0, len(qry_genes), 9):
            qry_genes[i] = f"Q{i}"
        for i in range(3, len(ref_genes), 13):
            ref_genes[i] = f"R{i}"
    if rows_edit == "empty":
        ref = _empty_rows(ref, [0, 1, 50, 51, 52])
        qry = _empty_rows(qry, [3, 7])
    return ref, qry, L, ref_genes, qry_genes, run_kw


def _empty_rows(m, rows):
    rows = set(rows)
    parts_i, parts_d, ptr = [], [], [0]
    for i in range(m.n_rows):
        a, b = int(m.indptr[i]), int(m.indptr[i + 1])
        if i in rows:
            a = b
        parts_i.append(m.indices[a:b])
        parts_d.append(m.data[a:b])
        ptr.append(ptr[-1] + (b - a))
    return synth.CSR(m.n_rows, m.n_cols, np.concatenate(parts_d).astype(np.float32),
                     np.concatenate(parts_i).astype(np.int32), np.array(ptr, np.int32), m.labels)


def checksum(ref, qry, ref_genes, qry_genes):
    h = hashlib.sha256()
    for m in (ref, qry):
        for a in (m.data, m.indices, m.indptr, m.labels):
            h.update(np.ascontiguousarray(a).tobytes())
    h.update("\n".join(ref_genes).encode())
    h.update("\n".join(qry_genes).encode())
    return h.hexdigest()


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden")
    os.makedirs(out_dir, exist_ok=True)
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import cusingler as ref_module  # the reference's own module, compiled from its sources

    meta = {}
    for name in CASES:
        ref, qry, L, ref_genes, qry_genes, run_kw = build_case(name)
        labels = synth.names("CT", L)
        cells = [f"c{i}" for i in range(qry.n_rows)]
        kw = dict(quantile=80, finetune_thre=0.05, finetune_times=0)
        kw.update(run_kw)
        res = ref_module.run(8, 0, ref.n_rows, ref.n_cols, ref.data.tolist(), ref.indices.tolist(),
                             ref.indptr.astype(np.int64).tolist(), qry.n_rows, qry.n_cols, qry.data.tolist(),
                             qry.indices.tolist(), qry.indptr.astype(np.int64).tolist(), labels,
                             ref.labels.tolist(), cells, ref_genes, qry_genes, **kw)
        assert [r[0] for r in res] == cells
        first = np.array([labels.index(r[1]) for r in res], np.int32)
        final = np.array([labels.index(r[2]) for r in res], np.int32)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), first=first, final=final)
        meta[name] = {"checksum": checksum(ref, qry, ref_genes, qry_genes), "run_kwargs": kw,
                      "n_qry": int(qry.n_rows), "n_labels": L}
        print(name, "first", np.bincount(first, minlength=L).tolist(), "final changed", int((first != final).sum()),
              flush=True)
    with open(os.path.join(out_dir, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
