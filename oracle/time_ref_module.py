"""TEST INFRASTRUCTURE ONLY: times the reference's own GPU module (oracle/_ref/cusingler*.so, built
from the reference sources for sm_100a by `make -C oracle ref`) on seeded synthetic workloads, as a
comparison point for the B200 path.  It is never part of the product path.

The reference's `run()` takes Python lists, so the list conversion is done before the clock starts;
the timed call includes the reference's own host stages (marker training, gene filter, value codes),
its score step and its per-cell fine-tune loop, as a user of `run()` would see them.

Usage (on a machine with a GPU, from the repository root):
    python oracle/time_ref_module.py [--workload small|mid] [--n-qry N]
Prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from cusingler_b200 import synth  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="small", choices=["small", "mid"])
    ap.add_argument("--n-qry", type=int, default=0, help="query cells (default: the workload's)")
    ap.add_argument("--cores", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    sys.path.insert(0, os.path.join(HERE, "_ref"))
    import cusingler as ref_module  # the reference's own module

    wl = synth.WORKLOADS[args.workload]
    world = synth.make_world(wl, 0)
    ref = synth.generate(world, wl.n_ref, 0)
    n_qry = args.n_qry or wl.n_qry
    qry = synth.generate(world, n_qry, 1)
    labels = synth.names("CT", wl.n_labels)
    genes = synth.names("G", ref.n_cols)
    cells = [f"c{i}" for i in range(qry.n_rows)]
    t0 = time.perf_counter()
    ref_args = (ref.data.tolist(), ref.indices.tolist(), ref.indptr.astype("int64").tolist())
    qry_args = (qry.data.tolist(), qry.indices.tolist(), qry.indptr.astype("int64").tolist())
    conv_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = ref_module.run(args.cores, 0, ref.n_rows, ref.n_cols, *ref_args, qry.n_rows, qry.n_cols, *qry_args,
                         labels, ref.labels.tolist(), cells, genes, genes, quantile=80, finetune_thre=0.05,
                         finetune_times=0)
    run_s = time.perf_counter() - t0
    assert len(res) == qry.n_rows
    print(json.dumps({"impl": "reference GPU module (sm_100a build of the reference sources)",
                      "workload": f"{args.workload}: {ref.n_rows} ref x {qry.n_rows} query x {ref.n_cols} genes, "
                                  f"{wl.n_labels} labels",
                      "cores": args.cores, "run_s": run_s, "cells_per_s": qry.n_rows / run_s,
                      "list_conversion_s": conv_s}), flush=True)


if __name__ == "__main__":
    main()
