#!/usr/bin/env python
"""Benchmark: query cells/s annotated on B200 (SingleR first + final labels).

Workload (default): the mid-size exact-correlation configuration, 20,000 reference cells x 25,000
genes, 100,000 query cells, ~6 % nonzero float32 CSR of log2(1+x), 30 labels; seeded synthetic
data (no public dataset here).  One step = one full annotation (score step + fine-tune) of the
100,000-cell query batch; the reference preparation (marker training, reference ranks) is done once
before timing and reported as ref_prep_s.

  value  : cells/s with the query CSR already resident in HBM (device pointers into the C ABI)
  e2e    : cells/s through the same C ABI call from pinned host buffers (H2D inside the timed region)
  parity : labels of cells spread over the batch against the oracle (both arithmetic orders), with
           every flip between the exact and the FP32-order arithmetic checked to be a near-tie

Other workloads (--workload):
  stress  60 labels in 12 families of 5 near-identical labels, 50,000 reference x 500,000 query cells
          (fine-tune batching stress); the proposal network is trained on 200,000 cells of the same
          generator
  full    120 labels in 20 families of 6, 100,000 reference cells x 30,000 genes; the timed step is one
          65,536-cell batch
With --stream-cells N (any workload) the chosen form is also streamed over N query cells in
--batch-cells batches from pinned host memory through sgr_annotate_stream (cycling
--distinct-batches seeded batches; 16 x 65,536 distinct cells give the 1,048,576 fresh cells of the
proposal-inference configuration), with p50 / p99 batch latency and agreement with the plain form.

`--impl reference` times the CPU restatement of the reference's path (oracle/, the reference's own
code has no CPU path for its kernels) on every host core, on a bounded sample of the same workload.

Multi-GPU (torchrun): weak scaling, each rank annotates its own query batch with the reference
replicated; no collective in the data path, the max over ranks of the device time is reported.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from cusingler_b200 import synth  # noqa: E402

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0
NEAR_TIE = 1e-5

# DRAM bytes per query row of each score-step kernel, from one ncu capture of the 8,192-query case
# of the mid workload (profiles/corr_tc_mid_8192q.md, select_first_mid_8192q.md,
# rank_kernel_mid_8192q.md: read + write); a launch's traffic is this times its query rows (each
# row's traffic is the same).
TRAFFIC_PER_QUERY = {
    "corr": (1.170260e9 + 0.632710e9) / 8192,
    "select": (0.657572e9 + 4.554752e6) / 8192,
    "rank": (0.098440e9 + 6.304e6) / 8192,
}


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, FALLBACK_BF16_TFLOPS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
            # nvidia-smi's start-up (NVML initialisation) takes driver time: let it finish before the
            # timed steps, whose host round trips it would otherwise stall; its first sample is the
            # clock at the start of the region
            t0 = time.monotonic()
            while not self.rows and self.proc.poll() is None and time.monotonic() - t0 < 10.0:
                time.sleep(0.005)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


DEFAULT_QRY = {"full": 65536}  # the full workload's timed step is one streaming batch


def make_data(args, rank: int):
    wl = synth.WORKLOADS[args.workload]
    world = synth.make_world(wl, 0)
    n_ref = args.n_ref or wl.n_ref
    n_qry = args.n_qry or DEFAULT_QRY.get(args.workload, wl.n_qry)
    ref = synth.generate(world, n_ref, 0)
    qry = synth.generate(world, n_qry, 1 + 1000 * rank)
    return wl, world, ref, qry


def workload_desc(args, wl, n_ref, n_qry):
    """The same string in both arms (the driver compares the arms' configs)."""
    return (f"{args.workload}: {n_ref} ref x {n_qry} query x {wl.n_genes} genes, {wl.n_labels} labels, "
            f"{wl.density:.3f} density")


def oracle_labels(ref, sub, names, genes, mode, cores):
    """Oracle first / final labels, decision margins and the seconds of its score + fine-tune."""
    from oracle import oracle as O

    orc = O.Oracle(O.Problem(ref, sub, names, ref.labels, genes, genes), cores)
    orc.train()
    t0 = time.perf_counter()
    first, _, _, _ = orc.score(mode=mode)
    m_first = orc.margins(0)
    final, _ = orc.finetune(mode=mode)
    dt = time.perf_counter() - t0
    return first, final, m_first, orc.margins(1), dt


def cpu_reference(args, wl, ref, qry, steps, warmup, sample):
    """The CPU restatement of the reference path (oracle, FP32 reference order), all host threads,
    on `sample` query cells per step.  Returns (cells/s, cores, seconds per step)."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    names = synth.names("CT", wl.n_labels)
    genes = synth.names("G", ref.n_cols)
    times = []
    for s in range(warmup + steps):
        a = (s * sample) % max(1, qry.n_rows - sample)
        sub = qry.rows(a, a + sample)
        dt = oracle_labels(ref, sub, names, genes, O.MODE_FP32REF, cores)[4]
        if s >= warmup:
            times.append(dt)
    per_step = sum(times) / len(times)
    return sample / per_step, cores, per_step


def reference_prep(ref, qry, names, genes, sample=256):
    """The reference's own host preparation (its io.cpp compiled from the reference sources into
    oracle/_ref): gene intersection, marker training, and the marker-column filter of the full
    reference and of `sample` query cells, all host threads.  The counterpart of ref_prep_s; None
    when oracle/_ref was not built."""
    from oracle import oracle as O

    if O.ref_lib() is None:
        return None
    cores = os.cpu_count() or 1
    sub = qry.rows(0, min(sample, qry.n_rows))
    prob = O.Problem(ref, sub, names, ref.labels, genes, genes)
    sys.stdout.flush()
    saved = os.dup(1)
    try:  # the reference prints its matrix shapes on stdout; keep the bench line alone there
        with open(os.devnull, "w") as null:
            os.dup2(null.fileno(), 1)
            t0 = time.perf_counter()
            host = O.RefHost(prob, cores)
            dt = time.perf_counter() - t0
    finally:
        os.dup2(saved, 1)
        os.close(saved)
    del host
    return {"seconds": dt, "cores": cores, "kind": "reference",
            "stages": f"prepareData .. trainData .. generateDenseMatrix, full reference and {sub.n_rows} "
                      "query cells"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl, _, ref, qry = make_data(args, 0)
    value, cores, per_step = cpu_reference(args, wl, ref, qry, args.steps, args.warmup, args.cpu_sample)
    line = {
        "metric": "query cells/s annotated (first + final label)", "value": value, "unit": "cells/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1000, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_desc(args, wl, ref.n_rows, qry.n_rows), "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": cores, "kind": "port",
                         "sample": f"{args.cpu_sample} query cells per step, full reference"},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def parity_leg(args, ann, abi, local, wl, ref, qry, names, genes, plain_labels, chosen_labels):
    """Labels of `args.parity_cells` cells spread evenly over the batch against the oracle.

    * the device's exact mode on those cells vs the oracle's exact formula (bit-exact expected);
    * the device's fp32ref mode vs the oracle's FP32-order restatement (bit-exact expected);
    * the timed batch's labels (plain and chosen form) vs the FP32 order: every difference must be a
      near-tie, a cell one of whose decisions compared two values less than 1e-5 apart.
    Also returns the CPU baseline: the oracle's FP32-order time on these cells, all host threads."""
    from oracle import oracle as O

    n = min(args.parity_cells, qry.n_rows)
    idx = np.unique(np.linspace(0, qry.n_rows - 1, n).round().astype(np.int64))
    sub = qry.take(idx)
    cores = os.cpu_count() or 1
    f32, fin32, m32_first, m32_final, t32 = oracle_labels(ref, sub, names, genes, O.MODE_FP32REF, cores)
    fx, finx, _, _, _ = oracle_labels(ref, sub, names, genes, O.MODE_EXACT, cores)
    gx_first, gx_final = ann.annotate(sub)
    a32 = abi.Annotator(gpuid=local, mode=abi.MODE_FP32REF)
    a32.train(ref, ref.labels, names, genes, genes)
    g32_first, g32_final = a32.annotate(sub)
    a32.close()

    def flips(first, final):
        df = np.nonzero(first != f32)[0]
        dn = np.nonzero(final != fin32)[0]
        near = int((m32_first[df] < NEAR_TIE).sum() + (m32_final[dn] < NEAR_TIE).sum())
        return {"first_mismatch": int(df.size), "final_mismatch": int(dn.size), "near_ties": near,
                "unexplained": int(df.size + dn.size - near)}

    out = {
        "cells": int(idx.size), "sample": f"{idx.size} cells evenly spaced over the {qry.n_rows}-cell batch",
        "near_tie": NEAR_TIE,
        "exact_vs_oracle_exact": {"first_mismatch": int((gx_first != fx).sum()),
                                  "final_mismatch": int((gx_final != finx).sum())},
        "fp32ref_vs_oracle_fp32": {"first_mismatch": int((g32_first != f32).sum()),
                                   "final_mismatch": int((g32_final != fin32).sum())},
        "plain_batch_vs_oracle_fp32": flips(plain_labels[0][idx], plain_labels[1][idx]),
        "plain_batch_vs_oracle_exact": {"first_mismatch": int((plain_labels[0][idx] != fx).sum()),
                                        "final_mismatch": int((plain_labels[1][idx] != finx).sum())},
    }
    if chosen_labels is not None:
        out["chosen_batch_vs_oracle_fp32"] = flips(chosen_labels[0][idx], chosen_labels[1][idx])
    cpu = {"value": idx.size / t32, "unit": "cells/s", "cores": cores, "kind": "port",
           "sample": f"{idx.size} query cells spread over the batch, full reference, {t32:.1f} s "
                     "(oracle, FP32 reference order, score step + fine-tune)"}
    return out, cpu


def stream_leg(args, ann, torch, world, wl, rank, learned):
    """Streams `args.stream_cells` query cells through sgr_annotate_stream in `args.batch_cells`
    batches of pinned host memory (cycling `args.distinct_batches` seeded batches), timed with CUDA
    events around whole passes; agreement of the learned labels with a plain pass of the distinct
    batches."""
    nb_distinct = max(1, args.distinct_batches)
    pinned, keep = [], []
    from cusingler_b200 import abi
    for j in range(nb_distinct):
        b = synth.generate(world, args.batch_cells, 10 + j + 1000 * rank)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        d, i, p = pin(b.data), pin(b.indices), pin(b.indptr.astype(np.int32))
        keep.append((d, i, p))
        pinned.append(abi.SgrCsr(b.n_rows, b.n_cols, d.data_ptr(), i.data_ptr(), p.data_ptr(), 0))
    n_batches = max(1, -(-args.stream_cells // args.batch_cells))
    batches = [pinned[k % nb_distinct] for k in range(n_batches)]
    cells = sum(b.n_rows for b in batches)
    h2d = sum(int(keep[k % nb_distinct][2][-1]) * 8 + 4 * (batches[k].n_rows + 1) for k in range(n_batches))
    run = lambda bs, lr: ann.annotate_stream(bs, learned=lr, min_confidence=args.min_confidence,  # noqa: E731
                                             check_fraction=args.check_fraction)
    run(batches[:min(2, n_batches)], learned)  # grows the buffers
    stream = torch.cuda.current_stream()
    times, lat, stats = [], [], None
    for it in range(args.stream_passes):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        first, final, ms, stats = run(batches, learned)
        ev1.record(stream)
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1))
        lat.extend(ms.tolist())
    ms_pass = min(times)
    out = {"cells": cells, "batches": n_batches, "batch_cells": args.batch_cells, "distinct_batches": nb_distinct,
           "form": "learned" if learned else "plain", "ms_per_pass": ms_pass,
           "cells_per_s": cells / (ms_pass / 1000.0), "h2d_bytes_per_pass": h2d,
           "batch_latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                "max": float(np.max(lat))},
           "note": "pinned host batches, upload of batch i + 1 overlapped with batch i; the batch list cycles "
                   "the distinct seeded batches"}
    if learned:
        out["stats"] = stats
        pf, pfin, _, _ = run(pinned, False)
        n0 = sum(b.n_rows for b in pinned)
        out["agreement_vs_plain"] = float((final[:n0] == pfin).mean())
        out["first_equal_plain"] = bool(np.array_equal(first[:n0], pf))
    return out


def sweep(args, ann, abi, torch, csr_dev, stream):
    """Device stage times of the score step (rank, correlation, selection) for every score-step
    shape the autotuner chooses from, on the device-resident batch; first labels must not change."""
    base = None
    shapes = [(pair, gm, mb, sel) for pair in (0, 1) for gm in (1, 16, 64) for mb in (256, 1024)
              for sel in (0, 1, 16)]
    for pair, gm, mb, sel in shapes:
        for what, value in ((5, pair), (6, gm), (2, mb), (7, sel)):
            ann.set_tuning(what, value)
        ann.score_first(csr_dev)
        torch.cuda.synchronize()
        ann.reset_timings()
        ann.set_profiling(True)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            first, _, _ = ann.score_first(csr_dev)
        ev1.record(stream)
        torch.cuda.synchronize()
        ann.set_profiling(False)
        t = ann.timings()
        if base is None:
            base = first
        print(json.dumps({"corr_pair": pair, "corr_gm": gm, "score_chunk_mb": mb, "select_form": sel,
                          "score_step_ms": ev0.elapsed_time(ev1) / args.steps,
                          **{k: t[k] / args.steps for k in ("rank_ms", "corr_ms", "select_ms")},
                          "first_labels_unchanged": bool(np.array_equal(first, base))}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mid", choices=list(synth.WORKLOADS))
    ap.add_argument("--n-ref", type=int, default=0)
    ap.add_argument("--n-qry", type=int, default=0)
    ap.add_argument("--mode", default="exact", choices=["exact", "fp32ref"])
    ap.add_argument("--cpu-sample", type=int, default=96)
    ap.add_argument("--parity-cells", type=int, default=512,
                    help="cells of the batch checked against the oracle (0: no parity leg)")
    ap.add_argument("--form", default="both", choices=["plain", "learned", "both"])
    ap.add_argument("--mlp-train-cells", type=int, default=200000)
    ap.add_argument("--mlp-epochs", type=int, default=40)
    ap.add_argument("--min-confidence", type=float, default=0.98)
    ap.add_argument("--check-fraction", type=float, default=0.01)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp16", action="store_true", help="skip the FP16-operand correlation variant")
    ap.add_argument("--ft-heavy", type=int, default=0,
                    help="pin the fine-tune split threshold and skip the autotuner (profiling runs)")
    ap.add_argument("--ft-warps", type=int, default=8, help="with --ft-heavy: warps per work-queue CTA")
    ap.add_argument("--stream-cells", type=int, default=0, help="stream this many query cells (0: no stream leg)")
    ap.add_argument("--batch-cells", type=int, default=65536)
    ap.add_argument("--distinct-batches", type=int, default=8)
    ap.add_argument("--stream-passes", type=int, default=2)
    ap.add_argument("--sweep", action="store_true",
                    help="time the score step for every score-step shape on the batch (device stage times, one "
                         "JSON line per shape) instead of the bench line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        run_reference_arm(args)
        return

    import torch

    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from cusingler_b200 import abi

    wl, world, ref, qry = make_data(args, rank)
    L = wl.n_labels
    names = synth.names("CT", L)
    genes = synth.names("G", ref.n_cols)
    mode = abi.MODE_EXACT if args.mode == "exact" else abi.MODE_FP32REF
    ann = abi.Annotator(gpuid=local, mode=mode)
    t0 = time.perf_counter()
    ann.train(ref, ref.labels, names, genes, genes)
    ref_prep_s = time.perf_counter() - t0
    info = ann.info()
    stream = torch.cuda.current_stream()
    ann.set_stream(stream.cuda_stream)

    dev = torch.device("cuda", local)
    d_data = torch.from_numpy(qry.data).to(dev)
    d_idx = torch.from_numpy(qry.indices).to(dev)
    d_ptr = torch.from_numpy(qry.indptr.astype(np.int32)).to(dev)
    csr_dev = abi.device_csr(qry.n_rows, qry.n_cols, d_data.data_ptr(), d_idx.data_ptr(), d_ptr.data_ptr())

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.sweep:
        sweep(args, ann, abi, torch, csr_dev, stream)
        ann.close()
        return

    use_learned = args.form in ("learned", "both") and mode == abi.MODE_EXACT
    mlp_info = None
    if use_learned:
        # proposal network: trained once on plain-method labels of a separate seeded query set
        t0 = time.perf_counter()
        train_q = synth.generate(world, args.mlp_train_cells, 2 + 1000 * rank)
        tf, tfin, tsc = ann.annotate(train_q, with_scores=True)
        del train_q
        t1 = time.perf_counter()
        loss = ann.mlp_train(tsc, tfin, epochs=args.mlp_epochs, batch=4096, lr=1e-3, weight_decay=0.01, seed=rank)
        mlp_info = {"train_cells": args.mlp_train_cells, "epochs": args.mlp_epochs, "label_s": t1 - t0,
                    "train_s": time.perf_counter() - t1, "final_loss": loss,
                    "min_confidence": args.min_confidence, "check_fraction": args.check_fraction}

    def run_plain(csr):
        return ann.annotate(csr)

    def run_learned(csr):
        f, fin, st = ann.annotate_learned(csr, min_confidence=args.min_confidence,
                                          check_fraction=args.check_fraction)
        return f, fin, st

    # autotuner: launch shapes timed per form, outside the timed region, on a separate seeded query
    # sample of the same workload (large enough that the learned form routes a representative set
    # of cells to the fine-tune)
    tune_sample = synth.generate(world, min(qry.n_rows, 50000), 3 + 1000 * rank)
    tuning = {}

    def tune(learned):
        if args.ft_heavy:
            ann.set_tuning(0, args.ft_warps)
            ann.set_tuning(1, args.ft_heavy)
            tuning["learned" if learned else "plain"] = {"pinned": True, "ft_warps": args.ft_warps,
                                                          "ft_heavy": args.ft_heavy, "score_chunk_mb": 1024,
                                                          "corr_pair": 0, "corr_gm": 16, "select_warps": 1,
                                                          "pipeline": 0, "corr_wide": 18}
            apply_tuning("learned" if learned else "plain")  # the recorded shapes are the ones timed
            return
        tuning["learned" if learned else "plain"] = ann.autotune(
            tune_sample, learned=learned, min_confidence=args.min_confidence, check_fraction=args.check_fraction)

    def apply_tuning(name):
        t = tuning.get(name)
        if t:
            ann.set_tuning(0, t["ft_warps"])
            ann.set_tuning(1, t["ft_heavy"])
            ann.set_tuning(2, t["score_chunk_mb"])
            if mode == abi.MODE_EXACT:
                ann.set_tuning(5, t["corr_pair"])
            ann.set_tuning(6, t["corr_gm"])
            ann.set_tuning(7, t["select_warps"])
            if mode == abi.MODE_EXACT:
                ann.set_tuning(9, t["pipeline"])
                ann.set_tuning(10, t["corr_wide"])

    def timed(fn, csr, steps, name):
        for _ in range(args.warmup):
            out = fn(csr)
        barrier()
        ann.reset_timings()
        ann.set_profiling(True)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            barrier()
            torch.cuda.nvtx.range_push(name)  # lets a profiler capture the timed steps alone
            ev0.record(stream)
            for _ in range(steps):
                out = fn(csr)
            ev1.record(stream)
            torch.cuda.nvtx.range_pop()
            barrier()
        ann.set_profiling(False)
        return max_over_ranks(ev0.elapsed_time(ev1) / steps), ann.timings(), clk.summary(), out

    def ft_stats(tm, steps):
        return {"ft_cells_per_step": tm["ft_cells"] / steps,
                "ft_rounds_per_cell": tm["ft_cell_rounds"] / max(1, tm["ft_cells"]),
                "ft_candidates_per_cell": tm["ft_candidates"] / max(1, tm["ft_cells"])}

    form_lines = {}
    plain_out = None
    if args.form in ("plain", "both") or not use_learned:
        tune(False)
        ms_plain, tm_plain, clk_plain, plain_out = timed(run_plain, csr_dev, args.steps, "plain")
        form_lines["plain"] = {"value": world_size * qry.n_rows / (ms_plain / 1000.0), "ms_per_step": ms_plain,
                               **ft_stats(tm_plain, args.steps)}
    else:
        plain_out = ann.annotate(csr_dev)
    if use_learned:
        tune(True)
        ms_l, tm_l, clk_l, out_l = timed(run_learned, csr_dev, args.steps, "learned")
        agree = float((out_l[1] == plain_out[1]).mean())
        form_lines["learned"] = {"value": world_size * qry.n_rows / (ms_l / 1000.0), "ms_per_step": ms_l,
                                 "agreement_vs_plain": agree, "first_equal_plain": bool(np.array_equal(out_l[0],
                                                                                                       plain_out[0])),
                                 "stats": out_l[2], **ft_stats(tm_l, args.steps)}
    chosen = "learned" if use_learned and form_lines["learned"]["agreement_vs_plain"] >= 0.999 else "plain"
    if chosen == "learned":
        ms, tm, clk, fn_chosen, chosen_out = ms_l, tm_l, clk_l, run_learned, out_l
    else:
        ms, tm, clk, fn_chosen, chosen_out = ms_plain, tm_plain, clk_plain, run_plain, plain_out
    value = world_size * qry.n_rows / (ms / 1000.0)
    apply_tuning(chosen)  # the chosen form's launch shapes for the e2e leg

    # e2e: host (pinned) inputs through the same call, upload inside the timed region
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h_data, h_idx, h_ptr = pin(qry.data), pin(qry.indices), pin(qry.indptr.astype(np.int32))
    csr_host = abi.SgrCsr(qry.n_rows, qry.n_cols, h_data.data_ptr(), h_idx.data_ptr(), h_ptr.data_ptr(), 0)
    e2e_steps = max(1, min(args.steps, 3))
    host_out = fn_chosen(csr_host)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(e2e_steps):
        host_out = fn_chosen(csr_host)
    ev1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1) / e2e_steps)
    e2e_labels_equal = bool(np.array_equal(host_out[0], chosen_out[0]) and np.array_equal(host_out[1], chosen_out[1]))
    h2d = qry.data.nbytes + qry.indices.nbytes + 4 * (qry.n_rows + 1)
    d2h = 2 * 4 * qry.n_rows
    del h_data, h_idx, h_ptr

    # FP16-operand correlation variant beside the exact INT8 form: score step only, same batch
    fp16 = None
    if mode == abi.MODE_EXACT and world_size == 1 and not args.no_fp16 and info.n_common <= 2048:
        def score_ms():
            ann.score_first(csr_dev)
            barrier()
            ann.reset_timings()
            ann.set_profiling(True)
            for _ in range(args.steps):
                out = ann.score_first(csr_dev)
            barrier()
            ann.set_profiling(False)
            t = ann.timings()
            return t["corr_ms"] / args.steps, t["total_ms"] / args.steps, out
        corr_exact, step_exact, (f_e, s_e, _) = score_ms()
        ann.set_tuning(4, 1)
        corr_f16, step_f16, (f_h, s_h, _) = score_ms()
        sub = qry.rows(0, min(qry.n_rows, 2000))
        raw_f16 = ann.debug_scores(sub)
        ann.set_tuning(4, 0)
        raw_exact = ann.debug_scores(sub)
        fp16 = {"corr_ms": corr_f16, "corr_ms_exact_int8": corr_exact, "score_step_ms": step_f16,
                "score_step_ms_exact_int8": step_exact,
                "max_abs_err_label_scores": float(np.nanmax(np.abs(s_h.astype(np.float64) - s_e))),
                "max_abs_err_scores_2000_cells": float(np.nanmax(np.abs(raw_f16.astype(np.float64) - raw_exact))),
                "first_label_agreement": float((f_h == f_e).mean()),
                "note": "FP16 ranks (exact for G <= 2048), FP32 accumulation; error against the exact FP64 scores"}
        del raw_f16, raw_exact

    stream_out = None
    if args.stream_cells > 0 and world_size == 1:
        del d_data, d_idx, d_ptr
        torch.cuda.empty_cache()
        stream_out = stream_leg(args, ann, torch, world, wl, rank, use_learned)

    hbm, bf16, src = peaks()
    steps = args.steps
    stages = {k: tm[k] / steps for k in ("rank_ms", "corr_ms", "select_ms", "finetune_ms", "mlp_ms")}
    corr_launch_ms = tm["corr_ms"] / max(1, tm["corr_launches"])
    corr_ops_launch = tm["corr_ops"] / max(1, tm["corr_launches"])
    rank_launch_ms = tm["rank_ms"] / max(1, tm["rank_launches"])
    rank_bytes_launch = tm["rank_bytes"] / max(1, tm["rank_launches"])
    int8_peak = 2 * bf16  # dense int8 = 2x dense bf16 on B200; no int8 figure is measured
    rows_corr = qry.n_rows / max(1, tm["corr_launches"] / steps)
    rows_rank = qry.n_rows / max(1, tm["rank_launches"] / steps)
    rows_sel = qry.n_rows / max(1, tm["select_launches"] / steps)
    mid = args.workload == "mid"
    roof_corr = {"kernel": "score-step correlation", "bound": "tensor",
                 "achieved": corr_ops_launch / (corr_launch_ms / 1000) / 1e12, "peak": int8_peak,
                 "unit": "TFLOP/s", "traffic": TRAFFIC_PER_QUERY["corr"] * rows_corr if mid else None,
                 "peak_note": f"int8 dense = 2 x {src} bf16 cuBLAS ({bf16} TFLOP/s)"}
    roof_corr["frac"] = roof_corr["achieved"] / roof_corr["peak"]
    roof_rank = {"kernel": "gather + rank", "bound": "hbm",
                 "achieved": rank_bytes_launch / (rank_launch_ms / 1000) / 1e9, "peak": hbm, "unit": "GB/s",
                 "traffic": TRAFFIC_PER_QUERY["rank"] * rows_rank if mid else None,
                 "peak_note": f"{src} copy bandwidth"}
    roof_rank["frac"] = roof_rank["achieved"] / roof_rank["peak"]
    sel_launch_ms = tm["select_ms"] / max(1, tm["select_launches"])
    sel_bytes_launch = tm["select_bytes"] / max(1, tm["select_launches"])
    roof_sel = {"kernel": "per-label quantile select", "bound": "hbm",
                "achieved": sel_bytes_launch / (sel_launch_ms / 1000) / 1e9, "peak": hbm, "unit": "GB/s",
                "traffic": TRAFFIC_PER_QUERY["select"] * rows_sel if mid else None,
                "peak_note": f"{src} copy bandwidth"}
    roof_sel["frac"] = roof_sel["achieved"] / roof_sel["peak"]
    # the dominant kernel with a roofline of its own: fine-tune is reported in stages_ms (it is bound by
    # issue and L1 gathers over L2-resident data, not by HBM or the tensor pipe)
    cands = [(stages["corr_ms"], roof_corr), (stages["rank_ms"], roof_rank), (stages["select_ms"], roof_sel)]
    dominant = max(cands, key=lambda c: c[0])[1]

    parity = cpu = None
    if rank == 0 and world_size == 1 and args.parity_cells > 0 and mode == abi.MODE_EXACT:
        parity, cpu = parity_leg(args, ann, abi, local, wl, ref, qry, names, genes, plain_out,
                                 chosen_out if chosen != "plain" else None)
    if args.no_cpu_baseline:
        cpu = None
    elif cpu is None and rank == 0 and world_size == 1:
        v, cores, per = cpu_reference(args, wl, ref, qry, 1, 0, args.cpu_sample)
        cpu = {"value": v, "unit": "cells/s", "cores": cores, "kind": "port",
               "sample": f"{args.cpu_sample} query cells of the same batch, full reference, {per:.1f} s"}
    ref_prep_cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        ref_prep_cpu = reference_prep(ref, qry, names, genes)

    if rank == 0:
        line = {
            "metric": "query cells/s annotated (first + final label)", "value": value, "unit": "cells/s",
            "n_gpus": world_size, "steps": steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int8" if mode == abi.MODE_EXACT else "f32", "data": "synthetic",
            "config": {"workload": workload_desc(args, wl, ref.n_rows, qry.n_rows),
                       "form": f"{chosen} ({args.mode})", "l2": "inputs larger than L2 (query CSR "
                                                             f"{h2d / 1e9:.2f} GB)",
                       "marker_genes": info.n_common, "finetune_genes": info.n_thre,
                       "parallelism": f"query sharding x{world_size}"},
            "e2e": {"value": world_size * qry.n_rows / (e2e_ms / 1000.0), "unit": "cells/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "e2e_labels_equal_device_input": e2e_labels_equal,
            "gpu_launches": int(tm["launches"]),
            "roofline": dominant, "rooflines": [roof_corr, roof_rank, roof_sel],
            "stages_ms": stages, "ref_prep_s": ref_prep_s, "ref_prep_reference": ref_prep_cpu,
            "forms": form_lines, "mlp": mlp_info,
            "tuning": tuning, "fp16_variant": fp16, "parity": parity, "stream": stream_out,
            **ft_stats(tm, steps),
            "clocks": clk, "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ann.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
