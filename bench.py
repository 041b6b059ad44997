#!/usr/bin/env python
"""Benchmark: query cells/s annotated on B200 (SingleR first + final labels).

Workload (default): the mid-size exact-correlation configuration, 20,000 reference cells x 25,000
genes, 100,000 query cells, ~6 % nonzero float32 CSR of log2(1+x), 30 labels; seeded synthetic
data (no public dataset here).  One step = one full annotation (score step + fine-tune) of the
100,000-cell query batch; the reference preparation (marker training, reference ranks) is done once
before timing and reported as ref_prep_s.

  value : cells/s with the query CSR already resident in HBM (device pointers into the C ABI)
  e2e   : cells/s through the same C ABI call from pinned host buffers (H2D inside the timed region)

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


# DRAM bytes per query row of each score-step kernel, from one ncu capture of the 8,192-query case
# (profiles/corr_tc_mid_8192q.md, select_first_mid_8192q.md, rank_kernel_mid_8192q.md: read +
# write); a launch's traffic is this times its query rows (each row's traffic is the same).
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


def make_data(args, rank: int):
    wl = synth.WORKLOADS[args.workload]
    world = synth.make_world(wl, 0)
    n_ref = args.n_ref or wl.n_ref
    n_qry = args.n_qry or wl.n_qry
    ref = synth.generate(world, n_ref, 0)
    qry = synth.generate(world, n_qry, 1 + 1000 * rank)
    return wl, ref, qry


def cpu_reference(args, wl, ref, qry, steps, warmup, sample):
    """The CPU restatement of the reference path (oracle), all host threads, on `sample` query
    cells per step.  Returns (cells/s, cores, seconds per step)."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    L = wl.n_labels
    names = synth.names("CT", L)
    genes = synth.names("G", ref.n_cols)
    times = []
    for s in range(warmup + steps):
        a = (s * sample) % max(1, qry.n_rows - sample)
        sub = qry.rows(a, a + sample)
        orc = O.Oracle(O.Problem(ref, sub, names, ref.labels, genes, genes), cores)
        orc.train()
        t0 = time.perf_counter()
        orc.score(mode=O.MODE_FP32REF)
        orc.finetune(mode=O.MODE_FP32REF)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
    per_step = sum(times) / len(times)
    return sample / per_step, cores, per_step


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl, ref, qry = make_data(args, 0)
    value, cores, per_step = cpu_reference(args, wl, ref, qry, args.steps, args.warmup, args.cpu_sample)
    line = {
        "metric": "query cells/s annotated (first + final label)", "value": value, "unit": "cells/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1000, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {wl.n_ref} ref x {wl.n_qry} query x {wl.n_genes} genes, "
                               f"{wl.n_labels} labels", "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": cores, "kind": "port",
                         "sample": f"{args.cpu_sample} query cells per step, full reference"},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


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
    ap.add_argument("--form", default="both", choices=["plain", "learned", "both"])
    ap.add_argument("--mlp-train-cells", type=int, default=200000)
    ap.add_argument("--mlp-epochs", type=int, default=40)
    ap.add_argument("--min-confidence", type=float, default=0.98)
    ap.add_argument("--check-fraction", type=float, default=0.01)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ft-heavy", type=int, default=0,
                    help="pin the fine-tune split threshold and skip the autotuner (profiling runs)")
    ap.add_argument("--ft-warps", type=int, default=8, help="with --ft-heavy: warps per work-queue CTA")
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

    wl, ref, qry = make_data(args, rank)
    L = wl.n_labels
    names = synth.names("CT", L)
    genes = synth.names("G", ref.n_cols)
    mode = abi.MODE_EXACT if args.mode == "exact" else abi.MODE_FP32REF
    ann = abi.Annotator(gpuid=local, mode=mode)
    t0 = time.perf_counter()
    ann.train(ref, ref.labels, names, genes, genes)
    ref_prep_s = time.perf_counter() - t0
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

    use_learned = args.form in ("learned", "both") and mode == abi.MODE_EXACT
    mlp_info = None
    if use_learned:
        # proposal network: trained once on plain-method labels of a separate seeded query set
        t0 = time.perf_counter()
        train_q = synth.generate(synth.make_world(wl, 0), args.mlp_train_cells, 2 + 1000 * rank)
        tf, tfin, tsc = ann.annotate(train_q, with_scores=True)
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
    tune_sample = synth.generate(synth.make_world(wl, 0), min(qry.n_rows, 50000), 3 + 1000 * rank)
    tuning = {}

    def tune(learned):
        if args.ft_heavy:
            ann.set_tuning(0, args.ft_warps)
            ann.set_tuning(1, args.ft_heavy)
            tuning["learned" if learned else "plain"] = {"pinned": True, "ft_warps": args.ft_warps,
                                                          "ft_heavy": args.ft_heavy, "score_chunk_mb": 1024}
            return
        tuning["learned" if learned else "plain"] = ann.autotune(
            tune_sample, learned=learned, min_confidence=args.min_confidence, check_fraction=args.check_fraction)

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

    form_lines = {}
    ms_plain = tm_plain = clk_plain = None
    if args.form in ("plain", "both") or not use_learned:
        tune(False)
        ms_plain, tm_plain, clk_plain, out = timed(run_plain, csr_dev, args.steps, "plain")
        plain_final = out[1]
        form_lines["plain"] = {"value": world_size * qry.n_rows / (ms_plain / 1000.0), "ms_per_step": ms_plain}
    else:
        plain_final = ann.annotate(csr_dev)[1]
    if use_learned:
        tune(True)
        ms_l, tm_l, clk_l, out = timed(run_learned, csr_dev, args.steps, "learned")
        agree = float((out[1] == plain_final).mean())
        form_lines["learned"] = {"value": world_size * qry.n_rows / (ms_l / 1000.0), "ms_per_step": ms_l,
                                 "agreement_vs_plain": agree, "stats": out[2]}
    chosen = "learned" if use_learned and form_lines["learned"]["agreement_vs_plain"] >= 0.999 else "plain"
    if chosen == "learned":
        ms, tm, clk = ms_l, tm_l, clk_l
        fn_chosen = run_learned
    else:
        ms, tm, clk = ms_plain, tm_plain, clk_plain
        fn_chosen = run_plain
    value = world_size * qry.n_rows / (ms / 1000.0)

    t = tuning.get(chosen)
    if t:  # the chosen form's launch shapes for the e2e leg
        ann.set_tuning(0, t["ft_warps"])
        ann.set_tuning(1, t["ft_heavy"])
        ann.set_tuning(2, t["score_chunk_mb"])

    # e2e: host (pinned) inputs through the same call, upload inside the timed region
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h_data, h_idx, h_ptr = pin(qry.data), pin(qry.indices), pin(qry.indptr.astype(np.int32))
    csr_host = abi.SgrCsr(qry.n_rows, qry.n_cols, h_data.data_ptr(), h_idx.data_ptr(), h_ptr.data_ptr(), 0)
    e2e_steps = max(1, min(args.steps, 3))
    fn_chosen(csr_host)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(e2e_steps):
        fn_chosen(csr_host)
    ev1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1) / e2e_steps)
    h2d = qry.data.nbytes + qry.indices.nbytes + 4 * (qry.n_rows + 1)
    d2h = 2 * 4 * qry.n_rows

    # FP16-operand correlation variant beside the exact INT8 form: score step only, same batch
    fp16 = None
    if mode == abi.MODE_EXACT and world_size == 1:
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
    roof_corr = {"kernel": "score-step correlation", "bound": "tensor",
                 "achieved": corr_ops_launch / (corr_launch_ms / 1000) / 1e12, "peak": int8_peak,
                 "unit": "TFLOP/s", "traffic": TRAFFIC_PER_QUERY["corr"] * rows_corr,
                 "peak_note": f"int8 dense = 2 x {src} bf16 cuBLAS ({bf16} TFLOP/s)"}
    roof_corr["frac"] = roof_corr["achieved"] / roof_corr["peak"]
    roof_rank = {"kernel": "gather + rank", "bound": "hbm",
                 "achieved": rank_bytes_launch / (rank_launch_ms / 1000) / 1e9, "peak": hbm, "unit": "GB/s",
                 "traffic": TRAFFIC_PER_QUERY["rank"] * rows_rank, "peak_note": f"{src} copy bandwidth"}
    roof_rank["frac"] = roof_rank["achieved"] / roof_rank["peak"]
    sel_launch_ms = tm["select_ms"] / max(1, tm["select_launches"])
    sel_bytes_launch = tm["select_bytes"] / max(1, tm["select_launches"])
    roof_sel = {"kernel": "per-label quantile select", "bound": "hbm",
                "achieved": sel_bytes_launch / (sel_launch_ms / 1000) / 1e9, "peak": hbm, "unit": "GB/s",
                "traffic": TRAFFIC_PER_QUERY["select"] * rows_sel, "peak_note": f"{src} copy bandwidth"}
    roof_sel["frac"] = roof_sel["achieved"] / roof_sel["peak"]
    # the dominant kernel with a roofline of its own: fine-tune is reported in stages_ms (it is bound by
    # issue and L1 gathers over L2-resident data, not by HBM or the tensor pipe)
    cands = [(stages["corr_ms"], roof_corr), (stages["rank_ms"], roof_rank), (stages["select_ms"], roof_sel)]
    dominant = max(cands, key=lambda c: c[0])[1]

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        v, cores, per = cpu_reference(args, wl, ref, qry, 1, 0, args.cpu_sample)
        cpu = {"value": v, "unit": "cells/s", "cores": cores, "kind": "port",
               "sample": f"{args.cpu_sample} query cells of the same batch, full reference, {per:.1f} s"}

    if rank == 0:
        line = {
            "metric": "query cells/s annotated (first + final label)", "value": value, "unit": "cells/s",
            "n_gpus": world_size, "steps": steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int8" if mode == abi.MODE_EXACT else "f32", "data": "synthetic",
            "config": {"workload": f"{args.workload}: {ref.n_rows} ref x {qry.n_rows} query x {ref.n_cols} genes, "
                                   f"{L} labels, {qry.nnz / (qry.n_rows * qry.n_cols):.3f} density",
                       "form": f"{chosen} ({args.mode})", "l2": "inputs larger than L2 (query CSR "
                                                             f"{h2d / 1e9:.2f} GB)",
                       "parallelism": f"query sharding x{world_size}"},
            "e2e": {"value": world_size * qry.n_rows / (e2e_ms / 1000.0), "unit": "cells/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(tm["launches"] / steps * steps),
            "roofline": dominant, "rooflines": [roof_corr, roof_rank, roof_sel],
            "stages_ms": stages, "ref_prep_s": ref_prep_s, "forms": form_lines, "mlp": mlp_info,
            "tuning": tuning, "fp16_variant": fp16,
            "ft_rounds_per_cell": tm["ft_cell_rounds"] / max(1, tm["cells"]),
            "clocks": clk, "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ann.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
