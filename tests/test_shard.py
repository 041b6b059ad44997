"""Query sharding across ranks on CPU: the row split, and two gloo ranks whose gathered labels equal
the unsharded run (the oracle stands in for the per-rank device call, so no GPU is needed)."""

import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from cusingler_b200 import shard, synth
from oracle import oracle as O
from tests import helpers as H


@pytest.mark.parametrize("world", [1, 2, 3, 7])
def test_row_ranges_cover_and_balance(world):
    rng = np.random.default_rng(world)
    for n in (0, 1, 5, 200):
        lens = rng.integers(0, 50, size=n)
        indptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        rr = shard.row_ranges(indptr, world)
        assert len(rr) == world
        assert rr[0][0] == 0 and rr[-1][1] == n
        for (a, b), (c, d) in zip(rr, rr[1:]):
            assert a <= b == c <= d
        if n and indptr[-1]:
            per = [int(indptr[b] - indptr[a]) for a, b in rr]
            assert max(per) - indptr[-1] / world <= lens.max() + 1


def test_shard_of_slices_rows():
    ref, qry, L = H.dataset("tiny")
    lo, hi, part = shard.shard_of(qry, 2, 1)
    assert part.n_rows == hi - lo and hi == qry.n_rows
    assert np.array_equal(part.data, qry.data[qry.indptr[lo]:qry.indptr[hi]])
    assert part.indptr[0] == 0 and part.indptr[-1] == qry.indptr[hi] - qry.indptr[lo]


def _oracle_annotate(ref, part, L):
    prob = O.Problem(ref, part, synth.names("CT", L), ref.labels, synth.names("G", ref.n_cols),
                     synth.names("G", part.n_cols))
    orc = O.Oracle(prob)
    orc.train()
    first, _, _, _ = orc.score(mode=O.MODE_EXACT)
    final, _ = orc.finetune(mode=O.MODE_EXACT)
    return first, final


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ref, qry, L = H.dataset("tiny")
        first, final = shard.annotate_sharded(lambda part: _oracle_annotate(ref, part, L), qry)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), first=first, final=final)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_match_unsharded():
    ref, qry, L = H.dataset("tiny")
    want_first, want_final = _oracle_annotate(ref, qry, L)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(2, _free_port(), d), nprocs=2, join=True, start_method="spawn")
        for r in range(2):
            got = np.load(os.path.join(d, f"rank{r}.npz"))
            assert np.array_equal(got["first"], want_first)
            assert np.array_equal(got["final"], want_final)


def _device_rank_main(rank, world, port, out_dir):
    """One rank of the device-sharded run: its own context on cuda:0 annotates its row block through
    libsgr.so, and the labels are gathered over gloo."""
    import torch.distributed as dist

    from cusingler_b200 import abi

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prob = H.problem("families")
        a = abi.Annotator(gpuid=0)
        a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
        first, final = shard.annotate_sharded(lambda part: a.annotate(part), prob.qry)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), first=first, final=final)
        a.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_ranks_drive_the_library_and_gather():
    """Two processes, each with its own context on cuda:0 (independent kernels, no rank waits on
    another's kernels), annotate their row blocks through the C ABI; the gathered labels equal the
    oracle's unsharded labels."""
    want = H.oracle_run("families", 1)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_device_rank_main, args=(2, _free_port(), d), nprocs=2, join=True,
                           start_method="spawn")
        for r in range(2):
            got = np.load(os.path.join(d, f"rank{r}.npz"))
            assert np.array_equal(got["first"], want["first"])
            assert np.array_equal(got["final"], want["final"])
