"""Edge cases on the GPU: empty query, constant rows (NaN scores), one-cell labels, unsorted CSR
columns, gene-name intersection, malformed inputs, and the drop-in module."""

import numpy as np
import pytest

from cusingler_b200 import abi, synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _csr_from_rows(rows, n_cols):
    data, idx, ptr = [], [], [0]
    for r in rows:
        for c, v in r:
            idx.append(c)
            data.append(v)
        ptr.append(len(idx))
    return synth.CSR(len(rows), n_cols, np.array(data, np.float32), np.array(idx, np.int32),
                     np.array(ptr, np.int32), np.zeros(len(rows), np.int32))


def _run_both(prob, mode, tuning=()):
    a = abi.Annotator(gpuid=0, mode=mode)
    for what, value in tuning:
        a.set_tuning(what, value)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    first, scores, flags = a.score_first(prob.qry)
    final, rounds = a.finetune(prob.qry, flags)
    orc = O.Oracle(prob)
    orc.train()
    of, os_, ofl, _ = orc.score(mode=0 if mode == abi.MODE_FP32REF else 1)
    ofin, orounds = orc.finetune(mode=0 if mode == abi.MODE_FP32REF else 1)
    assert H.ulp_diff(scores, os_).max() == 0
    assert np.array_equal(first, of)
    assert np.array_equal(flags, ofl.astype(np.uint8))
    assert np.array_equal(final, ofin)
    assert np.array_equal(rounds, orounds)
    return first, final


@pytest.mark.parametrize("mode", [abi.MODE_FP32REF, abi.MODE_EXACT])
def test_constant_and_empty_rows(mode):
    """Constant query rows give all-NaN scores (first label = last label, no flags, final 0);
    constant reference rows make NaN-bearing score lists sorted in libstdc++'s order."""
    ref, qry, L = H.dataset("tiny")
    rows_q = [list(zip(qry.indices[qry.indptr[i]:qry.indptr[i + 1]], qry.data[qry.indptr[i]:qry.indptr[i + 1]]))
              for i in range(40)]
    rows_q[3] = []                       # all implicit zeros
    rows_q[5] = [(c, 1.0) for c in range(qry.n_cols)]  # every gene equal
    rows_r = [list(zip(ref.indices[ref.indptr[i]:ref.indptr[i + 1]], ref.data[ref.indptr[i]:ref.indptr[i + 1]]))
              for i in range(ref.n_rows)]
    for i in (0, 1, 50, 51, 52):
        rows_r[i] = []
    q = _csr_from_rows(rows_q, qry.n_cols)
    r = _csr_from_rows(rows_r, ref.n_cols)
    prob = O.Problem(r, q, synth.names("CT", L), ref.labels, synth.names("G", ref.n_cols),
                     synth.names("G", qry.n_cols))
    first, final = _run_both(prob, mode)
    assert first[3] == L - 1 and final[3] == 0


@pytest.mark.parametrize("mode", [abi.MODE_FP32REF, abi.MODE_EXACT])
def test_single_cell_labels_and_unsorted_columns(mode):
    ref, qry, L = H.dataset("tiny")
    codes = ref.labels.copy()
    codes[0] = L          # two extra labels with one reference cell each
    codes[1] = L + 1
    rng = np.random.default_rng(0)
    qd, qi = qry.data.copy(), qry.indices.copy()
    for i in range(qry.n_rows):   # shuffle column order within each query row
        a, b = qry.indptr[i], qry.indptr[i + 1]
        p = rng.permutation(b - a)
        qd[a:b], qi[a:b] = qd[a:b][p], qi[a:b][p]
    q = synth.CSR(qry.n_rows, qry.n_cols, qd, qi, qry.indptr, qry.labels)
    prob = O.Problem(ref, q, synth.names("CT", L + 2), codes, synth.names("G", ref.n_cols),
                     synth.names("G", qry.n_cols))
    _run_both(prob, mode)


@pytest.mark.parametrize("mode", [abi.MODE_FP32REF, abi.MODE_EXACT])
def test_dense_rows_take_the_large_sort_tier(mode):
    """Rows with more marker entries than the rank kernel's small sort buffer (512) are ranked by
    its second, large-buffer launch: dense rows with distinct, tied and negative values, in the
    query and in the reference, ranked bit-exactly and annotated like the oracle (13 labels,
    over a thousand marker genes)."""
    ref, qry, L = H.dataset("small")
    rng = np.random.default_rng(7)

    def rows_of(m, n):
        return [list(zip(m.indices[m.indptr[i]:m.indptr[i + 1]], m.data[m.indptr[i]:m.indptr[i + 1]]))
                for i in range(n)]

    def dense(n_cols, kind):
        if kind == 0:    # distinct values
            v = rng.permutation(n_cols).astype(np.float32) + 0.5
        elif kind == 1:  # few distinct values: long tie runs
            v = rng.integers(1, 6, n_cols).astype(np.float32)
        else:            # mixed signs with some stored zeros
            v = np.round(rng.normal(0, 2, n_cols), 1).astype(np.float32)
        return list(zip(range(n_cols), v))

    rows_q = rows_of(qry, 64)
    for i, kind in ((2, 0), (9, 1), (17, 2), (30, 0)):
        rows_q[i] = dense(qry.n_cols, kind)
    rows_r = rows_of(ref, ref.n_rows)
    for i, kind in ((4, 0), (120, 1), (333, 2)):
        rows_r[i] = dense(ref.n_cols, kind)
    q = _csr_from_rows(rows_q, qry.n_cols)
    r = _csr_from_rows(rows_r, ref.n_cols)
    prob = O.Problem(r, q, synth.names("CT", L), ref.labels, synth.names("G", ref.n_cols),
                     synth.names("G", qry.n_cols))
    _run_both(prob, mode)
    a = abi.Annotator(gpuid=0, mode=mode)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    assert len(a.u32(0)) > 512
    orc = O.Oracle(prob)
    orc.train()
    d_qry = a.debug_ranks(prob.qry)
    d_ref = a.debug_ranks()
    for i in range(q.n_rows):
        assert np.array_equal(d_qry[i], orc.rank_row(1, i)), i
    for i in (3, 4, 5, 119, 120, 333):
        assert np.array_equal(d_ref[i], orc.rank_row(0, i)), i


@pytest.mark.parametrize("select_form", [0, 1, 16])
def test_long_labels_ties_and_nan_lists(select_form):
    """Long score lists in exact mode.  Five labels, four of them over 1,024 reference cells: one long
    label holds an empty reference row (its lists hold NaN and are sorted exactly), one holds 1,000
    copies of a single cell (the order statistic's value bin exceeds the 256-key buffer, so the radix
    selection decides), two take the bucket selection with extremes from the correlation; one query
    row is empty (a NaN row).  Scores, first labels, flags and final labels equal the oracle's."""
    w, ref, qry = synth.custom_dataset(6000, 128, 3000, 5, 0.08, seed=36)
    counts = np.bincount(ref.labels, minlength=5)
    assert (counts >= 1024).sum() == 4

    def rows_of(m):
        return [list(zip(m.indices[m.indptr[i]:m.indptr[i + 1]], m.data[m.indptr[i]:m.indptr[i + 1]]))
                for i in range(m.n_rows)]

    rows_r = rows_of(ref)
    by_label = [np.flatnonzero(ref.labels == l) for l in range(5)]
    copies = by_label[0][:1000]
    for i in copies[1:]:
        rows_r[i] = list(rows_r[copies[0]])
    rows_r[by_label[1][7]] = []
    rows_q = rows_of(qry)
    rows_q[5] = []
    r = _csr_from_rows(rows_r, ref.n_cols)
    q = _csr_from_rows(rows_q, qry.n_cols)
    prob = O.Problem(r, q, synth.names("CT", 5), ref.labels, synth.names("G", ref.n_cols),
                     synth.names("G", qry.n_cols))
    _run_both(prob, abi.MODE_EXACT, tuning=[(7, select_form)])


@pytest.mark.parametrize("mode,select_form", [(abi.MODE_EXACT, 1), (abi.MODE_EXACT, 16), (abi.MODE_FP32REF, 1)])
def test_tied_order_statistics_in_small_bins(mode, select_form):
    """Score lists whose order statistic k-1 lies in a run of tied values that fits the bucket
    selection's 256-key buffer.  One label holds 150 copies of one reference cell among 180 (the
    statistic's bin holds 150 to 180 keys: the bitonic sort ranks them), another 20 copies among 25
    (20 to 25 keys: the warp-shuffle rank, with ties).  Scores, first labels, flags and final labels
    equal the oracle's."""
    w, ref, qry = synth.custom_dataset(900, 96, 2000, 3, 0.08, seed=41)

    def rows_of(m):
        return [list(zip(m.indices[m.indptr[i]:m.indptr[i + 1]], m.data[m.indptr[i]:m.indptr[i + 1]]))
                for i in range(m.n_rows)]

    rows_r = rows_of(ref)
    by_label = [np.flatnonzero(ref.labels == l) for l in range(3)]
    keep0, keep1 = by_label[0][:180], by_label[1][:25]
    for i in keep0[1:150]:
        rows_r[i] = list(rows_r[keep0[0]])
    for i in keep1[1:20]:
        rows_r[i] = list(rows_r[keep1[0]])
    order = np.concatenate([keep0, keep1, by_label[2]])
    labels = ref.labels[order]
    r = _csr_from_rows([rows_r[i] for i in order], ref.n_cols)
    prob = O.Problem(r, qry, synth.names("CT", 3), labels, synth.names("G", ref.n_cols),
                     synth.names("G", qry.n_cols))
    # the construction: in every scored row, statistic k-1 of label 0 is tied 150+ times, of label 1
    # 20+ times (p = 0.8: k - 1 = 143 of 180 and 19 of 25 lie inside the copies' run of ranks)
    orc = O.Oracle(prob)
    orc.train()
    raw = orc.score(mode=1, raw=True)[3]
    for q in range(raw.shape[0]):
        for lab, k1, ties in ((0, 143, 150), (1, 19, 20)):
            v = np.sort(raw[q, labels == lab])
            if not np.isnan(v).any():
                assert (v == v[k1]).sum() >= ties, (q, lab)
    _run_both(prob, mode, tuning=[(7, select_form)])


def test_many_query_rows_tiled_scan():
    """9,000 query rows: the thre-pool compaction's exclusive scan over the rows' counts runs as
    4,096-row tiles in parallel (three tiles); scores, labels, flags and fine-tune rounds equal
    the oracle's."""
    w, ref, qry = synth.custom_dataset(600, 9000, 3000, 7, 0.08, seed=13)
    prob = O.Problem(ref, qry, synth.names("CT", 7), ref.labels, synth.names("G", ref.n_cols),
                     synth.names("G", qry.n_cols))
    _run_both(prob, abi.MODE_EXACT)


@pytest.mark.parametrize("pinned", [False, True])
def test_host_rows_copied_in_chunks(pinned):
    """A host query's rows are copied to the device one block of queries at a time, overlapped with
    the scoring of the blocks before.  With 1 MiB score blocks the 9,000-row query takes about 21
    blocks; scores, labels, flags and rounds equal the oracle's, through both the score-then-
    fine-tune calls and the one-call annotation.  From pageable memory every copy has landed before
    the call returns from queuing it; from page-locked memory the copies really run behind the
    scoring, so the waits between the copy stream and the compute stream are exercised."""
    w, ref, qry = synth.custom_dataset(600, 9000, 3000, 7, 0.08, seed=13)
    keep = None
    if pinned:
        import torch
        pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory()  # noqa: E731
        keep = (pin(qry.data), pin(qry.indices), pin(qry.indptr.astype(np.int32)))
        qry = synth.CSR(qry.n_rows, qry.n_cols, keep[0].numpy(), keep[1].numpy(), keep[2].numpy(), qry.labels)
    prob = O.Problem(ref, qry, synth.names("CT", 7), ref.labels, synth.names("G", ref.n_cols),
                     synth.names("G", qry.n_cols))
    a = abi.Annotator(gpuid=0, mode=abi.MODE_EXACT)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    a.set_tuning(2, 1)
    first, scores, flags = a.score_first(prob.qry)
    final, rounds = a.finetune(prob.qry, flags)
    orc = O.Oracle(prob)
    orc.train()
    of, os_, ofl, _ = orc.score(mode=1)
    ofin, orounds = orc.finetune(mode=1)
    assert H.ulp_diff(scores, os_).max() == 0
    assert np.array_equal(first, of)
    assert np.array_equal(flags, ofl.astype(np.uint8))
    assert np.array_equal(final, ofin)
    assert np.array_equal(rounds, orounds)
    first2, final2 = a.annotate(prob.qry)
    assert np.array_equal(first2, of) and np.array_equal(final2, ofin)


def test_gene_intersection():
    ref, qry, L = H.dataset("tiny")
    rg = synth.names("G", ref.n_cols)
    qg = synth.names("G", qry.n_cols)
    for i in range(0, len(qg), 9):
        qg[i] = f"Q{i}"
    prob = O.Problem(ref, qry, synth.names("CT", L), ref.labels, rg, qg)
    _run_both(prob, abi.MODE_FP32REF)


def test_empty_query_and_errors():
    ref, qry, L = H.dataset("tiny")
    a = abi.Annotator(gpuid=0)
    a.train(ref, ref.labels, synth.names("CT", L), synth.names("G", ref.n_cols), synth.names("G", qry.n_cols))
    empty = synth.CSR(0, qry.n_cols, np.zeros(0, np.float32), np.zeros(0, np.int32), np.zeros(1, np.int32),
                      np.zeros(0, np.int32))
    first, scores, flags = a.score_first(empty)
    assert first.shape == (0,)
    bad = synth.CSR(2, qry.n_cols, np.ones(2, np.float32), np.array([1, qry.n_cols + 5], np.int32),
                    np.array([0, 1, 2], np.int32), np.zeros(2, np.int32))
    with pytest.raises(abi.SgrError) as e:
        a.score_first(bad)
    assert e.value.status == 1
    nanq = synth.CSR(1, qry.n_cols, np.array([np.nan], np.float32), np.array([int(a.u32(0)[0])], np.int32),
                     np.array([0, 1], np.int32), np.zeros(1, np.int32))
    with pytest.raises(abi.SgrError):
        a.score_first(nanq)
    # the context stays usable after an error
    first, _, _ = a.score_first(qry)
    assert first.shape == (qry.n_rows,)


def test_dropin_run_matches_oracle():
    from cusingler import cusingler
    prob = H.problem("tiny")
    ref, qry = prob.ref, prob.qry
    cells = [f"cell{i}" for i in range(qry.n_rows)]
    res = cusingler.run(8, 0, ref.n_rows, ref.n_cols, ref.data, ref.indices, ref.indptr,
                        qry.n_rows, qry.n_cols, qry.data, qry.indices, qry.indptr,
                        prob.label_names, prob.celltypes, cells, prob.ref_genes, prob.qry_genes,
                        quantile=80, finetune_thre=0.05, finetune_times=0)
    o = H.oracle_run("tiny", 1)
    assert [r[0] for r in res] == cells
    assert [r[1] for r in res] == [prob.label_names[i] for i in o["first"]]
    assert [r[2] for r in res] == [prob.label_names[i] for i in o["final"]]


def test_autotune_keeps_results():
    """The autotuner times every launch-shape candidate, leaves the fastest set, and the annotation
    afterwards still equals the oracle's."""
    prob = H.problem("families")
    a = abi.Annotator(gpuid=0)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    t = a.autotune(prob.qry)
    # score step: 5 correlation forms (this marker count allows the two-accumulator split) x 2 tile
    # orders x 2 block sizes x 3 selection forms
    assert t["trials"] == 20 and t["score_trials"] == 60 and t["pipeline"] in (0, 1)
    assert t["corr_wide"] in (0, 8, 16, 18)
    assert t["ft_warps"] in (8, 32) and t["ft_heavy"] in (4, 6, 9, 16, 1 << 30)
    assert t["score_chunk_mb"] in (256, 1024) and 0 < t["best_ms"] <= t["worst_ms"]
    assert t["corr_pair"] in (0, 1) and t["corr_gm"] in (1, 16) and t["select_warps"] in (0, 1, 16)
    first, final = a.annotate(prob.qry)
    o = H.oracle_run("families", 1)
    assert np.array_equal(first, o["first"]) and np.array_equal(final, o["final"])


@pytest.mark.parametrize("learned", [False, True])
def test_stream_of_batches_matches_one_call(learned):
    """sgr_annotate_stream over uneven page-locked batches (one of them empty) gives the labels of
    one sgr_annotate / sgr_annotate_learned call over the whole query, and per-batch latencies."""
    import torch

    prob = H.problem("families")
    a = abi.Annotator(gpuid=0)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    q = prob.qry
    if learned:
        f0, fin0, sc = a.annotate(q, with_scores=True)
        a.mlp_train(sc, fin0, epochs=5, batch=64, seed=1)
        want_first, want_final, _ = a.annotate_learned(q, min_confidence=0.9, check_fraction=0.2)
    else:
        want_first, want_final = a.annotate(q)
    cuts = [0, 37, 37, 120, q.n_rows]
    pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory()  # noqa: E731
    batches, keep = [], []
    for lo, hi in zip(cuts, cuts[1:]):
        part = q.rows(lo, hi)
        t = (pin(part.data), pin(part.indices), pin(part.indptr.astype(np.int32)))
        keep.append(t)
        batches.append(abi.SgrCsr(part.n_rows, part.n_cols, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), 0))
    for _ in range(2):  # the second call reuses the context's batch buffers
        first, final, ms, st = a.annotate_stream(batches, learned=learned, min_confidence=0.9, check_fraction=0.2)
        assert np.array_equal(first, want_first) and np.array_equal(final, want_final)
        assert ms.shape == (len(batches),) and (ms >= 0).all()
        if learned:
            assert st["cells"] == q.n_rows and st["decided"] + st["finetuned"] == q.n_rows


@pytest.mark.parametrize("host_input", [False, True])
def test_pipelined_blocks_match_oracle(host_input):
    """With 1 MiB score blocks (six blocks of the 800-cell query) each block's fine-tune runs on a
    second stream while the next block is scored; first and final labels equal the oracle's, for a
    device query and for a page-locked host query whose rows are copied block by block."""
    import torch

    prob = H.problem("small")
    a = abi.Annotator(gpuid=0)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    a.set_tuning(2, 1)
    a.set_tuning(9, 1)
    q = prob.qry
    keep = None
    if host_input:
        pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory()  # noqa: E731
        keep = (pin(q.data), pin(q.indices), pin(q.indptr.astype(np.int32)))
        csr = abi.SgrCsr(q.n_rows, q.n_cols, keep[0].data_ptr(), keep[1].data_ptr(), keep[2].data_ptr(), 0)
    else:
        dev = torch.device("cuda", 0)
        keep = (torch.from_numpy(q.data).to(dev), torch.from_numpy(q.indices).to(dev),
                torch.from_numpy(q.indptr.astype(np.int32)).to(dev))
        csr = abi.device_csr(q.n_rows, q.n_cols, keep[0].data_ptr(), keep[1].data_ptr(), keep[2].data_ptr())
    res = H.oracle_run("small", 1)
    for _ in range(2):
        first, final = a.annotate(csr)
        assert np.array_equal(first, res["first"]) and np.array_equal(final, res["final"])


def test_pipelined_learned_matches_unpipelined():
    """The learned form with each block's routed cells fine-tuned on the second stream gives the same
    labels and routing counts as the one-pass learned form."""
    prob = H.problem("small")
    a = abi.Annotator(gpuid=0)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    f0, fin0, sc = a.annotate(prob.qry, with_scores=True)
    a.mlp_train(sc, fin0, epochs=5, batch=256, seed=1)
    a.set_tuning(2, 1)
    want = a.annotate_learned(prob.qry, min_confidence=0.9, check_fraction=0.2)
    a.set_tuning(9, 1)
    for _ in range(2):
        got = a.annotate_learned(prob.qry, min_confidence=0.9, check_fraction=0.2)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
        assert got[2] == want[2]
