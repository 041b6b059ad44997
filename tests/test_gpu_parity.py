"""GPU parity through the C ABI against the oracle.

Bars: ranks and gene indices bit-exact; fp32ref mode scores bit-exact with the oracle's restatement
of the reference's FP32 order (so labels are identical); exact mode scores bit-exact with the
oracle's exact formula, within 1e-5 absolute of the FP32 reference order, and labels identical
except at documented near-ties.
"""

import numpy as np
import pytest

from cusingler_b200 import abi
from tests import helpers as H

pytestmark = pytest.mark.gpu

KINDS = ["tiny", "families", "small"]


def annotator(kind, mode, base128=0):
    prob = H.problem(kind)
    a = abi.Annotator(gpuid=0, cores=8, mode=mode)
    a.set_tuning(11, base128)  # the limbs' split: two-accumulator (default) or base 128
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    return a, prob


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("base128", [0, 1])
def test_ranks_bit_exact(kind, base128):
    """Ranks reconstructed from the int8 limbs equal the oracle's, for either split of the limbs."""
    a, prob = annotator(kind, abi.MODE_EXACT, base128)
    res = H.oracle_run(kind, 1)
    orc = res["oracle"]
    d_ref = a.debug_ranks()
    d_qry = a.debug_ranks(prob.qry)
    for r in range(0, prob.ref.n_rows, max(1, prob.ref.n_rows // 200)):
        assert np.array_equal(d_ref[r], orc.rank_row(0, r)), r
    for q in range(prob.qry.n_rows):
        assert np.array_equal(d_qry[q], orc.rank_row(1, q)), q


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("base128", [0, 1])
def test_scores_fp32ref_bit_exact(kind, base128):
    a, prob = annotator(kind, abi.MODE_FP32REF, base128)
    raw = a.debug_scores(prob.qry)
    ref = H.oracle_run(kind, 0)["raw"]
    assert H.ulp_diff(raw, ref).max() == 0


@pytest.mark.parametrize("kind", KINDS)
def test_scores_exact(kind):
    a, prob = annotator(kind, abi.MODE_EXACT)
    raw = a.debug_scores(prob.qry)
    exact = H.oracle_run(kind, 1)["raw"]
    fp32 = H.oracle_run(kind, 0)["raw"]
    assert H.ulp_diff(raw, exact).max() == 0
    assert np.nanmax(np.abs(raw - fp32)) < 1e-5


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("mode", [abi.MODE_FP32REF, abi.MODE_EXACT])
def test_first_labels_and_flags(kind, mode):
    a, prob = annotator(kind, mode)
    first, scores, flags = a.score_first(prob.qry)
    res = H.oracle_run(kind, 0 if mode == abi.MODE_FP32REF else 1)
    assert H.ulp_diff(scores, res["scores"]).max() == 0
    assert np.array_equal(first, res["first"])
    assert np.array_equal(flags, res["flags"].astype(np.uint8))


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("mode", [abi.MODE_FP32REF, abi.MODE_EXACT])
def test_final_labels(kind, mode):
    a, prob = annotator(kind, mode)
    res = H.oracle_run(kind, 0 if mode == abi.MODE_FP32REF else 1)
    final, rounds = a.finetune(prob.qry, res["flags"].astype(np.uint8))
    assert np.array_equal(final, res["final"])
    assert np.array_equal(rounds, res["rounds"])


@pytest.mark.parametrize("times", [1, 2])
def test_finetune_times(times):
    a, prob = annotator("tiny", abi.MODE_FP32REF)
    res = H.oracle_run("tiny", 0, times)
    final, rounds = a.finetune(prob.qry, res["flags"].astype(np.uint8), times=times)
    assert np.array_equal(final, res["final"])
    assert rounds.max() <= times


def test_annotate_matches_steps():
    a, prob = annotator("small", abi.MODE_EXACT)
    first, final, scores = a.annotate(prob.qry, with_scores=True)
    res = H.oracle_run("small", 1)
    assert np.array_equal(first, res["first"]) and np.array_equal(final, res["final"])
    fp = H.oracle_run("small", 0)
    # exact vs the reference's FP32 order: scores within 1e-5, labels equal unless at a near-tie
    assert np.nanmax(np.abs(scores - fp["scores"])) < H.NEAR_TIE
    assert len(H.unexplained_flips(first, fp["first"], fp["margin_first"])) == 0
    assert len(H.unexplained_flips(final, fp["final"], fp["margin_final"])) == 0


@pytest.mark.parametrize("kind", ["tiny", "families", "small"])
@pytest.mark.parametrize("packed", [0, 1, 2])
def test_final_labels_both_row_scans(kind, packed):
    """The fine-tune row scan on two registers, on packed (count, e-sum) words, and on packed words
    with 32-bit run sums and masked run ends gives the oracle's final labels and round counts."""
    a, prob = annotator(kind, abi.MODE_EXACT)
    a.set_tuning(3, packed)
    res = H.oracle_run(kind, 1)
    final, rounds = a.finetune(prob.qry, res["flags"].astype(np.uint8))
    assert np.array_equal(final, res["final"])
    assert np.array_equal(rounds, res["rounds"])


@pytest.mark.parametrize("kind", ["tiny", "families", "small"])
@pytest.mark.parametrize("heavy", [2, 1 << 30])
@pytest.mark.parametrize("times", [0, 2])
def test_final_labels_spread_and_queue_paths(kind, heavy, times):
    """Every cell on the spread path (rounds spread over the GPU, two launches per round) or every
    cell on the work-queue kernel: the oracle's final labels and round counts either way."""
    a, prob = annotator(kind, abi.MODE_EXACT)
    a.set_tuning(1, heavy)
    res = H.oracle_run(kind, 1, times)
    final, rounds = a.finetune(prob.qry, res["flags"].astype(np.uint8), times=times)
    a.set_tuning(1, 6)
    assert np.array_equal(final, res["final"])
    assert np.array_equal(rounds, res["rounds"])


@pytest.mark.parametrize("kind", ["tiny", "small"])
@pytest.mark.parametrize("wide", [18, 0])
def test_fp16_variant_close_to_exact(kind, wide):
    """The FP16-operand correlation variant (FP32 accumulation, not exact), on 128 x 256 tiles with
    two alternating accumulators or on 128 x 160 tiles: every score within 1e-4 of the exact score
    (a bound of K x 2^-24 relative to the Cauchy-Schwarz bound of the sum), NaN where the exact score
    is NaN, and first labels that differ only at near-ties."""
    a, prob = annotator(kind, abi.MODE_EXACT)
    raw_exact = a.debug_scores(prob.qry)
    f_exact, s_exact, _ = a.score_first(prob.qry)
    a.set_tuning(10, wide)
    a.set_tuning(4, 1)
    raw_f16 = a.debug_scores(prob.qry)
    f16, s16, _ = a.score_first(prob.qry)
    a.set_tuning(4, 0)
    assert np.array_equal(np.isnan(raw_exact), np.isnan(raw_f16))
    assert np.nanmax(np.abs(raw_f16.astype(np.float64) - raw_exact)) < 1e-4
    assert np.nanmax(np.abs(s16.astype(np.float64) - s_exact)) < 1e-4
    assert (f16 == f_exact).mean() >= 0.99
    # back on the exact form, bit-exact again
    assert H.ulp_diff(a.debug_scores(prob.qry), raw_exact).max() == 0


@pytest.mark.parametrize("kind", ["tiny", "small"])
@pytest.mark.parametrize("base128,pair,wide,gm", [(0, 0, 18, 1), (0, 0, 18, 8), (0, 0, 16, 1), (0, 0, 16, 8),
                                                  (0, 0, 8, 1), (0, 0, 0, 1), (0, 1, 0, 8), (1, 0, 0, 8),
                                                  (1, 1, 0, 1), (1, 0, 18, 1)])
def test_correlation_forms_bit_exact(kind, base128, pair, wide, gm):
    """Every tensor-core form of the exact correlation gives the oracle's exact scores bit for bit, and
    the oracle's labels (query and reference counts that are not multiples of the tile sizes
    included): 128 x 256 tiles with two accumulators (8 or 16 epilogue warps, or 16 overlapping the
    next tile's products), 128 x 160 tiles with three, and their SM-pair form (tcgen05 cta_group::2),
    on either split of the limbs (the base-128 split has no two-accumulator form and takes the
    128 x 160 tiles), in band-by-band or grouped tile order."""
    a, prob = annotator(kind, abi.MODE_EXACT, base128)
    a.set_tuning(5, pair)
    a.set_tuning(10, wide)
    a.set_tuning(6, gm)
    raw = a.debug_scores(prob.qry)
    res = H.oracle_run(kind, 1)
    assert H.ulp_diff(raw, res["raw"]).max() == 0
    first, final = a.annotate(prob.qry)
    assert np.array_equal(first, res["first"]) and np.array_equal(final, res["final"])


@pytest.mark.parametrize("kind", ["tiny", "families", "small"])
@pytest.mark.parametrize("form", [0, 1, 8])
def test_selection_forms(kind, form):
    """The score-step selection as one warp per query row (form 0) and as 8-warp row-staging CTAs
    gives the oracle's label scores (ulp-equal), first labels and flags."""
    a, prob = annotator(kind, abi.MODE_EXACT)
    a.set_tuning(7, form)
    first, scores, flags = a.score_first(prob.qry)
    res = H.oracle_run(kind, 1)
    assert H.ulp_diff(scores, res["scores"]).max() == 0
    assert np.array_equal(first, res["first"])
    assert np.array_equal(flags, res["flags"].astype(np.uint8))
