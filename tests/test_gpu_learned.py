"""The learned proposal: its CUDA forward/backward against the numpy oracle, training, and the
learned annotate form against the plain form."""

import numpy as np
import pytest

from cusingler_b200 import abi
from oracle import mlp_oracle as M
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _trained(kind="families"):
    prob = H.problem(kind)
    a = abi.Annotator(gpuid=0, mode=abi.MODE_EXACT)
    a.train(prob.ref, prob.celltypes, prob.label_names, prob.ref_genes, prob.qry_genes)
    return a, prob


def test_gradients_match_oracle():
    a, prob = _trained("tiny")
    L = len(prob.label_names)
    rng = np.random.default_rng(0)
    scores = rng.uniform(0.0, 0.9, (300, L)).astype(np.float32)
    targets = rng.integers(0, L, 300).astype(np.int32)
    a.mlp_train(scores, targets, epochs=2, batch=128, seed=1)      # non-trivial weights
    X = np.maximum((scores - scores.max(1, keepdims=True)) * 20, -8).astype(np.float32)
    g, loss = a.mlp_debug_grads(X[:200], targets[:200])
    params, Lp, Hd = a.mlp_params()
    ref_loss, ref_g = M.loss_and_grads(params, Lp, Hd, X[:200], targets[:200])
    assert abs(loss - ref_loss) < 1e-4 * max(1.0, abs(ref_loss))
    rel = np.linalg.norm(g - ref_g) / np.linalg.norm(ref_g)
    assert rel < 1e-4, rel
    assert np.max(np.abs(g - ref_g)) < 1e-4 * np.max(np.abs(ref_g)) + 1e-7


def test_inference_matches_oracle():
    """mlp_predict (tensor-core inference, BF16 hi/lo split of the FP32 activations) against the
    oracle's float64 forward: confidences within 1e-4, labels equal wherever the top two logits are
    not within 1e-3 of each other."""
    a, prob = _trained("tiny")
    L = len(prob.label_names)
    rng = np.random.default_rng(4)
    scores = rng.uniform(0.0, 0.9, (3000, L)).astype(np.float32)
    targets = rng.integers(0, L, 3000).astype(np.int32)
    a.mlp_train(scores, targets, epochs=3, batch=256, seed=2)
    lab, conf = a.mlp_predict(scores)
    params, Lp, Hd = a.mlp_params()
    X = np.maximum((scores - scores.max(1, keepdims=True)) * 20, -8).astype(np.float32)
    logits = M.forward(params, Lp, Hd, X)
    z = logits - logits.max(1, keepdims=True)
    ref_conf = 1.0 / np.exp(z).sum(1)
    assert np.max(np.abs(conf - ref_conf)) < 1e-4
    top2 = np.sort(logits, 1)[:, -2:]
    clear = (top2[:, 1] - top2[:, 0]) > 1e-3
    assert np.array_equal(lab[clear], logits.argmax(1)[clear])


def test_training_learns_and_confident_proposals_agree():
    a, prob = _trained("tiny")
    first, scores, flags = a.score_first(prob.qry)
    final, _ = a.finetune(prob.qry, flags)
    loss0 = a.mlp_train(scores, final, epochs=1, batch=64, seed=3)
    loss1 = a.mlp_train(scores, final, epochs=300, batch=64, seed=3)
    assert loss1 < loss0
    lab, conf = a.mlp_predict(scores)
    assert (lab == final).mean() > 0.9
    f3, fin3, st3 = a.annotate_learned(prob.qry, min_confidence=0.98, check_fraction=0.0)
    assert np.array_equal(f3, first)
    assert st3["checked"] == 0 and st3["decided"] + st3["finetuned"] == st3["cells"]
    assert (fin3 == final).mean() >= 0.99


def test_learned_form_fallback_is_the_plain_result():
    a, prob = _trained("families")
    first, scores, flags = a.score_first(prob.qry)
    final, _ = a.finetune(prob.qry, flags)
    a.mlp_train(scores, final, epochs=100, batch=64, seed=3)
    # every confident proposal re-run plain: all labels are the plain labels, agreement is counted
    f2, fin2, st = a.annotate_learned(prob.qry, min_confidence=0.98, check_fraction=1.0)
    assert np.array_equal(f2, first)
    assert st["cells"] == prob.qry.n_rows and st["decided"] + st["finetuned"] == st["cells"]
    assert np.array_equal(fin2, final)
    assert st["check_agree"] <= st["checked"]
    # an impossible threshold sends every multi-candidate cell to the plain loop
    f4, fin4, st4 = a.annotate_learned(prob.qry, min_confidence=2.0, check_fraction=0.0)
    assert np.array_equal(fin4, final)
    multi = (flags.sum(1) > 1).sum()
    assert st4["finetuned"] == multi
