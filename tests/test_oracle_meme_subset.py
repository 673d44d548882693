"""MEME with a tested / background branch split (meme.hpp:84-92, :219-632), oracle on the CPU.

The reference has no MEME fixture with a background, so the oracle is pinned by
composition:
* its likelihood with a background reduces to pinned ones: with p1 = 1 and
  beta_bg = alpha omega1 every branch has one model, the all-tested FEL likelihood
  at (alpha, alpha omega1) (FEL is pinned to HyPhy 2.5 on CD2); with an empty
  background it is the all-branches MEME likelihood (pinned to HyPhy 2.5 on CD2
  and ADH), and the background rate enters only through the background branches;
* the searches reuse the pinned N-dimensional Nelder-Mead, and with every
  branch tested the generalised search gives the all-branches run exactly.
"""
import json

import numpy as np
import pytest


@pytest.fixture(scope="module")
def leaves(oracle, golden_dir):
    k = json.loads((golden_dir / "known_answers.json").read_text())["cd2_reduced_fel_leaves"]
    a = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = oracle.Tree.parse(k["newick"])
    tested = [bool(x) for x in t.is_leaf]
    bl = list(oracle.fel_run(t, a, k["params"], 0)["branch_lengths"])
    return k, a, t, tested, bl


def test_meme_lnl_reduces_to_fel_and_all_branches(oracle, leaves):
    k, a, t, tested, bl = leaves
    p = k["params"]
    for al, w1 in ((0.8, 0.3), (2.5, 0.9)):
        tot = sum(w * oracle.meme_lnl_at(t, a, p, bl, q, al, w1, 1.0, 7.0, tested, al * w1)
                  for q, w in enumerate(a.weights))
        ref = oracle.mg94_loglik(t, a, dict(p, alpha=1.0, beta=w1), al, bl)
        assert tot == pytest.approx(ref, rel=1e-11, abs=1e-9)
    for q in range(min(a.num_patterns, 4)):
        everyone = oracle.meme_lnl_at(t, a, p, bl, q, 1.3, 0.2, 0.6, 4.0)
        same = oracle.meme_lnl_at(t, a, p, bl, q, 1.3, 0.2, 0.6, 4.0, [True] * t.num_nodes(), 9.0)
        assert same == everyone
        bg = oracle.meme_lnl_at(t, a, p, bl, q, 1.3, 0.2, 0.6, 4.0, tested, 9.0)
        assert bg != everyone


def test_meme_tested_all_is_the_all_branches_run(oracle, leaves):
    k, a, t, _, _ = leaves
    every = [True] * t.num_nodes()
    r1 = oracle.meme_run(t, a, k["params"])
    r2 = oracle.meme_run_tested(t, a, k["params"], every)
    for key in ("alpha", "beta1", "p1", "beta_plus", "lrt", "p_value", "log_l_meme", "log_l_fel", "total_branch_length"):
        np.testing.assert_array_equal(np.asarray(r1[key]), np.asarray(r2[key]), err_msg=key)
    assert np.all(np.asarray(r2["beta_bg"]) == 0.0)


def test_meme_subset_oracle_leaves_run(oracle, leaves):
    k, a, t, tested, _ = leaves
    r = oracle.meme_run_tested(t, a, k["params"], tested)
    var = np.asarray(r["evals"]) > 0
    assert var.any()
    sp = np.array(a.site_pattern)
    for s in k["invariant_sites"]:
        assert r["p_value"][sp[s]] == 1.0 and r["lrt"][sp[s]] == 0.0
    assert np.all(np.asarray(r["lrt"]) >= 0.0)
    bg = np.asarray(r["beta_bg"])[var]
    assert np.all((bg >= 1e-4) & (bg <= 1e5))
    ebf = np.asarray(r["branch_ebf"])
    background = [i for i in range(t.num_nodes()) if i != t.root and not tested[i]]
    assert np.all(ebf[:, background] == 1.0)
    np.testing.assert_array_equal((ebf >= 100).sum(axis=1), r["branches_under_selection"])
    # the alternative nests the FEL baseline's model (p1 = 1, beta_bg free as in FEL's subset fit)
    lm, lf = np.asarray(r["log_l_meme"])[var], np.asarray(r["log_l_fel"])[var]
    assert np.mean(lm >= lf - 1e-3) > 0.9
