"""MEME per-site fits on the device against the oracle's restatement of the reference (meme.hpp:84-632).

Both run the reference's searches (FEL baseline, 4-D and 3-D bounded
Nelder-Mead from the same start grids) pattern by pattern.  The device
evaluates every likelihood by spectral pruning with its own eigensolver, so
the two agree to rounding on every evaluation; MEME's mixture likelihood is
multi-modal, so where a rounding-level difference changes one comparison in a
simplex search the two may settle in different optima.  The runs are held to
the reference's own acceptance against HyPhy 2.5 (tests/test_meme.cpp) and to
close agreement with the oracle on most patterns.
"""
import json

import numpy as np
import pytest

from gpu_helpers import problem_from_oracle
from gpu_helpers import ranks as _ranks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from hyphy3 import _capi
    c = _capi.Context(0)
    yield c
    c.close()


def _inputs(oracle, aln, params):
    base = dict(params)
    qs = oracle.mg94(aln, {**base, "alpha": 1.0, "beta": 0.0})["Q"]
    qn = oracle.mg94(aln, {**base, "alpha": 0.0, "beta": 1.0})["Q"]
    np.fill_diagonal(qs, 0.0)
    np.fill_diagonal(qn, 0.0)
    return np.asarray(aln.pi), qs, qn


def _hyphy_acceptance(k, lrt, pv):
    mle = np.array(k["mle"])
    assert np.corrcoef(lrt, mle[:, 5])[0, 1] >= k["min_pearson_lrt"]
    assert np.corrcoef(_ranks(lrt), _ranks(mle[:, 5]))[0, 1] >= k["min_spearman_lrt"]
    assert np.corrcoef(pv, mle[:, 6])[0, 1] >= k["min_pearson_p"]
    assert np.corrcoef(_ranks(pv), _ranks(mle[:, 6]))[0, 1] >= k["min_spearman_p"]


def _same_log_ebf(e_dev, e_ref):
    """log EBF = log L+ - log L1 at one branch.  The smaller of the two class likelihoods carries an
    absolute error of up to ~1e-11 of the larger one's in any FP64 evaluation, the reference's
    included (at a large omega the spectral transition matrices reach their small entries by
    cancelling terms of order one), so the tolerance grows as 1e-11 e^|log EBF|; beyond
    |log EBF| = 20 both sides must only lie beyond the same bound."""
    ld, lr = np.log(np.maximum(e_dev, 1e-300)), np.log(np.maximum(e_ref, 1e-300))
    big = np.abs(lr) > 20.0
    tol = 1e-5 + 1e-11 * np.exp(np.abs(lr[~big]))
    assert np.all(np.abs(ld[~big] - lr[~big]) <= tol), (ld[~big] - lr[~big], tol)
    assert np.all(np.sign(ld[big]) == np.sign(lr[big])) and np.all(np.abs(ld[big]) > 20.0)


def _case(oracle, golden_dir, name, fasta):
    k = json.loads((golden_dir / "known_answers.json").read_text())[name]
    a = oracle.Alignment.load(str(golden_dir / fasta))
    t = oracle.Tree.parse(k["newick"])
    return k, a, t


@pytest.fixture(scope="module")
def cd2(ctx, oracle, golden_dir):
    k, a, t = _case(oracle, golden_dir, "cd2_meme", "cd2.fna")
    ref = oracle.meme_run(t, a, k["params"])
    pi, qs, qn = _inputs(oracle, a, k["params"])
    pr = problem_from_oracle(ctx, oracle, t, a)
    dev = pr.meme_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=ref["branch_lengths"])
    return k, a, t, ref, dev


def test_meme_cd2_matches_oracle(cd2):
    _, _, _, ref, dev = cd2
    inv = np.asarray(ref["evals"]) == 0
    assert np.array_equal(dev["evaluations"] == 0, inv)
    assert np.all(dev["p_value"][inv] == 1.0) and np.all(dev["lrt"][inv] == 0.0)
    # the FEL baseline: same searches, same optima
    np.testing.assert_allclose(dev["log_l_fel"], ref["log_l_fel"], rtol=0, atol=1e-4)
    # MEME: the same optimum on most patterns, never a worse one by more than the search tolerance on many
    d = np.abs(dev["log_l_meme"] - np.asarray(ref["log_l_meme"]))
    assert np.mean(d[~inv] <= 1e-3) > 0.9
    same = (~inv) & (d <= 1e-4)
    np.testing.assert_allclose(dev["lrt"][same], np.asarray(ref["lrt"])[same], rtol=0, atol=5e-3)
    assert np.corrcoef(dev["lrt"][~inv], np.asarray(ref["lrt"])[~inv])[0, 1] > 0.99
    np.testing.assert_allclose(dev["p1"] + dev["p_plus"], 1.0, atol=1e-15)
    assert np.all((dev["p_value"] >= 0) & (dev["p_value"] <= 1))


def test_meme_cd2_ebf_matches_oracle(oracle, cd2):
    """The device's branch EBFs (one inside-outside pass) against the oracle's two re-prunings per
    branch (meme.hpp:484-588) at the device's own MLE."""
    k, a, t, ref, dev = cd2
    e_d = dev["branch_ebf"]
    assert np.all(e_d[:, t.root] == 1.0) and np.all(e_d >= 0)
    np.testing.assert_array_equal((e_d >= 100).sum(axis=1), dev["branches_under_selection"])
    fitted = np.asarray(ref["evals"]) > 0
    # EBFs are computed for the patterns that reach the test (beta+ > alpha and p+ > 1e-6 at the
    # alternative fit); the others keep 1 on every branch
    computed = fitted & np.any(e_d != 1.0, axis=1)
    assert np.all(computed[fitted & (dev["beta_plus"] > dev["alpha"]) & (dev["p_plus"] > 1e-6)])
    tested = np.flatnonzero(computed)
    assert len(tested) >= 10
    bl = ref["branch_lengths"]
    for i in tested:
        al = dev["alpha"][i]
        e_r = np.asarray(oracle.meme_ebf_at(t, a, k["params"], bl, int(i), al, dev["beta1"][i] / al, dev["p1"][i],
                                            dev["beta_plus"][i]))
        _same_log_ebf(e_d[i], e_r)
    assert np.mean(dev["branches_under_selection"] == np.asarray(ref["branches_under_selection"])) > 0.9


def test_meme_cd2_meets_reference_acceptance(cd2):
    k, a, _, _, dev = cd2
    sp = np.array(a.site_pattern)
    _hyphy_acceptance(k, dev["lrt"][sp], dev["p_value"][sp])


def test_meme_adh_meets_reference_acceptance(ctx, oracle, golden_dir):
    """tests/test_meme.cpp:106-144 (ADH, 23 taxa, 254 codons) against HyPhy 2.5, device only."""
    k, a, t = _case(oracle, golden_dir, "adh_meme", "adh.nex")
    fel = oracle.fel_run(t, a, k["params"], 0)          # conversion and FEL-time lengths only
    pi, qs, qn = _inputs(oracle, a, k["params"])
    pr = problem_from_oracle(ctx, oracle, t, a)
    dev = pr.meme_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=fel["branch_lengths"], with_ebf=False)
    sp = np.array(a.site_pattern)
    assert len(sp) == 254
    _hyphy_acceptance(k, dev["lrt"][sp], dev["p_value"][sp])


def test_meme_rejects_bad_arguments(ctx, oracle, golden_dir):
    from hyphy3 import _capi
    a = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = oracle.Tree.parse((golden_dir / "cd2_reduced.nwk").read_text())
    pr = problem_from_oracle(ctx, oracle, t, a)
    pi, qs, qn = _inputs(oracle, a, {"alpha": 1.0, "beta": 0.5, "theta": [1, 1, 1, 2, 1]})
    bl = np.array(t.branch_lengths)
    bad = bl.copy()
    bad[1] = -1.0
    with pytest.raises(_capi.H3GError):
        pr.meme_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=bad)
    badpi = pi.copy()
    badpi[0] = np.inf
    with pytest.raises(_capi.H3GError):
        pr.meme_run(pi=badpi, Qs=qs, Qn=qn, branch_lengths=bl)
    out = pr.meme_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=bl)
    assert np.all(out["lrt"] >= 0) and np.all((out["p_value"] >= 0) & (out["p_value"] <= 1))


def test_meme_analyzer_api(oracle, golden_dir):
    """hyphy3.MEMEAnalyzer(tree, aln, params).run() on the reference's CD2 case, site by site."""
    import _hyphy3 as h3
    k = json.loads((golden_dir / "known_answers.json").read_text())["cd2_meme"]
    a = h3.Alignment.load(str(golden_dir / "cd2.fna"))
    t = h3.Tree.from_newick(k["newick"])
    p = h3.MG94Parameters()
    p.alpha, p.beta = k["params"]["alpha"], k["params"]["beta"]
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = k["params"]["theta"]
    res = h3.MEMEAnalyzer(t, a, p).run()
    assert len(res) == 187
    lrt = np.array([r.lrt for r in res])
    pv = np.array([r.p_value for r in res])
    _hyphy_acceptance(k, lrt, pv)
    assert all(len(r.branch_ebf) == t.num_nodes() for r in res)
    m = h3.MEMEAnalyzer(t, a, p, "Internal")
    internal = [nd.id for nd in t.nodes if nd.id != t.root_id and not nd.is_leaf]
    assert m.num_tested == len(internal) and m.num_background == t.num_nodes() - 1 - len(internal)
    res = m.run()
    leaves = [nd.id for nd in t.nodes if nd.is_leaf]
    assert all(all(r.branch_ebf[i] == 1.0 for i in leaves) for r in res)
    assert any(r.beta_bg > 0.0 for r in res)


@pytest.fixture(scope="module")
def cd2_leaves(ctx, oracle, golden_dir):
    """CD2 with the leaves tested and the internal branches as background."""
    k, a, t = _case(oracle, golden_dir, "cd2_meme", "cd2.fna")
    tested = [bool(x) for x in t.is_leaf]
    ref = oracle.meme_run_tested(t, a, k["params"], tested)
    pi, qs, qn = _inputs(oracle, a, k["params"])
    pr = problem_from_oracle(ctx, oracle, t, a)
    dev = pr.meme_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=ref["branch_lengths"], tested=tested)
    return k, a, t, tested, ref, dev


def test_meme_subset_cd2_matches_oracle(cd2_leaves):
    _, _, t, tested, ref, dev = cd2_leaves
    inv = np.asarray(ref["evals"]) == 0
    assert np.array_equal(dev["evaluations"] == 0, inv)
    # the FEL baseline runs the branch-subset search: same searches, same optima
    np.testing.assert_allclose(dev["log_l_fel"], ref["log_l_fel"], rtol=0, atol=1e-4)
    d = np.abs(dev["log_l_meme"] - np.asarray(ref["log_l_meme"]))
    assert np.mean(d[~inv] <= 1e-3) > 0.9
    same = (~inv) & (d <= 1e-4)
    np.testing.assert_allclose(dev["lrt"][same], np.asarray(ref["lrt"])[same], rtol=0, atol=5e-3)
    assert np.corrcoef(dev["lrt"][~inv], np.asarray(ref["lrt"])[~inv])[0, 1] > 0.99
    assert np.all((dev["beta_bg"][~inv] >= 1e-4) & (dev["beta_bg"][~inv] <= 1e5))
    np.testing.assert_allclose(dev["total_branch_length"][same], np.asarray(ref["total_branch_length"])[same], rtol=1e-3)
    background = [i for i in range(t.num_nodes()) if i != t.root and not tested[i]]
    assert np.all(dev["branch_ebf"][:, background] == 1.0)


def test_meme_subset_cd2_ebf_matches_oracle(oracle, cd2_leaves):
    """Device EBFs with a background (k_meme_ebf<3>) against the oracle's re-prunings at the device's MLE."""
    k, a, t, tested, ref, dev = cd2_leaves
    e_d = dev["branch_ebf"]
    np.testing.assert_array_equal((e_d >= 100).sum(axis=1), dev["branches_under_selection"])
    fitted = np.asarray(ref["evals"]) > 0
    reach = np.flatnonzero(fitted & (dev["beta_plus"] > dev["alpha"]) & (dev["p_plus"] > 1e-6))
    assert len(reach) >= 5
    bl = ref["branch_lengths"]
    for i in reach:
        al = dev["alpha"][i]
        bg = dev["beta_bg"][i] if dev["beta_bg"][i] > 0.0 else dev["beta1"][i]
        e_r = np.asarray(oracle.meme_ebf_at(t, a, k["params"], bl, int(i), al, dev["beta1"][i] / al, dev["p1"][i],
                                            dev["beta_plus"][i], tested, bg))
        _same_log_ebf(e_d[i], e_r)
