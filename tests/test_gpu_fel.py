"""FEL per-site fits on the device against the oracle's restatement of the reference (fel.hpp:326-572).

Both run the reference's search (grid, bounded Nelder-Mead, Brent) pattern by
pattern; the device evaluates every likelihood in FP64 by spectral pruning
with its own eigensolver, so the searches follow the same path and the fitted
values agree to the optimisers' tolerance.  The CD2 run is also held to the
reference's own acceptance against HyPhy 2.5 (tests/test_fel_cd2_parity.cpp).
"""
import json

import numpy as np
import pytest

from gpu_helpers import problem_from_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from hyphy3 import _capi
    c = _capi.Context(0)
    yield c
    c.close()


def _fel_inputs(oracle, aln, params):
    base = dict(params)
    qs = oracle.mg94(aln, {**base, "alpha": 1.0, "beta": 0.0})["Q"]
    qn = oracle.mg94(aln, {**base, "alpha": 0.0, "beta": 1.0})["Q"]
    np.fill_diagonal(qs, 0.0)
    np.fill_diagonal(qn, 0.0)
    return np.asarray(aln.pi), qs, qn


def _compare(dev, ref):
    lrt_d, lrt_r = dev["lrt"], np.asarray(ref["lrt"])
    # log-likelihoods of the fitted models agree to the optimisers' tolerance (1e-4 on the objective)
    np.testing.assert_allclose(dev["log_l_alt"], ref["log_l_alt"], rtol=0, atol=1e-4)
    np.testing.assert_allclose(dev["log_l_null"], ref["log_l_null"], rtol=0, atol=1e-4)
    np.testing.assert_allclose(lrt_d, lrt_r, rtol=0, atol=2e-4)
    np.testing.assert_allclose(dev["p_value"], ref["p_value"], rtol=0, atol=2e-4)
    # on flat objectives (a rate pinned at its bound) rounding-level likelihood differences can
    # change a comparison inside the simplex search, so only most searches take identical steps
    same_path = np.array(ref["evals"]) == dev["evaluations"]
    assert same_path.mean() > 0.75


def test_fel_cd2_matches_oracle_and_hyphy25(ctx, oracle, golden_dir):
    k = json.loads((golden_dir / "known_answers.json").read_text())["cd2_fel"]
    a = oracle.Alignment.load(str(golden_dir / "cd2.fna"))
    t = oracle.Tree.parse((golden_dir / "cd2_fitted.nwk").read_text())
    ref = oracle.fel_run(t, a, k["params"])
    pi, qs, qn = _fel_inputs(oracle, a, k["params"])
    pr = problem_from_oracle(ctx, oracle, t, a)
    dev = pr.fel_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=ref["branch_lengths"])
    _compare(dev, ref)
    sp = np.array(a.site_pattern)
    mle = np.array(k["mle"])
    assert np.corrcoef(dev["lrt"][sp], mle[:, 3])[0, 1] > k["min_pearson_lrt"]
    assert np.corrcoef(dev["p_value"][sp], mle[:, 4])[0, 1] > k["min_pearson_p"]
    inv = np.asarray(ref["evals"]) == 0
    assert np.all(dev["evaluations"][inv] == 0) and np.all(dev["p_value"][inv] == 1.0)


def test_fel_synthetic_with_gaps_and_ambiguity(ctx, oracle):
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=60, n_taxa=24)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    t = oracle.Tree.parse(wl.newick)
    params = {"alpha": 1.0, "beta": 0.4, "theta": wl.theta}
    ref = oracle.fel_run(t, a, params)
    pi, qs, qn = _fel_inputs(oracle, a, params)
    pr = problem_from_oracle(ctx, oracle, t, a)
    dev = pr.fel_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=ref["branch_lengths"])
    _compare(dev, ref)


def test_fel_rejects_bad_arguments(ctx, oracle, golden_dir):
    from hyphy3 import _capi
    a = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = oracle.Tree.parse((golden_dir / "cd2_reduced.nwk").read_text())
    pr = problem_from_oracle(ctx, oracle, t, a)
    pi, qs, qn = _fel_inputs(oracle, a, {"alpha": 1.0, "beta": 0.5, "theta": [1, 1, 1, 2, 1]})
    bl = np.array(t.branch_lengths)
    bad = bl.copy()
    bad[1] = np.nan
    with pytest.raises(_capi.H3GError):
        pr.fel_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=bad)
    with pytest.raises(_capi.H3GError):
        pr.fel_run(pi=pi, Qs=-qs, Qn=qn, branch_lengths=bl)
    out = pr.fel_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=bl)
    assert np.all(out["lrt"] >= 0) and np.all((out["p_value"] >= 0) & (out["p_value"] <= 1))


def test_fel_analyzer_api_matches_reference_test(oracle, golden_dir):
    """hyphy3.FELAnalyzer(tree, aln, params).run(): the reference's CD2 parity case, site by site."""
    import _hyphy3 as h3
    k = json.loads((golden_dir / "known_answers.json").read_text())["cd2_fel"]
    a = h3.Alignment.load(str(golden_dir / "cd2.fna"))
    t = h3.Tree.from_newick_file(str(golden_dir / "cd2_fitted.nwk"))
    p = h3.MG94Parameters()
    p.alpha, p.beta = k["params"]["alpha"], k["params"]["beta"]
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = k["params"]["theta"]
    res = h3.FELAnalyzer(t, a, p).run()
    assert len(res) == 187
    lrt = np.array([r.lrt for r in res])
    pv = np.array([r.p_value for r in res])
    mle = np.array(k["mle"])
    assert np.corrcoef(lrt, mle[:, 3])[0, 1] > k["min_pearson_lrt"]
    assert np.corrcoef(pv, mle[:, 4])[0, 1] > k["min_pearson_p"]
    oa = oracle.Alignment.load(str(golden_dir / "cd2.fna"))
    ot = oracle.Tree.parse((golden_dir / "cd2_fitted.nwk").read_text())
    ref = oracle.fel_run(ot, oa, k["params"])
    sp = np.array(oa.site_pattern)
    np.testing.assert_allclose(lrt, np.asarray(ref["lrt"])[sp], rtol=0, atol=2e-4)
    np.testing.assert_allclose([r.total_branch_length for r in res], np.asarray(ref["total_branch_length"])[sp],
                               rtol=1e-3, atol=1e-6)


def _leaves(t):
    return [bool(x) for x in t.is_leaf]


def test_fel_subset_cd2_matches_oracle(ctx, oracle, golden_dir):
    """Leaves tested, internal branches background (fel.hpp:462-572) on CD2, device vs oracle."""
    k = json.loads((golden_dir / "known_answers.json").read_text())["cd2_fel"]
    a = oracle.Alignment.load(str(golden_dir / "cd2.fna"))
    t = oracle.Tree.parse((golden_dir / "cd2_fitted.nwk").read_text())
    tested = _leaves(t)
    ref = oracle.fel_run_tested(t, a, k["params"], tested)
    pi, qs, qn = _fel_inputs(oracle, a, k["params"])
    pr = problem_from_oracle(ctx, oracle, t, a)
    dev = pr.fel_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=ref["branch_lengths"], tested=tested)
    _compare(dev, ref)
    var = np.asarray(ref["evals"]) > 0
    assert np.all(dev["beta_nuisance"][~var] == 0.0)
    assert np.all((dev["beta_nuisance"][var] >= 1e-4) & (dev["beta_nuisance"][var] <= 1000.0))
    # the split is a different model from the all-branches one
    full = pr.fel_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=ref["branch_lengths"])
    assert np.abs(full["log_l_alt"] - dev["log_l_alt"]).max() > 1e-3


def test_fel_tested_all_is_the_all_branches_run(ctx, oracle, golden_dir):
    a = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = oracle.Tree.parse((golden_dir / "cd2_reduced.nwk").read_text())
    params = {"alpha": 1.0, "beta": 0.5, "theta": [1, 1, 1, 2, 1]}
    pi, qs, qn = _fel_inputs(oracle, a, params)
    pr = problem_from_oracle(ctx, oracle, t, a)
    bl = np.array(t.branch_lengths)
    one = pr.fel_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=bl)
    two = pr.fel_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=bl, tested=[True] * t.num_nodes())
    for key in ("alpha", "beta", "log_l_alt", "log_l_null", "lrt", "evaluations"):
        np.testing.assert_array_equal(one[key], two[key])


def test_fel_analyzer_leaves_reference_case(oracle, golden_dir, known):
    """The reference's "Leaves" case (tests/test_fel.cpp:78-126) through hyphy3.FELAnalyzer."""
    import _hyphy3 as h3
    k = known["cd2_reduced_fel_leaves"]
    a = h3.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = h3.Tree.from_newick(k["newick"])
    p = h3.MG94Parameters()
    p.alpha, p.beta = k["params"]["alpha"], k["params"]["beta"]
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = k["params"]["theta"]
    s = h3.FELSettings()
    s.test_branches = k["test_branches"]
    f = h3.FELAnalyzer(t, a, p, s)
    assert (f.num_tested, f.num_background) == (k["num_tested"], k["num_background"])
    assert len(f.test_branch_names) == f.num_tested and len(f.bg_branch_names) == f.num_background
    res = f.run()
    assert len(res) == a.num_codons
    for i in k["invariant_sites"]:
        assert res[i].alpha == 0.0 and res[i].beta == 0.0 and res[i].p_value == 1.0
    oa = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    ot = oracle.Tree.parse(k["newick"])
    ref = oracle.fel_run_tested(ot, oa, k["params"], _leaves(ot))
    sp = np.array(oa.site_pattern)
    np.testing.assert_allclose([r.lrt for r in res], np.asarray(ref["lrt"])[sp], rtol=0, atol=2e-4)
    np.testing.assert_allclose([r.log_l_alt for r in res], np.asarray(ref["log_l_alt"])[sp], rtol=0, atol=1e-4)
    np.testing.assert_allclose([r.total_branch_length for r in res], np.asarray(ref["total_branch_length"])[sp],
                               rtol=1e-3, atol=1e-6)
