"""FEL per-site fits on the device against the oracle's restatement of the reference (fel.hpp:326-446).

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
    with pytest.raises(RuntimeError):
        s = h3.FELSettings()
        s.test_branches = "Internal"
        h3.FELAnalyzer(t, a, p, s)
