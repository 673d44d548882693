"""BUSTED from an alignment and a tree (busted.hpp:220-258, :1644-2607, :5969-6682) on the device.

GTR fit, full MG94 fit, then the unconstrained and constrained BUSTED fits (3 omega classes, free branch
lengths, with and without 3 synonymous-rate classes), held to the reference's acceptance against HyPhy 2.5 on
CD2 (tests/test_busted.cpp:17-101: GTR within 1, MG94 within 0.05, both BUSTED fits within 2.5, LRT within
1.5, p < 0.01) and its structural checks on ADH (:104-134).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cd2_busted(golden_dir):
    import _hyphy3 as h3
    aln = h3.Alignment.load(str(golden_dir / "cd2.fna"))
    tree = h3.Tree.from_newick_file(str(golden_dir / "cd2.nwk"))
    return h3.BUSTEDAnalyzer.create_and_fit(tree, aln)


def _check_fit_structure(res, n_sites):
    u, c = res.unconstrained.test_distribution, res.constrained.test_distribution
    assert res.lrt >= 0.0 and 0.0 <= res.p_value <= 1.0
    assert u.omegas[-1] >= 1.0 and c.omegas[-1] == 1.0
    assert all(0.0 <= w <= 1.0 for w in u.omegas[:-1] + c.omegas[:-1])
    assert sum(u.weights) == pytest.approx(1.0, abs=1e-12) and sum(c.weights) == pytest.approx(1.0, abs=1e-12)
    assert len(res.evidence_ratios) == n_sites == len(res.constrained_evidence_ratios)
    assert res.unconstrained.log_likelihood >= res.constrained.log_likelihood
    assert res.lrt == pytest.approx(2 * (res.unconstrained.log_likelihood - res.constrained.log_likelihood), abs=1e-9)


def test_busted_cd2_baseline_fits(cd2_busted, known):
    k = known["cd2_busted"]
    assert cd2_busted.has_gtr_fit
    assert abs(cd2_busted.gtr_log_l - k["gtr_log_l"]) < k["tol_gtr"]
    assert abs(cd2_busted.mg94_log_l - k["mg94_log_l"]) < k["tol_mg94"], cd2_busted.mg94_log_l


def test_busted_cd2_without_srv(cd2_busted):
    res = cd2_busted.run()
    _check_fit_structure(res, 187)
    # evidence ratios are site likelihood ratios of the two fits
    u, c = res.unconstrained, res.constrained
    import _hyphy3 as h3  # noqa: F401
    assert res.evidence_ratios[0] == pytest.approx(np.exp(u.site_log_likelihoods[0] - c.site_log_likelihoods[0]), rel=1e-12)


def test_busted_cd2_srv_matches_hyphy25(cd2_busted, known):
    import _hyphy3 as h3
    k = known["cd2_busted"]
    s = h3.BUSTEDSettings()
    s.srv = True
    s.num_rate_classes = 3
    s.num_syn_rate_classes = 3
    s.refine_branch_lengths = True
    res = cd2_busted.run(s)
    _check_fit_structure(res, 187)
    u, c = res.unconstrained, res.constrained
    info = (u.log_likelihood, c.log_likelihood, res.lrt, list(u.test_distribution.omegas), list(u.test_distribution.weights),
            list(c.test_distribution.omegas), list(c.test_distribution.weights))
    assert abs(u.log_likelihood - k["unconstrained_log_l"]) < k["tol_fit"], info
    assert abs(c.log_likelihood - k["constrained_log_l"]) < k["tol_fit"], info
    assert abs(res.lrt - k["lrt"]) < k["tol_lrt"], info
    assert res.p_value < k["max_p"]
    d = u.test_distribution
    assert len(d.syn_rates) == 3 and sum(d.syn_weights) == pytest.approx(1.0, abs=1e-12)
    assert np.dot(d.syn_rates, d.syn_weights) == pytest.approx(1.0, abs=1e-9)      # unit mean
    assert list(d.syn_rates) == sorted(d.syn_rates)


def test_busted_adh_structure(golden_dir):
    import _hyphy3 as h3
    aln = h3.Alignment.load(str(golden_dir / "adh.nex"))
    b = h3.BUSTEDAnalyzer.create_and_fit(h3.Tree.from_newick(aln.embedded_tree_newick), aln)
    res = b.run()
    _check_fit_structure(res, 254)
    assert len(res.unconstrained.branch_lengths) == b.tree.num_nodes()


def test_busted_auto_k_adh(golden_dir):
    """tests/test_busted.cpp:137-164: on ADH the AICc step-up over the null fits picks K = 2 and still detects
    positive selection."""
    import _hyphy3 as h3
    aln = h3.Alignment.load(str(golden_dir / "adh.nex"))
    b = h3.BUSTEDAnalyzer.create_and_fit(h3.Tree.from_newick(aln.embedded_tree_newick), aln)
    s = h3.BUSTEDSettings()
    s.auto_select_k = True
    s.max_k = 3
    s.refine_branch_lengths = True
    res = b.run(s)
    aicc = [f.aicc for f in res.k_null_fits]
    assert res.optimal_k == 2, aicc
    assert len(res.unconstrained.test_distribution.omegas) == 2 and len(res.constrained.test_distribution.omegas) == 2
    assert res.unconstrained.test_distribution.omegas[1] >= 1.0 and res.constrained.test_distribution.omegas[1] == 1.0
    assert res.lrt >= 0.0 and res.p_value <= 0.05, (res.lrt, res.p_value)


def test_busted_rejects_unsupported_modes(cd2_busted):
    import _hyphy3 as h3
    s = h3.BUSTEDSettings()
    s.error_sink = True
    with pytest.raises(Exception):
        cd2_busted.run(s)
    s = h3.BUSTEDSettings()
    s.relax_mode = True
    with pytest.raises(Exception):
        cd2_busted.run(s)


def test_busted_two_set_cd2(cd2_busted, golden_dir):
    """A test set that leaves background branches (busted.hpp:6413-6460): both fits carry a free 3-class
    background distribution; only the test set's last omega is held at 1 under the null."""
    import _hyphy3 as h3
    s = h3.BUSTEDSettings()
    s.test_branches = "Human,Chimp,Baboon,RhMonkey,Node3,Node2"
    res = cd2_busted.run(s)
    assert cd2_busted.num_background_branches > 0
    _check_fit_structure(res, 187)
    for fit in (res.unconstrained, res.constrained):
        b = fit.background_distribution
        assert fit.has_background_distribution and len(b.omegas) == 3
        assert all(0.0 <= o <= 1.0 for o in b.omegas[:2]) and b.omegas[2] >= 1.0
        assert sum(b.weights) == pytest.approx(1.0, abs=1e-12)
        w = np.asarray(h3.Alignment.load(str(golden_dir / "cd2.fna")).pattern_arrays()[2], dtype=float)
        assert float(np.dot(w, fit.site_log_likelihoods)) == pytest.approx(fit.log_likelihood, rel=1e-12)
    # busted.hpp:3146: the two-set likelihood at the fitted parameters reproduces the fit (lnL and per pattern)
    u = res.unconstrained
    cd2_busted.select_test_branches("Human,Chimp,Baboon,RhMonkey,Node3,Node2")
    lnl, pll = cd2_busted.evaluate_two_set_log_l(
        1.0, list(u.test_distribution.omegas), list(u.test_distribution.weights), list(u.background_distribution.omegas),
        list(u.background_distribution.weights), custom_branch_lengths=list(u.branch_lengths), custom_base_params=u.gtr_params)
    assert lnl == pytest.approx(u.log_likelihood, rel=1e-12)
    np.testing.assert_allclose(pll, u.site_log_likelihoods, rtol=1e-12, atol=1e-12)
    # the two-set alternative is at least as good as the one-set alternative restricted to the test branches'
    # classes on every branch (the background distribution can take the test distribution's values)
    one = cd2_busted.run()
    assert res.unconstrained.log_likelihood >= one.unconstrained.log_likelihood - 0.5
