"""RELAX on the device (relax.hpp:1625-2185): GTR fit, MG94 with separate test / reference omegas, the RELAX
null (k = 1) and alternative fits, LRT.  Held to the reference's acceptance against HyPhy 2.5.101 on Fig4E
(tests/test_relax.cpp:17-100; fixture fig4e_relax): branch sets, GTR log-likelihood, the MG94 omegas, the
alternative's gain over MG94, the null's range, k, the LRT and its p-value.
"""
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fig4e(golden_dir):
    import _hyphy3 as h3
    aln = h3.Alignment.load(str(golden_dir / "Fig4E.nex"))
    s = h3.RELAXSettings()
    s.p_value_threshold = 0.05
    relax = h3.RELAXAnalyzer.create(h3.Tree.from_newick(aln.embedded_tree_newick), aln, s)
    return relax, relax.run()


def test_relax_branch_sets(fig4e, known):
    relax, _ = fig4e
    k = known["fig4e_relax"]
    assert len(relax.test_branch_names) == k["num_test"]
    assert len(relax.ref_branch_names) == k["num_reference"]


def test_relax_fig4e_matches_hyphy(fig4e, known):
    _, res = fig4e
    k = known["fig4e_relax"]
    alt, null = res.alternative_fit, res.null_fit
    info = (res.gtr_log_likelihood, res.mg94_log_likelihood, res.mg94_omega_R, res.mg94_omega_T, alt.log_likelihood,
            null.log_likelihood, res.k, res.lrt, res.p_value, list(alt.reference_distribution.omegas),
            list(alt.reference_distribution.weights))
    assert abs(res.gtr_log_likelihood - k["gtr_log_l"]) < k["tol_gtr"], info
    assert res.mg94_omega_R < k["max_omega_R"] and res.mg94_omega_T > k["min_omega_T"], info
    assert alt.log_likelihood >= null.log_likelihood, info
    assert alt.log_likelihood >= res.mg94_log_likelihood - 0.5, info
    assert abs((alt.log_likelihood - res.mg94_log_likelihood) - k["alt_minus_mg94"]) < k["tol_alt_minus_mg94"], info
    assert alt.log_likelihood > k["min_alt"], info
    assert k["min_null"] < null.log_likelihood < k["max_null"], info
    assert res.k < k["max_k"], info
    assert res.is_relaxed and res.is_significant and not res.is_intensified, info
    assert abs(res.lrt - k["lrt"]) < k["tol_lrt"], info
    assert res.p_value < k["max_p"], info


def test_relax_fit_structure(fig4e):
    import numpy as np
    _, res = fig4e
    for fit in (res.alternative_fit, res.null_fit):
        w = fit.reference_distribution.weights
        assert sum(w) == pytest.approx(1.0, abs=1e-12) and list(fit.test_distribution.weights) == list(w)
        om_r, om_t = fit.reference_distribution.omegas, fit.test_distribution.omegas
        assert 0.0 <= om_r[0] <= 1.0 and 0.0 <= om_r[1] <= 1.0 and om_r[2] >= 1.0
        np.testing.assert_allclose([min(max(o ** fit.k, 1e-6), 1e4) if o > 1e-12 else 0.0 for o in om_r], om_t, rtol=1e-12)
    assert res.null_fit.k == 1.0
    assert res.lrt == pytest.approx(2 * (res.alternative_fit.log_likelihood - res.null_fit.log_likelihood), abs=1e-9)
