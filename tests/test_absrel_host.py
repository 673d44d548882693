"""aBSREL's host-side pieces (CPU only): the MG94 structure it builds generators from, and its
statistics (AICc, the mixture p-value, Holm-Bonferroni) against the reference's formulas."""
import math

import numpy as np


def test_structure_reproduces_the_library_generator(golden_dir):
    import _hyphy3 as h
    from hyphy3.absrel import MG94Structure
    a = h.Alignment.load(str(golden_dir / "adh.nex"))
    st = MG94Structure(np.asarray(a.pos_nuc_frequencies))
    for beta, theta in ((0.4, [1, 1, 1, 1, 1]), (2.3, [0.7, 1.3, 0.4, 2.2, 0.9])):
        p = h.MG94Parameters()
        p.beta = beta
        p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = theta
        ref = np.asarray(h.mg94_eigensystem(a, p)["Q"])
        assert np.max(np.abs(st.Q(theta, beta) - ref)) < 1e-15
        eps = 1e-6
        num = (st.Q(theta, beta + eps) - st.Q(theta, beta - eps)) / (2 * eps)
        assert np.max(np.abs(st.dQ_domega(theta) - num)) < 1e-8
        th2 = list(theta)
        th2[3] += eps
        th1 = list(theta)
        th1[3] -= eps
        num = (st.Q(th2, beta) - st.Q(th1, beta)) / (2 * eps)
        assert np.max(np.abs(st.dQ_dtheta(3, beta) - num)) < 1e-8


def test_statistics_match_the_reference_formulas():
    from hyphy3.absrel import aicc, holm_bonferroni, mixture_p_value
    for lrt in (0.5, 3.0, 12.0):
        assert abs(mixture_p_value(lrt) - (0.2 * math.erfc(math.sqrt(lrt / 2)) + 0.3 * math.exp(-lrt / 2))) < 1e-15
    assert mixture_p_value(0.0) == 1.0 and mixture_p_value(-1.0) == 1.0
    assert abs(aicc(-100.0, 5, 200) - (200.0 + 2 * 5 * 200 / (200 - 5 - 1))) < 1e-12
    assert aicc(-100.0, 5, 6) == 210.0
    adj = holm_bonferroni([0.01, 0.04, 0.03, 0.5])
    assert np.allclose(adj, [0.04, 0.09, 0.09, 0.5])
