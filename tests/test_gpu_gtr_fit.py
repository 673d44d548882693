"""GTR gradients and GTRFitter on the device (optimizer.hpp:33-200).

The gradient in every branch length and exchangeability is checked against central finite
differences of the oracle's GTR likelihood (pinned to HyPhy 2.5) at HyPhy's CD2 fit; the fitter is
held to the reference's own acceptance for its GTR fit: the log-likelihood of HyPhy 2.5's nucleotide
GTR fit within a relative 1e-4 (tests/test_fel_multi_dataset.cpp:195-196), on CD2 and ADH.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_gtr_gradients_match_oracle_differences(oracle, golden_dir, known):
    import _hyphy3 as h3
    k = known["cd2_gtr"]
    aln = h3.Alignment.load(str(golden_dir / k["alignment"])).to_nucleotide_alignment()
    t = h3.Tree.from_newick(k["newick"])
    p = h3.GTRParameters()
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = k["theta"]
    bl = t.get_branch_lengths()
    lnl, g_t, g_th = h3.compute_gtr_gradients(t, aln, p, bl)
    oa = oracle.nucleotide_patterns(oracle.Alignment.load(str(golden_dir / k["alignment"])))
    ot = oracle.Tree.parse(k["newick"])
    freqs = list(aln.nuc_frequencies)
    ref = lambda th, b: oracle.gtr_loglik(ot, oa, th, freqs, b)[0]
    assert lnl == pytest.approx(ref(k["theta"], bl), rel=1e-10)
    for i in range(t.num_nodes()):
        if i == t.root_id:
            continue
        h = 1e-5 * max(bl[i], 1e-3)
        up, dn = list(bl), list(bl)
        up[i] += h
        dn[i] = max(dn[i] - h, 0.0)
        fd = (ref(k["theta"], up) - ref(k["theta"], dn)) / (up[i] - dn[i])
        assert g_t[i] == pytest.approx(fd, rel=1e-4, abs=1e-3), i
    for x in range(5):
        h = 1e-5 * k["theta"][x]
        up, dn = list(k["theta"]), list(k["theta"])
        up[x] += h
        dn[x] -= h
        fd = (ref(up, bl) - ref(dn, bl)) / (2 * h)
        assert g_th[x] == pytest.approx(fd, rel=1e-4, abs=1e-3), x


@pytest.mark.parametrize("key,start", [("cd2_gtr", "cd2_fitted.nwk"), ("adh_gtr", None)])
def test_gtr_fitter_reaches_hyphy25_fit(golden_dir, known, key, start):
    import _hyphy3 as h3
    k = known[key]
    aln = h3.Alignment.load(str(golden_dir / k["alignment"]))
    if start:
        tree = h3.Tree.from_newick_file(str(golden_dir / start))
    else:                                            # HyPhy's topology with every length reset
        tree = h3.Tree.from_newick(k["newick"])
        tree.set_branch_lengths([0.1] * tree.num_nodes())
    res = h3.GTRFitter(tree, aln).fit()
    assert res.log_likelihood == pytest.approx(k["log_l"], rel=1e-4)
    assert res.log_likelihood > k["log_l"] - 1e-2
    assert res.converged
    th = [res.params.theta_AC, res.params.theta_AT, res.params.theta_CG, res.params.theta_CT, res.params.theta_GT]
    np.testing.assert_allclose(th, k["theta"], rtol=0.05)
    # AICc with K = 5 + branches, N = nucleotide sites (stats.hpp:114-121)
    B = tree.num_nodes() - 1
    N = 3 * aln.num_codons
    K = 5 + B
    assert res.aicc == pytest.approx(-2 * res.log_likelihood + 2 * K * N / (N - K - 1), rel=1e-12)
