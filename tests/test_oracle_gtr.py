"""Nucleotide GTR likelihood (likelihood.hpp:181-254, rate_matrix.hpp:14-104, alignment.hpp:832-890), CPU.

The oracle's GTR log-likelihood is pinned to HyPhy 2.5: at the nucleotide GTR fit recorded in the
reference's FEL ground truth for CD2 and ADH (rates, equilibrium frequencies, branch lengths) it
reproduces HyPhy's log-likelihood (the reference compares its own GTR fit with the same number at a
relative 1e-4, tests/test_fel_multi_dataset.cpp:195-196).  The host restatements used by the device
path (GTRMatrix, Alignment::to_nucleotide_alignment) match the oracle exactly or to rounding.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("key", ["cd2_gtr", "adh_gtr"])
def test_oracle_matches_hyphy25_gtr_fit(oracle, golden_dir, known, key):
    k = known[key]
    a = oracle.Alignment.load(str(golden_dir / k["alignment"]))
    t = oracle.Tree.parse(k["newick"])
    nuc = oracle.nucleotide_patterns(a)
    lnl, site = oracle.gtr_loglik(t, nuc, k["theta"], k["freqs"])
    assert lnl == pytest.approx(k["log_l"], rel=1e-6)
    assert sum(nuc.weights) == 3 * a.num_codons
    assert len(site) == nuc.num_patterns


def test_gtr_matrix_properties(oracle):
    theta, freq = [0.5, 0.3, 0.7, 1.9, 0.4], [0.4, 0.1, 0.2, 0.3]
    g = oracle.gtr_matrix(theta, freq, 0.25)
    Q, P = np.array(g["Q"]), np.array(g["P"])
    pi = np.array(freq)
    np.testing.assert_allclose(Q.sum(1), 0.0, atol=1e-14)
    assert -(pi * np.diag(Q)).sum() == pytest.approx(1.0, rel=1e-14)         # mean rate 1
    np.testing.assert_allclose(pi[:, None] * Q, (pi[:, None] * Q).T, atol=1e-15)   # reversible
    np.testing.assert_allclose(P.sum(1), 1.0, atol=1e-13)
    assert np.all(P >= 0) and max(g["lam"]) <= 0.0


def test_host_gtr_matrix_matches_oracle(oracle):
    import _hyphy3 as h3
    theta, freq = [0.5, 0.3, 0.7, 1.9, 0.4], [0.4, 0.1, 0.2, 0.3]
    p = h3.GTRParameters()
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = theta
    g = h3.GTRMatrix()
    g.update(p, freq)
    for t in (1e-6, 0.05, 0.7, 3.0):
        np.testing.assert_allclose(g.transition_matrix(t), np.array(oracle.gtr_matrix(theta, freq, t)["P"]), rtol=0, atol=1e-14)
    assert g.scale_factor == pytest.approx(oracle.gtr_matrix(theta, freq)["scale"], rel=1e-15)


@pytest.mark.parametrize("fname", ["cd2.fna", "adh.nex", "Fig4E.nex"])
def test_host_nucleotide_patterns_match_oracle(oracle, golden_dir, fname):
    import _hyphy3 as h3
    nuc = h3.Alignment.load(str(golden_dir / fname)).to_nucleotide_alignment()
    ref = oracle.nucleotide_patterns(oracle.Alignment.load(str(golden_dir / fname)))
    st, mk, w = nuc.pattern_arrays()
    np.testing.assert_array_equal(st, ref.states)
    np.testing.assert_array_equal(mk, ref.masks)
    np.testing.assert_array_equal(w, ref.weights)
    np.testing.assert_array_equal(nuc.site_to_pattern, ref.site_pattern)
    assert nuc.num_codons == 0 and nuc.num_nucleotides == len(nuc.site_to_pattern)
    np.testing.assert_array_equal(nuc.nuc_frequencies, ref.nuc_freq)
