"""Nucleotide GTR log-likelihood on the device (h3g_nuc_eval_from_P; likelihood.hpp:181-254).

Against the oracle (pinned to HyPhy 2.5's GTR fits of CD2 and ADH) per pattern and in total, on the
reference datasets at HyPhy's fit, on a simulated 256-taxon alignment with gaps and ambiguity, and
on a 300-taxon caterpillar tree (the deepest stack of open partials).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host(h3, newick, theta, freqs):
    t = h3.Tree.from_newick(newick)
    p = h3.GTRParameters()
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = theta
    g = h3.GTRMatrix()
    g.update(p, list(freqs))
    return t, g


@pytest.mark.parametrize("key", ["cd2_gtr", "adh_gtr"])
def test_gtr_at_hyphy_fit(oracle, golden_dir, known, key):
    import _hyphy3 as h3
    k = known[key]
    a = h3.Alignment.load(str(golden_dir / k["alignment"])).to_nucleotide_alignment()
    t, g = _host(h3, k["newick"], k["theta"], k["freqs"])
    lnl, site = h3.compute_gtr_log_likelihood(t, a, g)
    ref, ref_site = oracle.gtr_loglik(oracle.Tree.parse(k["newick"]),
                                      oracle.nucleotide_patterns(oracle.Alignment.load(str(golden_dir / k["alignment"]))),
                                      k["theta"], k["freqs"])
    assert lnl == pytest.approx(ref, rel=1e-12)
    np.testing.assert_allclose(site, ref_site, rtol=1e-12, atol=1e-12)
    assert lnl == pytest.approx(k["log_l"], rel=1e-6)
    # a codon alignment is converted to its nucleotide patterns first
    lc, _ = h3.compute_gtr_log_likelihood(t, h3.Alignment.load(str(golden_dir / k["alignment"])), g)
    assert lc == lnl


def _check_synthetic(oracle, names, seqs, newick, theta, freqs):
    import _hyphy3 as h3
    a = h3.Alignment.from_sequences(names, seqs).to_nucleotide_alignment()
    t, g = _host(h3, newick, theta, freqs)
    lnl, site = h3.compute_gtr_log_likelihood(t, a, g)
    ref, ref_site = oracle.gtr_loglik(oracle.Tree.parse(newick), oracle.nucleotide_patterns(oracle.Alignment.from_sequences(names, seqs)),
                                      theta, freqs)
    assert lnl == pytest.approx(ref, rel=1e-11)
    np.testing.assert_allclose(site, ref_site, rtol=1e-11, atol=1e-11)
    return a


def test_gtr_simulated_with_gaps_and_ambiguity(oracle):
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=600, n_taxa=256)
    a = _check_synthetic(oracle, wl.names, wl.seqs, wl.newick, [0.6, 0.3, 0.4, 2.2, 0.5], [0.3, 0.2, 0.25, 0.25])
    assert a.num_patterns > 500


def test_gtr_caterpillar_tree(oracle):
    rng = np.random.default_rng(4)
    n = 300
    names = [f"s{i}" for i in range(n)]
    newick = names[0] + ":0.1"
    for i in range(1, n):
        newick = f"({newick},{names[i]}:{0.02 + 0.1 * rng.random():.4f}):0.01"
    newick += ";"
    nuc = np.array(list("ACGTRYN-"))
    seqs = ["".join(rng.choice(nuc, 90, p=[0.24, 0.24, 0.24, 0.24, 0.01, 0.01, 0.01, 0.01])) for _ in range(n)]
    _check_synthetic(oracle, names, seqs, newick, [1.0, 0.5, 0.8, 3.0, 0.7], [0.25, 0.25, 0.25, 0.25])


def test_gtr_rejects_codon_problem():
    import _hyphy3 as h3
    from hyphy3 import _capi
    c = _capi.Context(0)
    try:
        # a codon problem (states up to 60) is refused by the nucleotide evaluator
        st = np.array([[3, 40]], dtype=np.int8)
        mk = np.array([[1 << 3, 1 << 40]], dtype=np.uint64)
        pr = _capi.Problem(c, np.array([-1, 0, 0], np.int32), np.array([0, 1, 1], np.uint8), np.array([-1, 0, 1], np.int32),
                           st, mk, np.array([1.0]))
        import ctypes as C
        P = np.tile(np.eye(4), (3, 1, 1))
        lnl = C.c_double()
        st_code = c.lib.h3g_nuc_eval_from_P(pr.h, P.ctypes.data_as(C.POINTER(C.c_double)),
                                            np.full(4, 0.25).ctypes.data_as(C.POINTER(C.c_double)), C.byref(lnl), None)
        assert st_code == _capi.H3G_ERR_ARG
        pr.close()
    finally:
        c.close()


def test_gtr_many_patterns_depth_first_path(oracle):
    """More patterns than the level-by-level walk takes (131072): the depth-first, thread-per-pattern kernel."""
    rng = np.random.default_rng(9)
    n = 16
    names = [f"t{i}" for i in range(n)]
    newick = "(" + ",".join(f"({names[2 * i]}:0.1,{names[2 * i + 1]}:0.2):0.05" for i in range(n // 2)) + ");"
    cols = 141000                                                   # a multiple of 3; almost every column distinct
    seqs = ["".join(rng.choice(np.array(list("ACGTRN-")), cols, p=[0.24, 0.24, 0.24, 0.24, 0.02, 0.01, 0.01]))
            for _ in range(n)]
    a = _check_synthetic(oracle, names, seqs, newick, [0.9, 0.4, 0.6, 2.5, 0.8], [0.3, 0.2, 0.2, 0.3])
    assert a.num_patterns >= 131072
