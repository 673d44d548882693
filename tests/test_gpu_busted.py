"""BUSTED likelihood core on the device: evaluate_log_l and the EM expectation steps
(busted.hpp:509-660, :662-975, :978-1134) through hyphy3.BUSTEDAnalyzer, against the
oracle's restatement of the reference loops."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(oracle, n_taxa, n_sites, seed_cfg=1):
    import _hyphy3 as h
    from hyphy3.simulate import make_workload
    wl = make_workload(seed_cfg, n_sites=n_sites, n_taxa=n_taxa)
    p = h.MG94Parameters()
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = wl.theta
    p.beta = 0.7
    b = h.BUSTEDAnalyzer(h.Tree.from_newick(wl.newick), h.Alignment.from_sequences(wl.names, wl.seqs), p)
    oa = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    ot = oracle.Tree.parse(wl.newick)
    base = {"alpha": 1.0, "beta": 0.7, "theta": list(wl.theta)}
    return b, oa, ot, base


@pytest.mark.parametrize("n_rates,background", [(1, False), (3, False), (2, True)])
def test_busted_core_matches_oracle(oracle, n_rates, background):
    b, oa, ot, base = _setup(oracle, 24, 150)
    n = ot.num_nodes()
    if background:
        b.is_test_branch = [i != ot.root and i % 3 != 1 for i in range(n)]
        b.mg94_background_omega = 0.45
    om, w = [0.05, 0.8, 4.0], [0.5, 0.35, 0.15]
    rates = [0.3, 1.0, 2.2][:n_rates] if n_rates > 1 else [1.0]
    rw = [0.3, 0.5, 0.2] if n_rates == 3 else ([0.4, 0.6] if n_rates == 2 else [1.0])
    s = 1.3
    bl = [s * x for x in b.branch_tau]
    is_test = [int(x) for x in b.is_test_branch]
    omega_bg = 0.45 if background else -1.0
    ref = oracle.busted_estep(ot, oa, base, bl, om, w, rates, rw, is_test, omega_bg)
    lnl, pll = b.evaluate_log_l(s, om, w, rates, rw)
    assert abs(lnl - ref["lnl"]) <= 1e-10 * abs(ref["lnl"])
    np.testing.assert_allclose(pll, ref["pattern_ll"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(b.compute_expected_weights(s, om, w, rates, rw), ref["weights"], rtol=1e-9, atol=1e-12)
    if n_rates > 1:
        np.testing.assert_allclose(b.compute_expected_syn_weights(s, om, w, rates, rw), ref["syn_weights"], rtol=1e-9,
                                   atol=1e-12)
    # custom branch lengths replace branch_tau (then scaled by s)
    custom = [0.8 * x for x in b.branch_tau]
    ref2 = oracle.busted_estep(ot, oa, base, [s * x for x in custom], om, w, rates, rw, is_test, omega_bg)
    assert abs(b.evaluate_log_l(s, om, w, rates, rw, custom)[0] - ref2["lnl"]) <= 1e-10 * abs(ref2["lnl"])


def test_busted_em_iterations_climb(oracle):
    """Weight-only EM on the device: every E-step/M-step pair raises lnL and the weights converge."""
    b, *_ = _setup(oracle, 32, 300)
    om, w = [0.05, 0.6, 3.0], [1 / 3, 1 / 3, 1 / 3]
    rates, rw = [0.4, 1.0, 1.9], [1 / 3, 1 / 3, 1 / 3]
    last = b.evaluate_log_l(1.0, om, w, rates, rw)[0]
    for _ in range(8):
        w2 = b.compute_expected_weights(1.0, om, w, rates, rw)
        rw = b.compute_expected_syn_weights(1.0, om, w, rates, rw)
        w = w2
        cur = b.evaluate_log_l(1.0, om, w, rates, rw)[0]
        assert cur >= last - 1e-8
        last = cur
    assert abs(sum(w) - 1.0) < 1e-12 and abs(sum(rw) - 1.0) < 1e-12
    assert all(1e-6 <= x <= 1 - 1e-6 for x in w)
