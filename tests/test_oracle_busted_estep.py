"""BUSTED EM expectation steps (busted.hpp:662-975, :978-1134) and evaluate_log_l (:509-660) in the oracle.

The oracle restates the reference's loops (per test branch and class,
w_k post_m V.(P_k D)/L_m).  The device computes the same shares from the class-
and rate-weight gradients of one mixture evaluation (w_k dlnL/dw_k, rho_m dlnL/drho_m);
this test pins that identity on the CPU with the oracle's own gradients, plus the
normalisation and the evaluate_log_l sentinel behaviour.  There is no reference test of
the E-steps alone (tests/test_busted.cpp runs whole fits through the GTR fitter).
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def case(oracle):
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=80, n_taxa=12)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    t = oracle.Tree.parse(wl.newick)
    base = {"alpha": 1.0, "beta": 1.0, "theta": wl.theta}
    return a, t, base


@pytest.mark.parametrize("n_rates,background", [(1, False), (3, False), (2, True)])
def test_estep_equals_weight_gradient_identity(oracle, case, n_rates, background):
    a, t, base = case
    n = t.num_nodes()
    om, w = [0.05, 0.8, 4.0], [0.5, 0.35, 0.15]
    rates = [0.3, 1.0, 2.2][:n_rates] if n_rates > 1 else [1.0]
    rw = [0.3, 0.5, 0.2][:n_rates] if n_rates > 1 else [1.0]
    if n_rates == 2:
        rw = [0.4, 0.6]
    is_test = [int(i != t.root and (not background or i % 3 != 1)) for i in range(n)]
    omega_bg = 0.6 if background else -1.0
    bl = [1.7 * x for x in t.branch_lengths]
    e = oracle.busted_estep(t, a, base, bl, om, w, rates, rw, is_test, omega_bg)
    cls = [dict(base, beta=o) for o in om]
    bg = dict(base, beta=omega_bg) if background else None
    r = oracle.mixture_eval(t, a, cls, w, bg, [bool(x) for x in is_test], rates if n_rates > 1 else [],
                            rw if n_rates > 1 else [], bl, False, True, True)
    # evaluate_log_l: the same per-pattern log-sum-exp and -1e20 sentinel
    assert abs(e["lnl"] - r["lnl"]) <= 1e-10 * abs(r["lnl"])
    ok = np.asarray(e["pattern_ll"]) > -1e19
    total = float(np.dot(np.asarray(a.weights)[ok], np.ones(ok.sum())))
    n_test = sum(is_test)
    acc = np.asarray(w) * np.asarray(r["grad_class_w"])
    assert abs(acc.sum() - n_test * total) <= 1e-8 * n_test * total      # sum_k w_k V.P_k D = V.P_mix D = L
    expect = np.clip(acc / (n_test * total), 1e-6, 1 - 1e-6)
    np.testing.assert_allclose(e["weights"], expect / expect.sum(), rtol=1e-9, atol=1e-12)
    if n_rates > 1:
        accs = np.asarray(rw) * np.asarray(r["grad_rate_w"])
        expect = np.clip(accs / total, 1e-6, 1 - 1e-6)
        np.testing.assert_allclose(e["syn_weights"], expect / expect.sum(), rtol=1e-9, atol=1e-12)
    else:
        assert list(e["syn_weights"]) == [1.0]


def test_estep_moves_weights_uphill(oracle, case):
    """An EM step never lowers the likelihood (weights only, everything else fixed)."""
    a, t, base = case
    om, w = [0.05, 0.8, 4.0], [0.2, 0.2, 0.6]
    rates, rw = [0.3, 1.0, 2.2], [0.2, 0.2, 0.6]
    bl = list(t.branch_lengths)
    e0 = oracle.busted_estep(t, a, base, bl, om, w, rates, rw, [], -1.0)
    e1 = oracle.busted_estep(t, a, base, bl, om, e0["weights"], rates, e0["syn_weights"], [], -1.0)
    assert e1["lnl"] >= e0["lnl"] - 1e-9
