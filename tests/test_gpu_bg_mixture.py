"""Mixtures on background branches (h3g_model_desc.has_bg > 1 with bg_w): the RELAX and two-set BUSTED
likelihood (relax.hpp:571-803; busted.hpp:3146-3683), P_b = sum_j v_j exp(Q_j t_b) on background branches
next to P_b = sum_k w_k exp(Q_k t_b) on test branches, synonymous-rate classes as separate passes.

The log-likelihood and per-pattern values are checked against the oracle's pruning of the same mixed
matrices (loglik_from_P, rate classes combined per pattern by log-sum-exp); the gradients in branch lengths,
background weights and background omegas against central differences of that oracle likelihood, and against
the one-background-model path when every background class has the same omega.
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, dq_theta, eigensystems, problem_from_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from hyphy3 import _capi
    c = _capi.Context(0)
    yield c
    c.close()


def _setup(oracle, n_taxa=12, n_sites=60):
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=n_sites, n_taxa=n_taxa)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    is_test = [(i % 3 == 0) and i != t.root for i in range(t.num_nodes())]
    return t, a, wl, is_test


def _oracle_lnl(oracle, t, a, theta, is_test, om, w, bom, bw, bl, rates=(1.0,), rw=(1.0,)):
    n = t.num_nodes()
    per_rate = []
    for r in rates:
        Ps = []
        for b in range(n):
            if b == t.root:
                Ps.append(np.eye(61))
                continue
            oms, ws = (om, w) if is_test[b] else (bom, bw)
            Ps.append(sum(wk * np.array(oracle.transition_matrix(a, {"alpha": 1.0, "beta": o, "theta": theta}, r * bl[b]))
                          for o, wk in zip(oms, ws)))
        per_rate.append(np.array(oracle.loglik_from_P(t, a, Ps, list(a.pi))[1]))
    site = np.logaddexp.reduce(np.stack([np.log(q) + s for q, s in zip(rw, per_rate)]), axis=0)
    return float(np.dot(a.weights, site)), site


def _device(ctx, oracle, t, a, theta, is_test, om, w, bom, bw, bl, rates=(1.0,), rw=(1.0,)):
    from hyphy3 import _capi
    models = [{"alpha": 1.0, "beta": o, "theta": theta} for o in list(om) + list(bom)]
    Q, lam, U, V, mu = eigensystems(oracle, a, models)
    nm = len(models)
    dirs = []
    for k in range(nm):
        d = np.zeros((nm, 61, 61)); d[k] = dq_beta(a, models[k]); dirs.append(d)
    for x in range(5):
        dirs.append(np.stack([dq_theta(a, x, m) for m in models]))
    pr = problem_from_oracle(ctx, oracle, t, a)
    pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=w, is_test=np.array(is_test, dtype=np.uint8),
                 rates=list(rates), rate_w=list(rw), dQ=np.stack(dirs), bg_w=bw)
    return pr.eval(np.array(bl), _capi.WANT_LNL | _capi.WANT_SITE_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL)


@pytest.mark.parametrize("rates,rw", [((1.0,), (1.0,)), ((0.4, 1.0, 2.2), (0.3, 0.5, 0.2))])
def test_background_mixture_matches_oracle(ctx, oracle, rates, rw):
    t, a, wl, is_test = _setup(oracle)
    om, w = [0.05, 0.6, 3.0], [0.5, 0.4, 0.1]
    bom, bw = [0.02, 0.3, 1.5], [0.3, 0.5, 0.2]
    bl = list(t.branch_lengths)
    out = _device(ctx, oracle, t, a, wl.theta, is_test, om, w, bom, bw, bl, rates, rw)
    ref, ref_site = _oracle_lnl(oracle, t, a, wl.theta, is_test, om, w, bom, bw, bl, rates, rw)
    assert out["lnl"] == pytest.approx(ref, rel=1e-11)
    np.testing.assert_allclose(out["site_lnl"], ref_site, rtol=1e-10, atol=1e-10)
    f = lambda **kw: _oracle_lnl(oracle, t, a, wl.theta, is_test, kw.get("om", om), w, kw.get("bom", bom), kw.get("bw", bw),
                                 kw.get("bl", bl), rates, rw)[0]
    h = 1e-5       # steps large enough that the oracle's rounding (~1e-12 in lnL) stays far below the tolerance
    for j in range(3):                                   # background weights (unconstrained partials)
        up, dn = list(bw), list(bw)
        up[j] += h; dn[j] -= h
        assert out["grad_bg_w"][j] == pytest.approx((f(bw=up) - f(bw=dn)) / (2 * h), rel=1e-5, abs=1e-5), j
    for j in range(3):                                   # background omegas: directions 3..5
        up, dn = list(bom), list(bom)
        hj = 1e-4 * max(bom[j], 0.05)
        up[j] += hj; dn[j] -= hj
        assert out["grad_dir"][3 + j] == pytest.approx((f(bom=up) - f(bom=dn)) / (2 * hj), rel=1e-5, abs=1e-5), j
    for b in [i for i in range(t.num_nodes()) if i != t.root][:6]:
        up, dn = list(bl), list(bl)
        hb = 1e-5 * max(bl[b], 1e-2)
        up[b] += hb; dn[b] -= hb
        assert out["grad_t"][b] == pytest.approx((f(bl=up) - f(bl=dn)) / (2 * hb), rel=1e-5, abs=1e-5), b


def test_equal_background_classes_reduce_to_one_model(ctx, oracle):
    """Background classes that share one omega mix to that model alone: same lnL and gradients as the one-model
    path, the omega gradients split across the classes and every weight gradient equal."""
    t, a, wl, is_test = _setup(oracle)
    om, w = [0.05, 0.6, 3.0], [0.5, 0.4, 0.1]
    bl = list(t.branch_lengths)
    out = _device(ctx, oracle, t, a, wl.theta, is_test, om, w, [0.4, 0.4], [0.7, 0.3], bl)
    one = _device(ctx, oracle, t, a, wl.theta, is_test, om, w, [0.4], [1.0], bl)
    assert out["lnl"] == pytest.approx(one["lnl"], rel=1e-12)
    np.testing.assert_allclose(out["grad_t"], one["grad_t"], rtol=1e-9, atol=1e-9)
    assert out["grad_dir"][3] + out["grad_dir"][4] == pytest.approx(one["grad_dir"][3], rel=1e-9)
    assert out["grad_bg_w"][0] == pytest.approx(out["grad_bg_w"][1], rel=1e-9)
    np.testing.assert_allclose(out["grad_dir"][5:10], one["grad_dir"][4:9], rtol=1e-9, atol=1e-9)   # theta


def test_bad_background_descriptors_are_rejected(ctx, oracle):
    from hyphy3 import _capi
    t, a, wl, is_test = _setup(oracle, n_taxa=6, n_sites=10)
    models = [{"alpha": 1.0, "beta": o, "theta": wl.theta} for o in (0.3, 0.5, 0.9)]
    Q, lam, U, V, mu = eigensystems(oracle, a, models)
    pr = problem_from_oracle(ctx, oracle, t, a)
    with pytest.raises(_capi.H3GError):              # two background models without weights
        pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=[1.0], has_bg=2,
                     is_test=np.array(is_test, dtype=np.uint8))
    with pytest.raises(_capi.H3GError):              # non-finite background weights
        pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=[1.0], is_test=np.array(is_test, dtype=np.uint8),
                     bg_w=[0.5, float("nan")])
