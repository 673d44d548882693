"""Split-precision tensor-core path vs the FP64 oracle.

Accuracy bar of the mixed path: |dlnL|/|lnL| <= 1e-7 and gradient relative error
(2-norm over all reported components) <= 1e-5 against FP64 on the same inputs.
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, dq_theta, eigensystems, problem_from_oracle

pytestmark = pytest.mark.gpu
LNL_TOL = 1e-7
GRAD_TOL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    from hyphy3 import _capi
    c = _capi.Context(0)
    yield c
    c.close()


def _norm_rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _workload(oracle, config, **kw):
    from hyphy3.simulate import make_workload
    wl = make_workload(config, **kw)
    return oracle.Tree.parse(wl.newick), oracle.Alignment.from_sequences(wl.names, wl.seqs), wl


@pytest.mark.parametrize("case", ["cd2_reduced", "adh", "config0"])
def test_mixed_branch_gradients(ctx, oracle, golden_dir, known, case):
    from hyphy3 import _capi
    if case == "cd2_reduced":
        a = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
        t = oracle.Tree.parse(known["cd2_reduced"]["newick"])
        p = {"alpha": 1.0, "beta": 0.5, "theta": [1, 1, 1, 2, 1]}
        bl = np.array(t.branch_lengths)
    elif case == "adh":
        a = oracle.Alignment.load(str(golden_dir / "adh.nex"))
        t = oracle.Tree.parse(a.embedded_tree)
        p = {"alpha": 1.0, "beta": 0.4, "theta": [1, 1, 1, 1, 1]}
        bl = np.array([0.0 if i == t.root else 0.05 for i in range(t.num_nodes())])
    else:
        t, a, wl = _workload(oracle, 0)
        p = {"alpha": 1.0, "beta": 0.5, "theta": wl.theta}
        bl = np.array(t.branch_lengths)
    Q, lam, U, V, _ = eigensystems(oracle, a, [p])
    pr = problem_from_oracle(ctx, oracle, t, a)
    lnl, g = pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=bl, precision=_capi.PREC_MIXED)
    ref_l, ref_g = oracle.branch_length_gradients(t, a, p, list(bl))
    assert abs(lnl - ref_l) / abs(ref_l) <= LNL_TOL
    assert _norm_rel(g, ref_g) <= GRAD_TOL


@pytest.mark.parametrize("n_rates,partition", [(1, False), (2, True)])
def test_mixed_mixture_all_gradients(ctx, oracle, n_rates, partition):
    from hyphy3 import _capi
    t, a, wl = _workload(oracle, 1, n_sites=300, n_taxa=32)
    om, w = [0.1, 1.0, 5.0], [0.6, 0.3, 0.1]
    cls = [{"alpha": 1.0, "beta": o, "theta": wl.theta} for o in om]
    bg = {"alpha": 1.0, "beta": 0.7, "theta": wl.theta}
    is_test = [(i % 3 != 1) or not partition for i in range(t.num_nodes())]
    rates, rw = ([0.4, 1.6], [0.5, 0.5]) if n_rates > 1 else ([1.0], [1.0])
    models = cls + ([bg] if partition else [])
    Q, lam, U, V, mu = eigensystems(oracle, a, models)
    nm = len(models)
    dirs = []
    for k in range(3):
        d = np.zeros((nm, 61, 61)); d[k] = dq_beta(a, models[k]); dirs.append(d)
    for x in range(5):
        dirs.append(np.stack([dq_theta(a, x, mm) for mm in models]))
    pr = problem_from_oracle(ctx, oracle, t, a)
    pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=w, has_bg=partition,
                 is_test=np.array(is_test, dtype=np.uint8), rates=rates, rate_w=rw, dQ=np.stack(dirs),
                 precision=_capi.PREC_MIXED)
    bl = np.array(t.branch_lengths)
    out = pr.eval(bl, _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL)
    ref = oracle.mixture_eval(t, a, cls, w, bg if partition else None, is_test if partition else [],
                              rates if n_rates > 1 else [], rw if n_rates > 1 else [], list(bl), False, True, False)
    assert abs(out["lnl"] - ref["lnl"]) / abs(ref["lnl"]) <= LNL_TOL
    got = np.r_[out["grad_t"], out["grad_dir"][:3], out["grad_dir"][3:8], out["grad_class_w"]]
    exp = np.r_[ref["grad_t"], ref["grad_beta"], ref["grad_theta"], ref["grad_class_w"]]
    assert _norm_rel(got, exp) <= GRAD_TOL


def test_mixed_deep_tree_no_underflow(ctx, oracle):
    """A 128-taxon Yule tree with short and long branches: FP32 partials must not underflow."""
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    wl = make_workload(3, n_sites=128, n_taxa=128)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    p = {"alpha": 1.0, "beta": 0.3, "theta": wl.theta}
    Q, lam, U, V, _ = eigensystems(oracle, a, [p])
    pr = problem_from_oracle(ctx, oracle, t, a)
    bl = np.array(t.branch_lengths)
    lnl, g = pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=bl, precision=_capi.PREC_MIXED)
    ref_l, ref_g = oracle.branch_length_gradients(t, a, p, list(bl))
    assert abs(lnl - ref_l) / abs(ref_l) <= LNL_TOL
    assert _norm_rel(g, ref_g) <= GRAD_TOL


def test_mixed_extreme_branch_lengths_stay_finite(ctx, oracle):
    """Branch lengths pushed towards both ends (x e^{+-18}, clipped to [1e-8, 1e4], as an optimiser's
    first trial step does): the mixed path's lnL and gradients stay finite and its lnL follows
    FP64's (to 1e-6 here).  Products of nearly disjoint messages reach the FP32 subnormal range here; a node's last
    product is then renormalised (renorm_if_small), else the gradient operand's scale overflows."""
    from hyphy3 import _capi
    t, a, wl = _workload(oracle, 1, n_sites=300)
    p = {"alpha": 1.0, "beta": 0.5, "theta": list(wl.theta)}
    Q, lam, U, V, _ = eigensystems(oracle, a, [p])
    pr = problem_from_oracle(ctx, oracle, t, a)
    rng = np.random.default_rng(5)
    bl = np.array(t.branch_lengths) * np.exp(rng.choice([-18.0, 18.0], size=t.num_nodes()))
    bl = np.clip(bl, 1e-8, 1e4)
    bl[t.root] = 0.0
    l64, g64 = pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=bl, precision=_capi.PREC_FP64)
    lmx, gmx = pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=bl, precision=_capi.PREC_MIXED)
    assert np.isfinite(l64) and np.isfinite(lmx)
    assert np.all(np.isfinite(gmx)), np.flatnonzero(~np.isfinite(gmx))
    assert abs(lmx - l64) / abs(l64) <= 10 * LNL_TOL       # far outside the fitted regime: a looser bar
    pr.close()
