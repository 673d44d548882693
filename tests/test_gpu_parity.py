"""FP64 device path vs the CPU oracle on identical inputs, through the C ABI.

Tolerance: the FP64 path must agree with the oracle to 1e-10 relative (lnL) and
1e-10 of max(1, |g|max) for gradient vectors, on the same eigensystems.
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, dq_theta, eigensystems, problem_from_oracle, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def ctx():
    from hyphy3 import _capi
    c = _capi.Context(0)
    yield c
    c.close()


def _cd2(oracle, golden_dir, known):
    a = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = oracle.Tree.parse(known["cd2_reduced"]["newick"])
    return t, a


def _workload(oracle, config, **kw):
    from hyphy3.simulate import make_workload
    wl = make_workload(config, **kw)
    return oracle.Tree.parse(wl.newick), oracle.Alignment.from_sequences(wl.names, wl.seqs), wl


def test_branch_gradients_cd2_reduced(ctx, oracle, golden_dir, known):
    t, a = _cd2(oracle, golden_dir, known)
    p = {"alpha": 1.0, "beta": 0.5, "theta": [1, 1, 1, 2, 1]}
    Q, lam, U, V, mu = eigensystems(oracle, a, [p])
    pr = problem_from_oracle(ctx, oracle, t, a)
    bl = np.array(t.branch_lengths)
    lnl, g = pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=bl)
    ref_l, ref_g = oracle.branch_length_gradients(t, a, p, list(bl))
    assert abs(lnl - ref_l) / abs(ref_l) < TOL
    assert rel(g, ref_g) < TOL
    assert abs(lnl - known["cd2_reduced"]["point_mg94_logl"]) / 92.8 < 1e-9


def test_branch_gradients_adh(ctx, oracle, golden_dir):
    a = oracle.Alignment.load(str(golden_dir / "adh.nex"))
    t = oracle.Tree.parse(a.embedded_tree)
    p = {"alpha": 1.0, "beta": 0.4, "theta": [1, 1, 1, 1, 1]}
    Q, lam, U, V, _ = eigensystems(oracle, a, [p])
    pr = problem_from_oracle(ctx, oracle, t, a)
    bl = np.array([0.0 if i == t.root else 0.05 for i in range(t.num_nodes())])
    lnl, g = pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=bl)
    ref_l, ref_g = oracle.branch_length_gradients(t, a, p, list(bl))
    assert abs(lnl - ref_l) / abs(ref_l) < TOL
    assert rel(g, ref_g) < TOL


@pytest.mark.parametrize("config,kw", [(0, {}), (1, {"n_sites": 200, "n_taxa": 24})])
def test_branch_gradients_synthetic(ctx, oracle, config, kw):
    t, a, wl = _workload(oracle, config, **kw)
    p = {"alpha": 1.0, "beta": 0.5, "theta": wl.theta}
    Q, lam, U, V, _ = eigensystems(oracle, a, [p])
    pr = problem_from_oracle(ctx, oracle, t, a)
    bl = np.array(t.branch_lengths)
    lnl, g = pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=bl)
    ref_l, ref_g = oracle.branch_length_gradients(t, a, p, list(bl))
    assert abs(lnl - ref_l) / abs(ref_l) < TOL
    assert rel(g, ref_g) < TOL


@pytest.mark.parametrize("n_rates,partition", [(1, False), (1, True), (3, True)])
def test_mixture_lnl_and_all_gradients(ctx, oracle, n_rates, partition):
    from hyphy3 import _capi
    t, a, wl = _workload(oracle, 1, n_sites=150, n_taxa=20)
    om, w = [0.1, 1.0, 5.0], [0.6, 0.3, 0.1]
    cls = [{"alpha": 1.0, "beta": o, "theta": wl.theta} for o in om]
    bg = {"alpha": 1.0, "beta": 0.7, "theta": wl.theta}
    is_test = [(i % 3 != 1) or not partition for i in range(t.num_nodes())]
    rates = [0.3, 1.0, 1.7][:n_rates] if n_rates > 1 else [1.0]
    rw = [0.2, 0.5, 0.3][:n_rates] if n_rates > 1 else [1.0]
    models = cls + ([bg] if partition else [])
    Q, lam, U, V, mu = eigensystems(oracle, a, models)
    nm = len(models)
    dirs = []
    for k in range(3):
        d = np.zeros((nm, 61, 61)); d[k] = dq_beta(a, models[k]); dirs.append(d)
    if partition:
        d = np.zeros((nm, 61, 61)); d[3] = dq_beta(a, bg); dirs.append(d)
    for x in range(5):
        dirs.append(np.stack([dq_theta(a, x, m) for m in models]))
    pr = problem_from_oracle(ctx, oracle, t, a)
    pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=w, has_bg=partition,
                 is_test=np.array(is_test, dtype=np.uint8), rates=rates, rate_w=rw, dQ=np.stack(dirs))
    bl = np.array(t.branch_lengths)
    out = pr.eval(bl, _capi.WANT_LNL | _capi.WANT_SITE_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL)
    ref = oracle.mixture_eval(t, a, cls, w, bg if partition else None, is_test if partition else [],
                              rates if n_rates > 1 else [], rw if n_rates > 1 else [], list(bl), False, True, False)
    assert abs(out["lnl"] - ref["lnl"]) / abs(ref["lnl"]) < TOL
    assert rel(out["site_lnl"], ref["site_lnl"]) < TOL
    assert rel(out["grad_t"], ref["grad_t"]) < TOL
    q = 3
    assert rel(out["grad_dir"][:3], ref["grad_beta"]) < TOL
    if partition:
        assert rel(out["grad_dir"][3:4], [ref["grad_beta_bg"]]) < TOL
        q = 4
    assert rel(out["grad_dir"][q:q + 5], ref["grad_theta"]) < TOL
    assert rel(out["grad_class_w"], ref["grad_class_w"]) < TOL
    if n_rates > 1:
        assert rel(out["grad_rate_w"], ref["grad_rate_w"]) < TOL


def test_joint_frechet_normalized_time(ctx, oracle, golden_dir, known):
    from hyphy3 import _capi
    t, a = _cd2(oracle, golden_dir, known)
    p = {"alpha": 1.0, "beta": 0.45, "theta": [0.8, 1.2, 0.6, 1.8, 0.9]}
    Q, lam, U, V, mu = eigensystems(oracle, a, [p])
    dirs = [dq_beta(a, p)[None]] + [dq_theta(a, x, p)[None] for x in range(5)]
    pr = problem_from_oracle(ctx, oracle, t, a)
    pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, time_mode=_capi.TIME_NORMALIZED, dQ=np.stack(dirs))
    bl = np.array([0.0 if i == t.root else max(1e-4, x) for i, x in enumerate(t.branch_lengths)])
    out = pr.eval(bl, _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL)
    ref = oracle.joint_frechet_gradients(t, a, p, list(bl))
    assert abs(out["lnl"] - ref["lnl"]) / abs(ref["lnl"]) < TOL
    assert rel(out["grad_t"], ref["grad_t"]) < TOL
    assert rel(out["grad_dir"][:1], ref["grad_beta"]) < TOL
    assert rel(out["grad_dir"][1:6], ref["grad_theta"]) < TOL


def test_loglik_from_given_P_with_sentinel(ctx, oracle):
    t, a, wl = _workload(oracle, 1, n_sites=100, n_taxa=16)
    p = {"alpha": 1.0, "beta": 0.8, "theta": wl.theta}
    n = t.num_nodes()
    Ps = [np.eye(61) if i == t.root else oracle.transition_matrix(a, p, t.branch_lengths[i]) for i in range(n)]
    # one branch that forbids every change from codon 0 makes some patterns impossible
    Ps[3] = Ps[3].copy()
    Ps[3][:, :] = np.eye(61)
    pr = problem_from_oracle(ctx, oracle, t, a)
    lnl, site = pr.eval_from_P(np.stack(Ps), a.pi)
    ref_l, ref_site = oracle.loglik_from_P(t, a, Ps, a.pi)
    assert abs(lnl - ref_l) <= TOL * abs(ref_l)
    np.testing.assert_allclose(site, ref_site, rtol=TOL, atol=0)


def test_repeated_evaluations_are_bit_identical(ctx, oracle):
    from hyphy3 import _capi
    t, a, wl = _workload(oracle, 1, n_sites=300, n_taxa=32)
    p = {"alpha": 1.0, "beta": 0.5, "theta": wl.theta}
    Q, lam, U, V, mu = eigensystems(oracle, a, [p])
    pr = problem_from_oracle(ctx, oracle, t, a)
    pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, dQ=np.stack([dq_beta(a, p)[None]]))
    bl = np.array(t.branch_lengths)
    want = _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL
    r1 = {k: np.copy(v) if isinstance(v, np.ndarray) else v for k, v in pr.eval(bl, want).items()}
    r2 = pr.eval(bl, want)
    assert r1["lnl"] == r2["lnl"]
    np.testing.assert_array_equal(r1["grad_t"], r2["grad_t"])
    np.testing.assert_array_equal(r1["grad_dir"], r2["grad_dir"])


@pytest.mark.parametrize("newick", [
    "((T1:0.1,T2:0.2):0.05,(T3:0.1,T4:0.3):0.02);",                 # rooted, bifurcating root
    "((T1:0.1,T2:0.2,T3:0.05):0.1,T4:0.3,(T5:0.2,T6:0.0):0.1);",    # multifurcation, zero length
    "((T1:0.1,T2:0.2):0.05,T3:0.1,(T4:0.3,TX:0.2):0.02);",          # leaf without a sequence
])
def test_edge_topologies(ctx, oracle, newick):
    from hyphy3.simulate import make_workload
    wl = make_workload(0, n_sites=70, n_taxa=8)
    names = ["T1", "T2", "T3", "T4", "T5", "T6"]
    seqs = [s for nm, s in zip(wl.names, wl.seqs) if nm in names][:6]
    seqs[2] = "---" * 5 + seqs[2][15:]          # gaps
    seqs[1] = seqs[1][:9] + "NNN" + "RAC" + seqs[1][15:]   # ambiguity
    a = oracle.Alignment.from_sequences(names[:len(seqs)], seqs)
    t = oracle.Tree.parse(newick)
    p = {"alpha": 1.0, "beta": 0.5, "theta": wl.theta}
    Q, lam, U, V, _ = eigensystems(oracle, a, [p])
    pr = problem_from_oracle(ctx, oracle, t, a)
    bl = np.array(t.branch_lengths)
    lnl, g = pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=bl)
    ref_l, ref_g = oracle.branch_length_gradients(t, a, p, list(bl))
    assert abs(lnl - ref_l) / abs(ref_l) < TOL
    assert rel(g, ref_g) < TOL


def test_single_pattern_and_invalid_arguments(ctx, oracle):
    from hyphy3 import _capi
    a = oracle.Alignment.from_sequences(["A", "B", "C"], ["ATG", "ATG", "ATA"])
    t = oracle.Tree.parse("(A:0.1,B:0.2,C:0.3);")
    p = {"alpha": 1.0, "beta": 0.5, "theta": [1, 1, 1, 1, 1]}
    Q, lam, U, V, _ = eigensystems(oracle, a, [p])
    pr = problem_from_oracle(ctx, oracle, t, a)
    lnl, g = pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=np.array(t.branch_lengths))
    ref_l, ref_g = oracle.branch_length_gradients(t, a, p, list(t.branch_lengths))
    assert abs(lnl - ref_l) / abs(ref_l) < TOL and rel(g, ref_g) < TOL
    with pytest.raises(_capi.H3GError):
        _capi.Problem(ctx, np.array([-1, 0, 5], dtype=np.int32), np.array([0, 1, 1], dtype=np.uint8),
                      np.array([-1, 0, 1], dtype=np.int32), a.states, a.masks, a.weights)
    with pytest.raises(_capi.H3GError):
        pr.branch_length_gradients(pi=a.pi, Q=Q[0], lam=lam[0], U=U[0], V=V[0], bl=np.array([0.0, np.nan, 0.1, 0.1]))
