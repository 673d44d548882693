"""Model eigensystems solved on the device (h3g_eigen.cu) for the main engine.

A model installed as generators only (lam, U, V NULL) is diagonalised on the device.  Checks:
the eigensystem reconstructs Q and V = U^-1 to rounding; its transition matrices agree with the
oracle's Jacobi eigensystem within the two-solver floor (1e-10 absolute) and log-likelihoods
within 1e-11; an evaluation with the device eigensystem equals the oracle handed that same
eigensystem at 1e-10 (lnL, per-site, branch, omega, theta, class-weight and rate-weight
gradients); and the public API (which installs generators by default) matches the host
eigensolver's results at the floor.
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, dq_theta, problem_from_oracle, rel

pytestmark = pytest.mark.gpu


def _P(e, t):
    return np.maximum((e["U"] * np.exp(e["lam"] * t)) @ e["V"], 0.0)


@pytest.fixture(scope="module")
def ctx():
    from hyphy3 import _capi
    c = _capi.Context(0)
    yield c
    c.close()


def _cases(oracle, golden_dir, known):
    from hyphy3.simulate import make_workload
    k = known["cd2_reduced"]
    yield "cd2_reduced", oracle.Tree.parse(k["newick"]), oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna")), \
        {"alpha": 1.0, "beta": 0.45, "theta": [0.8, 1.2, 0.6, 1.8, 0.9]}
    a = oracle.Alignment.load(str(golden_dir / "adh.nex"))
    yield "adh", oracle.Tree.parse(a.embedded_tree), a, {"alpha": 1.0, "beta": 0.4, "theta": [1, 1, 1, 1, 1]}
    wl = make_workload(1, n_sites=300)
    yield "busted64", oracle.Tree.parse(wl.newick), oracle.Alignment.from_sequences(wl.names, wl.seqs), \
        {"alpha": 1.0, "beta": 0.5, "theta": list(wl.theta)}


def test_device_eigensystem_against_oracle(ctx, oracle, golden_dir, known):
    for name, t, a, p in _cases(oracle, golden_dir, known):
        own = oracle.mg94(a, p)
        Q = np.asarray(own["Q"])
        pr = problem_from_oracle(ctx, oracle, t, a)
        pr.set_model(pi=a.pi, Q=Q)
        dev = pr.get_eigensystem(0)
        S = Q.shape[0]
        # U diag(lam) V = Q and V U = I, to the rounding the sqrt(pi_j / pi_i) back-transformation leaves
        # (pi down to 1e-10 on cd2_reduced)
        rec = (dev["U"] * dev["lam"]) @ dev["V"]
        assert np.max(np.abs(rec - Q)) < 1e-10 * max(1.0, np.max(np.abs(Q))), name
        assert np.max(np.abs(dev["V"] @ dev["U"] - np.eye(S))) < 1e-10, name
        assert np.max(np.abs(np.sort(dev["lam"]) - np.sort(np.asarray(own["lam"])))) < 1e-12, name
        bl = [0.0 if i == t.root else (0.05 if name == "adh" else max(1e-4, x)) for i, x in enumerate(t.branch_lengths)]
        oe = {"U": np.asarray(own["U"]), "V": np.asarray(own["V"]), "lam": np.asarray(own["lam"])}
        Pd = [np.eye(S) if i == t.root else _P(dev, bl[i]) for i in range(t.num_nodes())]
        Po = [np.eye(S) if i == t.root else _P(oe, bl[i]) for i in range(t.num_nodes())]
        assert max(float(np.max(np.abs(x - y))) for x, y in zip(Pd, Po)) < 1e-10, name
        ld = oracle.loglik_from_P(t, a, Pd, np.asarray(a.pi))[0]
        lo = oracle.loglik_from_P(t, a, Po, np.asarray(a.pi))[0]
        assert abs(ld - lo) / abs(lo) < 1e-11, name
        # the engine with the device eigensystem == the oracle handed it
        lnl, g = pr.branch_length_gradients(pi=a.pi, Q=Q, lam=None, U=None, V=None, bl=np.array(bl))
        ref_l, ref_g = oracle.branch_length_gradients(t, a, dict(p, eig=dev), bl)
        assert abs(lnl - ref_l) / abs(ref_l) < 1e-10, name
        assert rel(g, ref_g) < 1e-10, name
        own_l, own_g = oracle.branch_length_gradients(t, a, p, bl)
        assert rel(g, own_g) < 5e-10, name
        pr.close()


def test_mixture_with_device_eigensystems(ctx, oracle):
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=150, n_taxa=20)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    models = [{"alpha": 1.0, "beta": om, "theta": list(wl.theta)} for om in wl.omegas]
    Q = np.stack([np.asarray(oracle.mg94(a, m)["Q"]) for m in models])
    nm = len(models)
    dirs = []
    for k in range(nm):
        d = np.zeros((nm, 61, 61))
        d[k] = dq_beta(a, models[k])
        dirs.append(d)
    for x in range(5):
        dirs.append(np.stack([dq_theta(a, x, m) for m in models]))
    pr = problem_from_oracle(ctx, oracle, t, a)
    rates, rw = [0.3, 1.0, 1.7], [0.2, 0.5, 0.3]
    pr.set_model(pi=a.pi, Q=Q, class_w=list(wl.omega_w), rates=rates, rate_w=rw, dQ=np.stack(dirs),
                 time_mode=_capi.TIME_NORMALIZED)
    eig = [pr.get_eigensystem(k) for k in range(nm)]
    bl = np.array(t.branch_lengths)
    out = pr.eval(bl, _capi.WANT_LNL | _capi.WANT_SITE_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL)
    cls = [dict(m, eig=e) for m, e in zip(models, eig)]
    ref = oracle.mixture_eval(t, a, cls, list(wl.omega_w), None, [], rates, rw, list(bl), True, True, False)
    assert abs(out["lnl"] - ref["lnl"]) / abs(ref["lnl"]) < 1e-10
    assert rel(out["site_lnl"], ref["site_lnl"]) < 1e-10
    assert rel(out["grad_t"], ref["grad_t"]) < 1e-10
    assert rel(out["grad_dir"][:nm], ref["grad_beta"]) < 1e-10
    assert rel(out["grad_dir"][nm:nm + 5], ref["grad_theta"]) < 1e-10
    assert rel(out["grad_class_w"], ref["grad_class_w"]) < 1e-10
    assert rel(out["grad_rate_w"], ref["grad_rate_w"]) < 1e-10
    pr.close()


def test_api_device_and_host_eigensolvers_agree(oracle, golden_dir):
    import _hyphy3 as h
    h.set_precision("fp64")
    a = h.Alignment.load(str(golden_dir / "adh.nex"))
    t = h.Tree.from_newick(a.embedded_tree_newick)
    p = h.MG94Parameters()
    p.beta = 0.4
    bl = [0.0 if i == t.root_id else 0.05 for i in range(t.num_nodes())]
    assert h.get_eigensolver() == "device"
    ld, gd = h.compute_branch_length_gradients(t, a, p, bl)
    h.set_eigensolver("host")
    try:
        lh, gh = h.compute_branch_length_gradients(t, a, p, bl)
    finally:
        h.set_eigensolver("device")
    assert abs(ld - lh) / abs(lh) < 1e-11
    assert rel(gd, gh) < 5e-10
