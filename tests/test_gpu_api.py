"""The reference-facing API (_hyphy3, hyphy3.autograd) on the device.

The API installs MG94 generators and the device diagonalises them (parallel cyclic
Jacobi, h3g_eigen.cu).  The oracle is handed that same eigensystem ("eig" in its
parameters; read back through h3g_model_get_eigensystem from the same generator), so
lnL and every gradient are compared like with like at the FP64 bound, 1e-10.  Against
the oracle's own Jacobi eigensystem the comparison is at the floor two correct FP64
eigensolvers leave (tests/test_eigen_floor.py pins it on the CPU for the host solver,
tests/test_gpu_eigen.py for the device one: gradients within 5e-10).
"""
import math

import numpy as np
import pytest

from gpu_helpers import rel

pytestmark = pytest.mark.gpu
TOL_API = 1e-10
TOL_EIG_FLOOR = 5e-10


_EIG_CTX = []


def host_eig(h3, aln, beta, theta=(1, 1, 1, 1, 1)):
    """The eigensystem the API installs for MG94(beta, theta) on aln, in the oracle's "eig" form: the
    device's (the default eigensolver: the same generator diagonalised by the same kernel through the
    C ABI) or, with set_eigensolver("host"), the host solver's."""
    from hyphy3 import _capi
    p = h3.MG94Parameters()
    p.beta = beta
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = theta
    e = h3.mg94_eigensystem(aln, p)
    if h3.get_eigensolver() == "host":
        return {"U": np.asarray(e["U"]), "V": np.asarray(e["V"]), "lam": np.asarray(e["lam"])}
    if not _EIG_CTX:
        _EIG_CTX.append(_capi.Context(0))
    pr = _capi.Problem(_EIG_CTX[0], np.array([-1, 0, 0, 0], dtype=np.int32), np.array([0, 1, 1, 1], dtype=np.uint8),
                       np.array([-1, 0, 1, 2], dtype=np.int32), np.zeros((1, 3), dtype=np.int8),
                       np.zeros((1, 3), dtype=np.uint64), np.ones(1))
    pr.set_model(pi=np.asarray(aln.codon_frequencies), Q=np.asarray(e["Q"]))
    out = pr.get_eigensystem(0)
    pr.close()
    return out


@pytest.fixture(scope="module")
def h3():
    import _hyphy3
    _hyphy3.set_precision("fp64")
    return _hyphy3


def test_point_loglik_matches_hyphy25(h3, known, golden_dir):
    k = known["cd2_reduced"]
    a = h3.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = h3.Tree.from_newick(k["newick"])
    p = h3.MG94Parameters()
    p.beta, p.theta_CT = 0.5, 2.0
    lnl = h3.compute_mg94_log_likelihood(t, a, p)
    assert abs(lnl - k["point_mg94_logl"]) / abs(k["point_mg94_logl"]) < 1e-9
    ll2, g = h3.compute_branch_length_gradients(t, a, p)
    assert abs(ll2 - lnl) < 1e-12 * abs(lnl)


def test_branch_gradients_api_vs_oracle(h3, oracle, golden_dir):
    a = h3.Alignment.load(str(golden_dir / "adh.nex"))
    t = h3.Tree.from_newick(a.embedded_tree_newick)
    b = oracle.Alignment.load(str(golden_dir / "adh.nex"))
    u = oracle.Tree.parse(b.embedded_tree)
    p = h3.MG94Parameters()
    p.beta = 0.4
    bl = [0.0 if i == t.root_id else 0.05 for i in range(t.num_nodes())]
    lnl, g = h3.compute_branch_length_gradients(t, a, p, bl)
    ref_l, ref_g = oracle.branch_length_gradients(u, b, {"alpha": 1.0, "beta": 0.4, "eig": host_eig(h3, a, 0.4)}, bl)
    assert abs(lnl - ref_l) / abs(ref_l) < TOL_API
    assert rel(g, ref_g) < TOL_API
    own_l, own_g = oracle.branch_length_gradients(u, b, {"alpha": 1.0, "beta": 0.4}, bl)
    assert abs(lnl - own_l) / abs(own_l) < TOL_API
    assert rel(g, own_g) < TOL_EIG_FLOOR


def test_joint_frechet_api_vs_oracle(h3, oracle, golden_dir, known):
    k = known["cd2_reduced"]
    a = h3.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = h3.Tree.from_newick(k["newick"])
    b = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    u = oracle.Tree.parse(k["newick"])
    p = h3.MG94Parameters()
    p.beta, p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = 0.45, 0.8, 1.2, 0.6, 1.8, 0.9
    bl = [0.0 if i == t.root_id else max(1e-4, x) for i, x in enumerate(t.get_branch_lengths())]
    th = [0.8, 1.2, 0.6, 1.8, 0.9]
    r = h3.compute_joint_frechet_gradients(t, a, p, bl)
    for eig, tol in ((host_eig(h3, a, 0.45, th), TOL_API), (None, TOL_EIG_FLOOR)):
        ref = oracle.joint_frechet_gradients(u, b, {"alpha": 1.0, "beta": 0.45, "theta": th, "eig": eig}, bl)
        assert abs(r["log_likelihood"] - ref["lnl"]) / abs(ref["lnl"]) < TOL_API
        assert rel(r["grad_branches"], ref["grad_t"]) < tol
        assert abs(r["grad_omega"] - ref["grad_beta"][0]) / (1 + abs(ref["grad_beta"][0])) < tol
        assert rel(r["grad_theta"], ref["grad_theta"]) < tol
    # partitioned: every third branch in the background with omega_bg = 0.9 (the background model's
    # eigensystem is the oracle's own here: the comparison is at the eigensolver floor)
    mask = [i % 3 != 2 for i in range(t.num_nodes())]
    r2 = h3.compute_joint_frechet_gradients(t, a, p, bl, mask, 0.9)
    ref2 = oracle.joint_frechet_gradients(u, b, {"alpha": 1.0, "beta": 0.45, "theta": th}, bl, mask, 0.9)
    assert abs(r2["log_likelihood"] - ref2["lnl"]) / abs(ref2["lnl"]) < TOL_API
    assert abs(r2["grad_omega_bg"] - ref2["grad_beta_bg"]) / (1 + abs(ref2["grad_beta_bg"])) < TOL_EIG_FLOOR


def test_mixture_api_vs_oracle(h3, oracle):
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=200, n_taxa=24)
    a = h3.Alignment.from_sequences(wl.names, wl.seqs)
    t = h3.Tree.from_newick(wl.newick)
    b = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    u = oracle.Tree.parse(wl.newick)
    base = h3.MG94Parameters()
    base.theta_AC, base.theta_AT, base.theta_CG, base.theta_CT, base.theta_GT = wl.theta
    bl = t.get_branch_lengths()
    r = h3.compute_mixture_gradients(t, a, base, bl, wl.omegas, wl.omega_w, [0.4, 1.6], [0.5, 0.5])
    for own in (False, True):
        cls = [{"alpha": 1.0, "beta": o, "theta": wl.theta, "eig": None if own else host_eig(h3, a, o, wl.theta)}
               for o in wl.omegas]
        tol = TOL_EIG_FLOOR if own else TOL_API
        ref = oracle.mixture_eval(u, b, cls, wl.omega_w, None, [], [0.4, 1.6], [0.5, 0.5], bl, False, True, False)
        assert abs(r["log_likelihood"] - ref["lnl"]) / abs(ref["lnl"]) < TOL_API
        assert rel(r["grad_branches"], ref["grad_t"]) < tol
        assert rel(r["grad_omegas"], ref["grad_beta"]) < tol
        assert rel(r["grad_weights"], ref["grad_class_w"]) < tol
        assert rel(r["grad_theta"], ref["grad_theta"]) < tol
        assert rel(r["grad_syn_weights"], ref["grad_rate_w"]) < tol
    # second call with the same model reuses the installed model and gives identical results
    r2 = h3.compute_mixture_gradients(t, a, base, bl, wl.omegas, wl.omega_w, [0.4, 1.6], [0.5, 0.5])
    assert r2["log_likelihood"] == r["log_likelihood"] and r2["grad_branches"] == r["grad_branches"]


def test_autograd_gradients_vs_finite_differences(h3, golden_dir):
    # python/tests/test_python_autograd.py:114-153
    import torch
    from hyphy3.autograd import tree_log_likelihood
    a = h3.Alignment.load(str(golden_dir / "adh.nex"))
    t = h3.Tree.from_newick(a.embedded_tree_newick)
    p = h3.MG94Parameters()
    p.alpha, p.beta = 1.0, 0.4
    init = [0.05 if i != t.root_id else 0.0 for i in range(t.num_nodes())]
    bl = torch.tensor(init, dtype=torch.float64, requires_grad=True)
    ll = tree_log_likelihood(bl, t, a, p)
    assert torch.isfinite(ll)
    ll.backward()
    ana = bl.grad.clone()
    eps = 1e-6
    for nid in range(t.num_nodes()):
        if nid == t.root_id:
            continue
        bp, bm = list(init), list(init)
        bp[nid] += eps
        bm[nid] -= eps
        num = (h3.compute_branch_length_gradients(t, a, p, bp)[0] - h3.compute_branch_length_gradients(t, a, p, bm)[0]) / (2 * eps)
        assert abs(ana[nid].item() - num) / max(abs(ana[nid].item()), abs(num), 1e-4) < 1e-5


def test_adam_branch_optimization_improves(h3, golden_dir):
    # python/tests/test_python_autograd.py:155-182
    import torch
    from hyphy3.autograd import tree_log_likelihood
    a = h3.Alignment.load(str(golden_dir / "adh.nex"))
    t = h3.Tree.from_newick(a.embedded_tree_newick)
    p = h3.MG94Parameters()
    p.alpha, p.beta = 1.0, 0.5
    init = [0.05 if i != t.root_id else 0.0 for i in range(t.num_nodes())]
    log_t = torch.tensor([math.log(max(x, 1e-6)) for x in init], dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([log_t], lr=0.05)
    l0 = tree_log_likelihood(torch.exp(log_t), t, a, p).item()
    for _ in range(5):
        opt.zero_grad()
        loss = -tree_log_likelihood(torch.exp(log_t), t, a, p)
        loss.backward()
        with torch.no_grad():
            log_t.grad[t.root_id] = 0.0
        opt.step()
    assert tree_log_likelihood(torch.exp(log_t), t, a, p).item() > l0 + 50.0


def test_mixture_autograd_function(h3):
    import torch
    from hyphy3.autograd import mixture_log_likelihood
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=120, n_taxa=16)
    a = h3.Alignment.from_sequences(wl.names, wl.seqs)
    t = h3.Tree.from_newick(wl.newick)
    bl = torch.tensor(t.get_branch_lengths(), dtype=torch.float64, requires_grad=True)
    om = torch.tensor(wl.omegas, dtype=torch.float64, requires_grad=True)
    w = torch.tensor(wl.omega_w, dtype=torch.float64, requires_grad=True)
    th = torch.tensor(wl.theta, dtype=torch.float64, requires_grad=True)
    ll = mixture_log_likelihood(bl, om, w, th, t, a)
    ll.backward()
    eps = 1e-6
    for k in range(3):
        op, omn = wl.omegas.copy(), wl.omegas.copy()
        op[k] += eps
        omn[k] -= eps
        fp = mixture_log_likelihood(bl.detach(), torch.tensor(op, dtype=torch.float64), w.detach(), th.detach(), t, a).item()
        fm = mixture_log_likelihood(bl.detach(), torch.tensor(omn, dtype=torch.float64), w.detach(), th.detach(), t, a).item()
        assert abs(om.grad[k].item() - (fp - fm) / (2 * eps)) / (1 + abs(om.grad[k].item())) < 1e-5
