"""The oracle's per-branch omega distributions (aBSREL's branch-site mixtures), CPU only.

Branch b mixes its own classes: P_b = sum_k w_k P(omega_k, t_b) over k in [bc[b], bc[b+1])
(absrel.hpp:262-276).  The likelihood equals the pruning of those mixed matrices built
explicitly (loglik_from_P), and the class-weight and omega gradients equal central
differences of the likelihood.
"""
import numpy as np


def _setup(oracle):
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=60, n_taxa=8)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    rng = np.random.default_rng(5)
    n = t.num_nodes()
    counts = [0 if b == t.root else int(rng.integers(1, 4)) for b in range(n)]
    bc = np.concatenate([[0], np.cumsum(counts)]).astype(int).tolist()
    K = bc[-1]
    omegas = list(rng.uniform(0.05, 3.0, size=K))
    w = []
    for b in range(n):
        x = rng.dirichlet(np.ones(counts[b])) if counts[b] else []
        w.extend(list(x))
    return wl, t, a, bc, omegas, w


def _eval(oracle, wl, t, a, bc, omegas, w):
    cls = [{"alpha": 1.0, "beta": o, "theta": list(wl.theta)} for o in omegas]
    return oracle.mixture_eval(t, a, cls, w, None, [], [], [], list(t.branch_lengths), False, True, False, False, bc)


def test_branch_class_likelihood_equals_explicit_mixtures(oracle):
    wl, t, a, bc, omegas, w = _setup(oracle)
    r = _eval(oracle, wl, t, a, bc, omegas, w)
    Ps = []
    for b in range(t.num_nodes()):
        if b == t.root:
            Ps.append(np.eye(61))
            continue
        P = np.zeros((61, 61))
        for k in range(bc[b], bc[b + 1]):
            P += w[k] * np.asarray(oracle.transition_matrix(a, {"alpha": 1.0, "beta": omegas[k], "theta": list(wl.theta)},
                                                            t.branch_lengths[b]))
        Ps.append(P)
    ref = oracle.loglik_from_P(t, a, Ps, np.asarray(a.pi))[0]
    assert abs(r["lnl"] - ref) <= 1e-12 * abs(ref)


def test_branch_class_gradients_vs_finite_differences(oracle):
    wl, t, a, bc, omegas, w = _setup(oracle)
    r = _eval(oracle, wl, t, a, bc, omegas, w)
    h = 1e-6
    for k in range(0, len(omegas), 3):
        wp, wm = list(w), list(w)
        wp[k] += h
        wm[k] -= h
        fd = (_eval(oracle, wl, t, a, bc, omegas, wp)["lnl"] - _eval(oracle, wl, t, a, bc, omegas, wm)["lnl"]) / (2 * h)
        assert abs(r["grad_class_w"][k] - fd) < 1e-5 * (1 + abs(fd)), k
        op, om = list(omegas), list(omegas)
        op[k] += h
        om[k] -= h
        fd = (_eval(oracle, wl, t, a, bc, op, w)["lnl"] - _eval(oracle, wl, t, a, bc, om, w)["lnl"]) / (2 * h)
        assert abs(r["grad_beta"][k] - fd) < 1e-5 * (1 + abs(fd)), k
