"""How far apart two correct FP64 eigensolvers put the likelihood (CPU only).

The library's host model (include/hyphy/core/h3_host.hpp, MG94Matrix: Householder
tridiagonalisation + implicit QL) and the oracle (cyclic Jacobi) both diagonalise the
symmetrised generator D^1/2 Q D^-1/2 (rate_matrix.hpp:236-249), as the reference does with
Eigen's SelfAdjointEigenSolver.  Their eigenvectors differ at rounding level; the
back-transformation by sqrt(pi_j / pi_i) magnifies that in the rows of rare codons
(pi down to 1e-10 on cd2_reduced).  This pins the resulting floor: transition matrices
within 1e-10 absolute and log-likelihoods within 1e-11 relative, so comparing the public
API (host eigensolver) with the oracle at the 1e-10 bound of the FP64 path is sound.
"""
import numpy as np
import pytest


def _P(e, t):
    U, V, lam = np.asarray(e["U"]), np.asarray(e["V"]), np.asarray(e["lam"])
    return np.maximum((U * np.exp(lam * t)) @ V, 0.0)


def _cases(oracle, golden_dir, known):
    import _hyphy3 as h
    from hyphy3.simulate import make_workload
    k = known["cd2_reduced"]
    yield ("cd2_reduced", h.Alignment.load(str(golden_dir / "cd2_reduced.fna")),
           oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna")), k["newick"], 0.45, [0.8, 1.2, 0.6, 1.8, 0.9], None)
    b = oracle.Alignment.load(str(golden_dir / "adh.nex"))
    yield ("adh", h.Alignment.load(str(golden_dir / "adh.nex")), b, b.embedded_tree, 0.4, [1, 1, 1, 1, 1], 0.05)
    wl = make_workload(1, n_sites=300)
    yield ("busted64", h.Alignment.from_sequences(wl.names, wl.seqs), oracle.Alignment.from_sequences(wl.names, wl.seqs),
           wl.newick, 0.5, list(wl.theta), None)


def test_host_and_oracle_eigensystems_agree_on_P_and_lnL(oracle, golden_dir, known):
    import _hyphy3 as h
    for name, ah, ao, newick, beta, theta, t_fixed in _cases(oracle, golden_dir, known):
        p = h.MG94Parameters()
        p.beta = beta
        p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = theta
        eh = h.mg94_eigensystem(ah, p)
        eo = oracle.mg94(ao, {"alpha": 1.0, "beta": beta, "theta": theta})
        assert np.max(np.abs(np.asarray(eh["Q"]) - np.asarray(eo["Q"]))) < 1e-14, name
        assert np.max(np.abs(np.sort(np.asarray(eh["lam"])) - np.sort(np.asarray(eo["lam"])))) < 1e-12, name
        t = oracle.Tree.parse(newick)
        bl = [0.0 if i == t.root else (t_fixed if t_fixed else max(1e-4, x)) for i, x in enumerate(t.branch_lengths)]
        Ph = [np.eye(61) if i == t.root else _P(eh, bl[i]) for i in range(t.num_nodes())]
        Po = [np.eye(61) if i == t.root else _P(eo, bl[i]) for i in range(t.num_nodes())]
        dP = max(float(np.max(np.abs(x - y))) for x, y in zip(Ph, Po))
        assert dP < 1e-10, (name, dP)
        pi = np.asarray(ao.pi)
        lh = oracle.loglik_from_P(t, ao, Ph, pi)[0]
        lo = oracle.loglik_from_P(t, ao, Po, pi)[0]
        assert abs(lh - lo) / abs(lo) < 1e-11, (name, lh, lo)


def _eig(h, aln, beta, theta):
    p = h.MG94Parameters()
    p.beta = beta
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = theta
    e = h.mg94_eigensystem(aln, p)
    return {"U": np.asarray(e["U"]), "V": np.asarray(e["V"]), "lam": np.asarray(e["lam"])}


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def test_gradient_floor_between_eigensolvers(oracle, golden_dir, known):
    """The oracle with the host's eigensystem against the oracle with its own: branch, omega and
    exchangeability gradients agree within 5e-10 of max(1, |g|max) (the bound the API tests use
    against the oracle's own eigensystem)."""
    import _hyphy3 as h
    ah = h.Alignment.load(str(golden_dir / "adh.nex"))
    ao = oracle.Alignment.load(str(golden_dir / "adh.nex"))
    t = oracle.Tree.parse(ao.embedded_tree)
    bl = [0.0 if i == t.root else 0.05 for i in range(t.num_nodes())]
    own = oracle.branch_length_gradients(t, ao, {"alpha": 1.0, "beta": 0.4}, bl)
    given = oracle.branch_length_gradients(t, ao, {"alpha": 1.0, "beta": 0.4, "eig": _eig(h, ah, 0.4, [1] * 5)}, bl)
    assert abs(own[0] - given[0]) / abs(own[0]) < 1e-11
    assert _rel(given[1], own[1]) < 5e-10
    k = known["cd2_reduced"]
    ah = h.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    ao = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = oracle.Tree.parse(k["newick"])
    th = [0.8, 1.2, 0.6, 1.8, 0.9]
    bl = [0.0 if i == t.root else max(1e-4, x) for i, x in enumerate(t.branch_lengths)]
    own = oracle.joint_frechet_gradients(t, ao, {"alpha": 1.0, "beta": 0.45, "theta": th}, bl)
    given = oracle.joint_frechet_gradients(t, ao, {"alpha": 1.0, "beta": 0.45, "theta": th, "eig": _eig(h, ah, 0.45, th)}, bl)
    assert abs(own["lnl"] - given["lnl"]) / abs(own["lnl"]) < 1e-11
    for key in ("grad_t", "grad_beta", "grad_theta"):
        assert _rel(given[key], own[key]) < 5e-10, key
