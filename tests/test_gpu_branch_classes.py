"""Per-branch omega distributions on the device (h3g_model_desc.branch_classes) vs the oracle.

Every branch mixes its own range of the class table (aBSREL's branch-site models); lnL,
per-site values, branch gradients, every class's weight partial, its omega gradient (one
direction per class) and the exchangeability gradients must match the oracle at 1e-10 (FP64),
and the mixed path at 1e-7 / 1e-5.
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, dq_theta, eigensystems, problem_from_oracle, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision_name", ["fp64", "mixed"])
def test_branch_classes_against_oracle(oracle, precision_name):
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=300, n_taxa=18)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    rng = np.random.default_rng(9)
    n = t.num_nodes()
    counts = [0 if b == t.root else int(rng.integers(1, 4)) for b in range(n)]
    bc = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    K = int(bc[-1])
    omegas = list(rng.uniform(0.05, 3.0, size=K))
    w = np.concatenate([rng.dirichlet(np.ones(c)) if c else np.zeros(0) for c in counts])
    models = [{"alpha": 1.0, "beta": o, "theta": list(wl.theta)} for o in omegas]
    Q, lam, U, V, mu = eigensystems(oracle, a, models)
    dirs = []
    for k in range(K):                       # d/d omega_k touches class k only
        d = np.zeros((K, 61, 61))
        d[k] = dq_beta(a, models[k])
        dirs.append(d)
    for x in (0, 3):                         # two exchangeabilities, every class
        dirs.append(np.stack([dq_theta(a, x, m) for m in models]))
    ctx = _capi.Context(0)
    pr = problem_from_oracle(ctx, oracle, t, a)
    prec = _capi.PREC_FP64 if precision_name == "fp64" else _capi.PREC_MIXED
    pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=w, dQ=np.stack(dirs), precision=prec,
                 branch_classes=bc)
    bl = np.array(t.branch_lengths)
    out = pr.eval(bl, _capi.WANT_LNL | _capi.WANT_SITE_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL)
    ref = oracle.mixture_eval(t, a, models, list(w), None, [], [], [], list(bl), False, True, False, False, bc.tolist())
    tl, tg = (1e-10, 1e-10) if precision_name == "fp64" else (1e-7, 1e-5)
    assert abs(out["lnl"] - ref["lnl"]) / abs(ref["lnl"]) < tl
    assert rel(out["site_lnl"], ref["site_lnl"]) < tl * 10
    assert rel(out["grad_t"], ref["grad_t"]) < tg
    assert rel(out["grad_class_w"], ref["grad_class_w"]) < tg
    assert rel(out["grad_dir"][:K], ref["grad_beta"]) < tg
    assert rel(out["grad_dir"][K:K + 2], [ref["grad_theta"][0], ref["grad_theta"][3]]) < tg
    # the same omega gradients from one per-model direction each (dQ_model) instead of K dense ones
    dense = np.copy(out["grad_dir"])
    pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=w, dQ=np.stack(dirs[K:]), precision=prec,
                 branch_classes=bc, dQ_model=np.stack([dq_beta(a, m) for m in models]))
    out2 = pr.eval(bl, _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL)
    assert out2["lnl"] == out["lnl"]
    assert np.array_equal(out2["grad_dir"][2:2 + K], dense[:K])
    assert np.array_equal(out2["grad_dir"][:2], dense[K:K + 2])
    # malformed ranges are rejected
    bad = bc.copy()
    bad[2] = bad[1]
    with pytest.raises(_capi.H3GError):
        pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=w, precision=prec, branch_classes=bad)
    pr.close()
    ctx.close()
