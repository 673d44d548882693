"""The benchmark workloads at their full sizes: device vs the CPU oracle through the C ABI.

* 64 taxa x 1000 codons (3 % gaps, 1 % ambiguous codons), omega classes {0.1, 1, 5} mixed
  at the P level: the whole alignment.
* 1024-taxon Yule tree x 5000 codons, omegas {0.2, 2} x 4 discrete-gamma synonymous-rate
  passes: the device evaluates every pattern with the weights of all but a seeded subset of
  256 set to 0; the oracle evaluates that subset alone.  Every term of lnL and of each
  gradient is a weighted sum over patterns, so both sides compute the same quantity.

Tolerances: FP64 1e-10 relative (lnL) and 1e-10 of max(1, |g|max) for gradient vectors, on
the oracle's eigensystems; mixed precision 1e-7 (lnL) and 1e-5 (gradients).
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, dq_theta, eigensystems, rel

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-10
TOL_MIXED_LNL = 1e-7
TOL_MIXED_GRAD = 1e-5
SUBSET = 256


@pytest.fixture(scope="module")
def ctx():
    from hyphy3 import _capi
    c = _capi.Context(0)
    yield c
    c.close()


def _directions(a, models):
    nm = len(models)
    dirs = []
    for k in range(nm):
        d = np.zeros((nm, 61, 61))
        d[k] = dq_beta(a, models[k])
        dirs.append(d)
    for x in range(5):
        dirs.append(np.stack([dq_theta(a, x, m) for m in models]))
    return np.stack(dirs)


def _case(oracle, config, subset):
    from hyphy3.simulate import make_workload
    wl = make_workload(config)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    models = [{"alpha": 1.0, "beta": om, "theta": list(wl.theta)} for om in wl.omegas]
    weights = np.array(a.weights, dtype=float)
    if subset:
        idx = np.sort(np.random.default_rng(20261203 + config).choice(a.num_patterns, subset, replace=False))
        keep = np.zeros_like(weights)
        keep[idx] = weights[idx]
        weights, sub = keep, a.select_patterns([int(i) for i in idx])
    else:
        idx, sub = np.arange(a.num_patterns), a
    rates, rw = (list(wl.rates), list(wl.rate_w)) if len(wl.rates) > 1 else ([], [])
    ref = oracle.mixture_eval(t, sub, models, list(wl.omega_w), None, [], rates, rw, list(t.branch_lengths),
                              False, True, False, True)
    return {"wl": wl, "t": t, "a": a, "models": models, "weights": weights, "idx": idx, "ref": ref,
            "eig": eigensystems(oracle, a, models), "dirs": _directions(a, models)}


@pytest.fixture(scope="module")
def c2(oracle):
    return _case(oracle, 1, 0)


@pytest.fixture(scope="module")
def c4(oracle):
    return _case(oracle, 3, SUBSET)


def _device(ctx, oracle, case, precision):
    from hyphy3 import _capi
    t, a, wl = case["t"], case["a"], case["wl"]
    l2t = oracle.leaf_map(t, a)
    n = t.num_nodes()
    leaf = np.array(t.is_leaf, dtype=np.uint8)
    taxon = np.array([l2t[i] if leaf[i] else -1 for i in range(n)], dtype=np.int32)
    pr = _capi.Problem(ctx, np.array(t.parent, dtype=np.int32), leaf, taxon, a.states, a.masks, case["weights"])
    Q, lam, U, V, mu = case["eig"]
    pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=list(wl.omega_w), rates=list(wl.rates),
                 rate_w=list(wl.rate_w), dQ=case["dirs"],
                 precision=_capi.PREC_MIXED if precision == "mixed" else _capi.PREC_FP64)
    out = pr.eval(np.array(t.branch_lengths), _capi.WANT_LNL | _capi.WANT_SITE_LNL | _capi.WANT_GRAD_T |
                  _capi.WANT_GRAD_GLOBAL)
    pr.close()
    return out


def _check(out, case, tol_lnl, tol_grad):
    ref = case["ref"]
    K = len(case["models"])
    assert abs(out["lnl"] - ref["lnl"]) / abs(ref["lnl"]) < tol_lnl
    site = np.asarray(out["site_lnl"])[case["idx"]]
    assert rel(site, ref["site_lnl"]) < tol_lnl * 10
    assert rel(out["grad_t"], ref["grad_t"]) < tol_grad
    assert rel(out["grad_dir"][:K], ref["grad_beta"]) < tol_grad
    assert rel(out["grad_dir"][K:K + 5], ref["grad_theta"]) < tol_grad
    assert rel(out["grad_class_w"], ref["grad_class_w"]) < tol_grad
    if len(case["wl"].rates) > 1:
        assert rel(out["grad_rate_w"], ref["grad_rate_w"]) < tol_grad


def test_busted64_full_fp64(ctx, oracle, c2):
    _check(_device(ctx, oracle, c2, "fp64"), c2, TOL_FP64, TOL_FP64)


def test_busted64_full_mixed(ctx, oracle, c2):
    _check(_device(ctx, oracle, c2, "mixed"), c2, TOL_MIXED_LNL, TOL_MIXED_GRAD)


def test_yule1024_subset_fp64(ctx, oracle, c4):
    _check(_device(ctx, oracle, c4, "fp64"), c4, TOL_FP64, TOL_FP64)


def test_yule1024_subset_mixed(ctx, oracle, c4):
    _check(_device(ctx, oracle, c4, "mixed"), c4, TOL_MIXED_LNL, TOL_MIXED_GRAD)
