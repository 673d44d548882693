"""Subtree checkpointing on the device: a memory budget below the full workspace cuts the tree into
blocks whose inside partials the outside pass recomputes (h3g_checkpoint.h).  The checkpointed
evaluation runs the same kernels in the same summation order, so every result must be
bit-identical to the unbudgeted one: lnL, per-site lnL and every gradient, FP64 and mixed, on the
1024-taxon x 5000-codon workload (4 rate passes) and, with forced block sizes down to 2, on the
64-taxon workload.
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, dq_theta

pytestmark = pytest.mark.gpu
WANT_ALL = 1 | 2 | 4 | 8


@pytest.fixture(scope="module")
def ctx():
    from hyphy3 import _capi
    c = _capi.Context(0)
    yield c
    c.close()


def _problem(ctx, oracle, config):
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    wl = make_workload(config)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    models = [{"alpha": 1.0, "beta": om, "theta": list(wl.theta)} for om in wl.omegas]
    nm = len(models)
    Q = np.stack([np.asarray(oracle.mg94(a, m)["Q"]) for m in models])
    dirs = []
    for k in range(nm):
        d = np.zeros((nm, 61, 61))
        d[k] = dq_beta(a, models[k])
        dirs.append(d)
    for x in range(5):
        dirs.append(np.stack([dq_theta(a, x, m) for m in models]))
    l2t = oracle.leaf_map(t, a)
    n = t.num_nodes()
    leaf = np.array(t.is_leaf, dtype=np.uint8)
    taxon = np.array([l2t[i] if leaf[i] else -1 for i in range(n)], dtype=np.int32)
    pr = _capi.Problem(ctx, np.array(t.parent, dtype=np.int32), leaf, taxon, a.states, a.masks, np.array(a.weights, dtype=float))
    args = dict(pi=a.pi, Q=Q, class_w=list(wl.omega_w), rates=list(wl.rates), rate_w=list(wl.rate_w), dQ=np.stack(dirs))
    return pr, args, np.array(t.branch_lengths)


def _same(a, b):
    assert a["lnl"] == b["lnl"]
    for k in ("site_lnl", "grad_t", "grad_dir", "grad_class_w", "grad_rate_w"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_yule1024_budget_is_bit_identical(ctx, oracle, precision):
    from hyphy3 import _capi
    pr, args, bl = _problem(ctx, oracle, 3)
    prec = _capi.PREC_MIXED if precision == "mixed" else _capi.PREC_FP64
    pr.set_model(precision=prec, **args)
    info0 = pr.checkpoint_info()
    assert info0["active"] == 0 and info0["workspace_bytes"] == info0["full_bytes"]
    full = pr.eval(bl, WANT_ALL)
    budget = info0["full_bytes"] // 6
    pr.set_memory_budget(budget)
    info = pr.checkpoint_info()
    assert info["active"] == 1 and info["workspace_bytes"] <= budget
    assert info["n_blocks"] > 1 and info["n_persistent"] == info["n_blocks"]
    ck = pr.eval(bl, WANT_ALL)
    _same(full, ck)
    # repeated and value-only evaluations on the checkpointed workspace
    _same(full, pr.eval(bl, WANT_ALL))
    assert pr.eval(bl, 1)["lnl"] == full["lnl"]
    # lifting the budget restores the full workspace
    pr.set_memory_budget(0)
    assert pr.checkpoint_info()["active"] == 0
    _same(full, pr.eval(bl, WANT_ALL))
    pr.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_busted64_forced_block_sizes(ctx, oracle, precision):
    from hyphy3 import _capi
    pr, args, bl = _problem(ctx, oracle, 1)
    pr.set_model(precision=_capi.PREC_MIXED if precision == "mixed" else _capi.PREC_FP64, **args)
    full = pr.eval(bl, WANT_ALL)
    for target in (2, 3, 9, 40):
        pr.set_memory_budget(0, target)
        info = pr.checkpoint_info()
        assert info["active"] == 1 and info["target"] == target
        _same(full, pr.eval(bl, WANT_ALL))
    pr.close()


def test_budget_too_small_is_an_error(ctx, oracle):
    from hyphy3 import _capi
    pr, args, bl = _problem(ctx, oracle, 1)
    pr.set_model(precision=_capi.PREC_FP64, **args)
    with pytest.raises(_capi.H3GError):
        pr.set_memory_budget(1 << 20)
    pr.set_memory_budget(0)
    assert np.isfinite(pr.eval(bl, 1)["lnl"])
    pr.close()


def test_api_memory_budget_is_bit_identical(ctx, oracle):
    """_hyphy3.set_memory_budget applies to the problems the engine creates: same results."""
    import _hyphy3 as h
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    wl = make_workload(1)
    pr, args, _ = _problem(ctx, oracle, 1)
    pr.set_model(precision=0, **args)
    full_bytes = pr.checkpoint_info()["full_bytes"]
    # at 64 taxa the matrices are a large fixed part of the workspace: the smallest fraction that a
    # plan meets
    budget = None
    for frac in (0.6, 0.7, 0.8, 0.9):
        try:
            pr.set_memory_budget(int(full_bytes * frac))
        except _capi.H3GError:
            continue
        if pr.checkpoint_info()["active"]:
            budget = int(full_bytes * frac)
            break
    assert budget is not None
    pr.close()
    tree = h.Tree.from_newick(wl.newick)
    aln = h.Alignment.from_sequences(wl.names, wl.seqs)
    base = h.MG94Parameters()
    base.theta_AC, base.theta_AT, base.theta_CG, base.theta_CT, base.theta_GT = wl.theta
    bl = list(tree.get_branch_lengths())
    call = (tree, aln, base, bl, list(wl.omegas), list(wl.omega_w), list(wl.rates), list(wl.rate_w))
    h.set_precision("fp64")
    ref = h.compute_mixture_gradients(*call)
    try:
        h.set_memory_budget(budget)
        assert h.get_memory_budget() == budget
        got = h.compute_mixture_gradients(*call)
    finally:
        h.set_memory_budget(0)
    assert got["log_likelihood"] == ref["log_likelihood"]
    for k in ("grad_branches", "grad_omegas", "grad_theta", "grad_weights", "site_log_likelihoods"):
        assert np.array_equal(np.asarray(got[k]), np.asarray(ref[k])), k


def test_first_evaluation_after_each_reallocation(ctx, oracle):
    """A new workspace is zeroed on the evaluations' stream before its first evaluation: ten
    reallocations (alternating A-accumulation chunks and checkpoint block sizes), each followed at
    once by a mixed evaluation, raise no expired wait, and that first evaluation equals the next one
    on the same workspace bit for bit.  Zeroing on the default stream instead raced with the first
    evaluation's published flags and, now and then, left a wait to expire."""
    from hyphy3 import _capi
    pr, args, bl = _problem(ctx, oracle, 1)
    pr.set_model(precision=_capi.PREC_MIXED, **args)
    ref = pr.eval(bl, WANT_ALL)
    for i in range(10):
        if i % 2:
            pr.set_memory_budget(0, 9 if i % 4 == 1 else 0)
        else:
            pr.set_tuning(a_chunk=256 if i % 4 == 0 else 512)
        first = pr.eval(bl, WANT_ALL)
        _same(first, pr.eval(bl, WANT_ALL))
        assert abs(first["lnl"] - ref["lnl"]) <= 1e-12 * abs(ref["lnl"])
    pr.close()
