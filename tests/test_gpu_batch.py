"""Batches of independent genes (h3g_batch_*) against one-at-a-time evaluation and the oracle.

Genes of uneven taxon count and length, each with its own tree and MG94xREV parameters, are
evaluated by one graph launch over a few slot workspaces; every gene's lnL, per-site values and
gradients must equal the same gene evaluated alone (bit for bit: the same kernels on the same
inputs), and the FP64 results must match the oracle at 1e-10.  A joint L-BFGS over all genes'
branch lengths, driven by batch evaluations, must raise every gene's likelihood.
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, eigensystems, problem_from_oracle, rel

pytestmark = pytest.mark.gpu


def _genes(oracle, count, seed=7):
    from hyphy3.simulate import random_unrooted_tree, simulate_alignment
    rng = np.random.default_rng(seed)
    out = []
    for g in range(count):
        nt = int(rng.integers(6, 40))
        ns = int(rng.integers(40, 260))
        theta = list(rng.uniform(0.5, 2.0, size=5))
        tree = random_unrooted_tree(nt, rng, 0.1)
        omega = float(rng.uniform(0.1, 1.5))
        names, seqs = simulate_alignment(tree, ns, rng, theta=theta, pos_freq=rng.dirichlet(np.ones(4), size=3),
                                         omegas=[omega], gap_frac=0.02, ambig_frac=0.01)
        t = oracle.Tree.parse(tree.newick())
        a = oracle.Alignment.from_sequences(names, seqs)
        out.append({"t": t, "a": a, "p": {"alpha": 1.0, "beta": omega, "theta": theta}})
    return out


def _install(ctx, oracle, gene, precision):
    from hyphy3 import _capi
    pr = problem_from_oracle(ctx, oracle, gene["t"], gene["a"])
    Q, lam, U, V, mu = eigensystems(oracle, gene["a"], [gene["p"]])
    dirs = dq_beta(gene["a"], gene["p"])[None, None]
    pr.set_model(pi=gene["a"].pi, Q=Q, lam=lam, U=U, V=V, mu=mu, dQ=dirs, precision=precision)
    return pr


@pytest.mark.parametrize("precision_name", ["fp64", "mixed"])
def test_batch_equals_single_problem_evaluations(oracle, precision_name):
    from hyphy3 import _capi
    prec = _capi.PREC_FP64 if precision_name == "fp64" else _capi.PREC_MIXED
    genes = _genes(oracle, 20)
    want = _capi.WANT_LNL | _capi.WANT_SITE_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL
    ctx = _capi.Context(0)
    bls = [np.array(g["t"].branch_lengths) for g in genes]
    single = []
    for g, bl in zip(genes, bls):
        pr = _install(ctx, oracle, g, prec)
        single.append({k: np.copy(v) if isinstance(v, np.ndarray) else v for k, v in pr.eval(bl, want).items()})
        pr.close()
    probs = [_install(ctx, oracle, g, prec) for g in genes]
    batch = _capi.Batch(ctx, probs, n_slots=4)
    for rep in range(2):                          # the second call replays the captured graph
        outs = batch.eval(bls, want)
        for g, (o, s) in enumerate(zip(outs, single)):
            assert o["lnl"] == s["lnl"], (rep, g)
            for k in ("site_lnl", "grad_t", "grad_dir"):
                assert np.array_equal(o[k], s[k]), (rep, g, k)
    ms, launches = batch.last_stats()
    assert ms > 0 and launches >= len(genes)
    # a gene of the batch cannot be evaluated alone while the batch lives
    with pytest.raises(_capi.H3GError) as exc:
        probs[0].eval(bls[0], want)
    assert exc.value.status == _capi.H3G_ERR_STATE
    if precision_name == "fp64":
        for g, o in zip(genes, outs):
            ref = oracle.mixture_eval(g["t"], g["a"], [g["p"]], [1.0], None, [], [], [], list(g["t"].branch_lengths),
                                      False, True, False)
            assert abs(o["lnl"] - ref["lnl"]) / abs(ref["lnl"]) < 1e-10
            assert rel(o["grad_t"], ref["grad_t"]) < 1e-10
            assert rel(o["grad_dir"][:1], ref["grad_beta"]) < 1e-10
    batch.close()
    # after the batch the problems work alone again once their model is reinstalled
    pr = probs[0]
    Q, lam, U, V, mu = eigensystems(oracle, genes[0]["a"], [genes[0]["p"]])
    pr.set_model(pi=genes[0]["a"].pi, Q=Q, lam=lam, U=U, V=V, mu=mu, dQ=dq_beta(genes[0]["a"], genes[0]["p"])[None, None],
                 precision=prec)
    assert pr.eval(bls[0], want)["lnl"] == single[0]["lnl"]
    ctx.close()


def test_joint_branch_length_fit_over_a_batch(oracle):
    from hyphy3 import _capi
    from hyphy3.batch import fit_branch_lengths
    genes = _genes(oracle, 12, seed=11)
    ctx = _capi.Context(0)
    probs = [_install(ctx, oracle, g, _capi.PREC_FP64) for g in genes]
    batch = _capi.Batch(ctx, probs, n_slots=3)
    start = [np.where(np.array(g["t"].parent) < 0, 0.0, 0.1) for g in genes]
    l0 = [o["lnl"] for o in batch.eval(start, _capi.WANT_LNL)]
    fit = fit_branch_lengths(batch, start, max_iter=60)
    assert fit["log_likelihood"] > sum(l0) + 1.0
    for g, (bl, lnl) in enumerate(zip(fit["branch_lengths"], fit["per_gene"])):
        assert lnl >= l0[g] - 1e-6
        ref = oracle.branch_length_gradients(genes[g]["t"], genes[g]["a"], genes[g]["p"], list(bl))
        assert abs(ref[0] - lnl) / abs(lnl) < 1e-10
    ctx.close()
