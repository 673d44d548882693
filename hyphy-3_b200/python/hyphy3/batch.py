"""Joint fits over batches of independent genes (hyphy3._capi.Batch, h3g_batch_*).

The reference fits each gene's branch lengths on its own (MG94Fitter::fit_full_model,
optimizer.hpp:909-1135, L-BFGS-B in log space over every branch length with the gene's
likelihood and analytic gradient).  Here all genes of a batch are fitted at once: one
bounded L-BFGS over the log branch lengths of every gene, the objective the summed
log-likelihood, each objective and gradient one batch evaluation -- one CUDA-graph launch
that evaluates every gene.  The genes share no parameter, so the joint optimum is every
gene's own optimum; the joint form keeps the whole batch in flight on the device.
"""
from __future__ import annotations

import numpy as np

from . import _capi


def fit_branch_lengths(batch: "_capi.Batch", start, *, max_iter: int = 200, tol: float = 1e-9,
                       bounds: tuple[float, float] = (1e-8, 1e4)) -> dict:
    """Maximise sum_g lnL_g over every gene's branch lengths (log scale, within `bounds`).

    start: one branch-length vector per gene (one entry per node; root entries ignored).
    Returns the summed and per-gene log-likelihoods, the fitted branch lengths, and the
    optimiser's iteration and evaluation counts."""
    from scipy.optimize import minimize

    probs = batch.problems
    idx = [np.flatnonzero(np.asarray(p.parent) >= 0) for p in probs]
    offs = np.cumsum([0] + [len(i) for i in idx])
    lo, hi = np.log(bounds[0]), np.log(bounds[1])
    x0 = np.concatenate([np.clip(np.log(np.maximum(np.asarray(b, dtype=float)[i], bounds[0])), lo, hi)
                         for b, i in zip(start, idx)])
    want = _capi.WANT_LNL | _capi.WANT_GRAD_T

    def unpack(x):
        out = []
        for g, p in enumerate(probs):
            bl = np.zeros(p.n)
            bl[idx[g]] = np.exp(x[offs[g]:offs[g + 1]])
            out.append(bl)
        return out

    def objective(x):
        bls = unpack(x)
        res = batch.eval(bls, want)
        val = -sum(r["lnl"] for r in res)
        grad = -np.concatenate([r["grad_t"][idx[g]] * bls[g][idx[g]] for g, r in enumerate(res)])
        return val, grad

    opt = minimize(objective, x0, jac=True, method="L-BFGS-B", bounds=[(lo, hi)] * len(x0),
                   options={"maxiter": max_iter, "ftol": tol, "gtol": 1e-6})
    bls = unpack(opt.x)
    res = batch.eval(bls, _capi.WANT_LNL)
    per_gene = [r["lnl"] for r in res]
    return {"log_likelihood": float(sum(per_gene)), "per_gene": per_gene, "branch_lengths": bls,
            "iterations": int(opt.nit), "evaluations": int(opt.nfev), "converged": bool(opt.success)}
