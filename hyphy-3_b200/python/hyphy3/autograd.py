"""PyTorch autograd integration (python/hyphy3/autograd.py:19-53 of the reference).

PhylogeneticTreeLogLikelihood keeps the reference's signature
apply(branch_lengths, tree, aln, params): forward runs the device
inside-outside pass (lnL and dlnL/dt for every branch in one evaluation),
backward scales the cached gradient by grad_output.  MixtureTreeLogLikelihood
adds the BUSTED-style mixture with gradients for the branch lengths, omega
classes, mixture weights and the five nucleotide exchangeabilities.
"""
import torch

import _hyphy3


class PhylogeneticTreeLogLikelihood(torch.autograd.Function):
    """Differentiable MG94 log-likelihood ln L(t); backward uses the analytic adjoint gradient."""

    @staticmethod
    def forward(ctx, branch_lengths, tree, aln, params):
        bl_list = branch_lengths.detach().cpu().tolist()
        ll, grads = _hyphy3.compute_branch_length_gradients(tree, aln, params, bl_list)
        ctx.grads = torch.tensor(grads, dtype=branch_lengths.dtype, device=branch_lengths.device)
        return torch.tensor(ll, dtype=branch_lengths.dtype, device=branch_lengths.device)

    @staticmethod
    def backward(ctx, grad_output):
        return grad_output * ctx.grads, None, None, None


def tree_log_likelihood(branch_lengths, tree, aln, params=None):
    """Convenience wrapper returning a differentiable scalar tensor."""
    if params is None:
        params = _hyphy3.MG94Parameters()
    return PhylogeneticTreeLogLikelihood.apply(branch_lengths, tree, aln, params)


class MixtureTreeLogLikelihood(torch.autograd.Function):
    """BUSTED-style omega mixture: differentiable in branch lengths, omegas, weights and thetas."""

    @staticmethod
    def forward(ctx, branch_lengths, omegas, weights, thetas, tree, aln, syn_rates=None, syn_weights=None,
                is_test_branch=None, omega_bg=-1.0):
        base = _hyphy3.MG94Parameters()
        th = thetas.detach().cpu().tolist()
        base.theta_AC, base.theta_AT, base.theta_CG, base.theta_CT, base.theta_GT = th
        r = _hyphy3.compute_mixture_gradients(
            tree, aln, base, branch_lengths.detach().cpu().tolist(), omegas.detach().cpu().tolist(),
            weights.detach().cpu().tolist(), syn_rates or [1.0], syn_weights or [1.0], is_test_branch, omega_bg)
        kw = dict(dtype=branch_lengths.dtype, device=branch_lengths.device)
        ctx.g = (torch.tensor(r["grad_branches"], **kw), torch.tensor(r["grad_omegas"], **kw),
                 torch.tensor(r["grad_weights"], **kw), torch.tensor(r["grad_theta"], **kw))
        return torch.tensor(r["log_likelihood"], **kw)

    @staticmethod
    def backward(ctx, grad_output):
        gb, go, gw, gt = ctx.g
        return (grad_output * gb, grad_output * go, grad_output * gw, grad_output * gt,
                None, None, None, None, None, None)


def mixture_log_likelihood(branch_lengths, omegas, weights, thetas, tree, aln, **kw):
    return MixtureTreeLogLikelihood.apply(branch_lengths, omegas, weights, thetas, tree, aln,
                                          kw.get("syn_rates"), kw.get("syn_weights"), kw.get("is_test_branch"),
                                          kw.get("omega_bg", -1.0))
