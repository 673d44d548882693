"""The bounded-wait error path of the mixed-precision persistent passes, on one GPU.

Every device wait is bounded; when one expires the kernel records it and finishes, and
the evaluation reports H3G_ERR_TIMEOUT instead of hanging.  Here the waits on other
items' flags look for a value that no item ever publishes (h3g_problem_set_wait_limit
with `unmatched`), with a limit of one poll, so every such wait expires at once: no
fault, no hang.  The same problem then evaluates normally and reproduces the result it
gave before, bit for bit.
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, eigensystems, problem_from_oracle

pytestmark = pytest.mark.gpu


def test_expired_flag_wait_reports_timeout_and_recovers(oracle):
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=300, n_taxa=32)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    models = [{"alpha": 1.0, "beta": om, "theta": list(wl.theta)} for om in wl.omegas]
    Q, lam, U, V, mu = eigensystems(oracle, a, models)
    dirs = np.zeros((1, len(models), 61, 61))
    dirs[0, 0] = dq_beta(a, models[0])
    ctx = _capi.Context(0)
    pr = problem_from_oracle(ctx, oracle, t, a)
    pr.set_model(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=list(wl.omega_w), dQ=dirs,
                 precision=_capi.PREC_MIXED)
    want = _capi.WANT_LNL | _capi.WANT_SITE_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL
    bl = np.array(t.branch_lengths)
    ref = {k: np.copy(v) if isinstance(v, np.ndarray) else v for k, v in pr.eval(bl, want).items()}

    pr.set_wait_limit(polls=1, unmatched=True)
    with pytest.raises(_capi.H3GError) as exc:
        pr.eval(bl, want)
    assert exc.value.status == _capi.H3G_ERR_TIMEOUT
    # device-resident form: the timeout surfaces when the result is read
    pr.stage_branch_lengths(bl)
    pr.eval_resident(want)
    with pytest.raises(_capi.H3GError) as exc:
        pr.read_result(want)
    assert exc.value.status == _capi.H3G_ERR_TIMEOUT

    pr.set_wait_limit(polls=0, unmatched=False)
    out = pr.eval(bl, want)
    assert out["lnl"] == ref["lnl"]
    for k in ("site_lnl", "grad_t", "grad_dir", "grad_class_w"):
        assert np.array_equal(out[k], ref[k]), k
    pr.close()
    ctx.close()
