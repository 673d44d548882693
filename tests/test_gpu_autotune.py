"""The launch-shape autotuner (h3g_autotune) and explicit tunings.

A tuning changes only launch shapes (A-accumulation pattern chunk, persistent CTAs per SM,
Frechet branch groups): results must stay within rounding of the untuned evaluation and, in
FP64, within 1e-10 of the oracle.  The tuner's choice is recorded for the problem's shape: a
second problem of the same shape starts from it.
"""
import numpy as np
import pytest

from gpu_helpers import dq_beta, eigensystems, problem_from_oracle, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision_name", ["fp64", "mixed"])
def test_autotune_keeps_results_and_records_the_choice(oracle, precision_name):
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    prec = _capi.PREC_FP64 if precision_name == "fp64" else _capi.PREC_MIXED
    wl = make_workload(1, n_sites=600, n_taxa=40)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    models = [{"alpha": 1.0, "beta": om, "theta": list(wl.theta)} for om in wl.omegas]
    Q, lam, U, V, mu = eigensystems(oracle, a, models)
    dirs = np.stack([np.stack([dq_beta(a, m) if j == k else np.zeros((61, 61)) for j, m in enumerate(models)])
                     for k in range(len(models))])
    kw = dict(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=list(wl.omega_w), dQ=dirs, precision=prec)
    want = _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL
    bl = np.array(t.branch_lengths)
    ctx = _capi.Context(0)
    pr = problem_from_oracle(ctx, oracle, t, a)
    pr.set_model(**kw)
    base = {k: np.copy(v) if isinstance(v, np.ndarray) else v for k, v in pr.eval(bl, want).items()}
    best, ms = pr.autotune(bl, want, reps=2)
    assert ms > 0 and best["a_chunk"] % 128 == 0 and best["ctas_per_sm"] in (1, 2) and best["frechet_groups"] >= 1
    assert pr.get_tuning() == best
    tuned = pr.eval(bl, want)
    # lnL does not depend on the launch shapes; the gradients' A sums are regrouped: rounding of FP64
    # partial sums (FP64 path), FP32 accumulator groups (mixed path, well inside its 1e-5 bound)
    assert abs(tuned["lnl"] - base["lnl"]) <= 1e-13 * abs(base["lnl"])
    gtol = 1e-11 if precision_name == "fp64" else 1e-6
    assert rel(tuned["grad_t"], base["grad_t"]) < gtol
    assert rel(tuned["grad_dir"], base["grad_dir"]) < gtol
    if precision_name == "fp64":
        ref = oracle.mixture_eval(t, a, models, list(wl.omega_w), None, [], [], [], list(bl), False, True, False)
        assert abs(tuned["lnl"] - ref["lnl"]) / abs(ref["lnl"]) < 1e-10
        assert rel(tuned["grad_t"], ref["grad_t"]) < 1e-10
    # explicit shapes are honoured and validated
    pr.set_tuning(a_chunk=256, ctas_per_sm=1, frechet_groups=3)
    assert pr.get_tuning() == {"a_chunk": 256, "ctas_per_sm": 1, "frechet_groups": 3}
    alt = pr.eval(bl, want)
    assert abs(alt["lnl"] - base["lnl"]) <= 1e-13 * abs(base["lnl"])
    assert rel(alt["grad_t"], base["grad_t"]) < gtol
    with pytest.raises(_capi.H3GError):
        pr.set_tuning(a_chunk=200)
    # a new problem of the same shape starts from the recorded tuning
    pr2 = problem_from_oracle(ctx, oracle, t, a)
    pr2.set_model(**kw)
    assert pr2.get_tuning() == best
    pr2.close()
    pr.close()
    ctx.close()
