"""The oracle's two forms of the mixture evaluation agree (CPU only).

`tiled=True` is the reference's batched shape (64-pattern tiles, S x 64 products per
branch, per-column 1e150 rescaling: likelihood.hpp:479-762, :1151-1197); the default is
the per-pattern form.  Every product sums over k in the same order, so lnL, the per-site
values and the branch gradients are identical; the global gradients go through A_b sums
in another order and agree to rounding.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("config,kw,rates", [(1, {"n_sites": 200, "n_taxa": 20}, False),
                                             (3, {"n_sites": 90, "n_taxa": 40}, True)])
def test_tiled_equals_per_pattern(oracle, config, kw, rates):
    from hyphy3.simulate import make_workload
    wl = make_workload(config, **kw)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    t = oracle.Tree.parse(wl.newick)
    cls = [{"alpha": 1.0, "beta": om, "theta": list(wl.theta)} for om in wl.omegas]
    r, rw = (list(wl.rates), list(wl.rate_w)) if rates else ([], [])
    bg = {"alpha": 1.0, "beta": 0.7, "theta": list(wl.theta)}
    is_test = [i % 3 != 1 for i in range(t.num_nodes())]
    out = [oracle.mixture_eval(t, a, cls, list(wl.omega_w), bg, is_test, r, rw, list(t.branch_lengths),
                               True, True, True, tiled) for tiled in (False, True)]
    assert out[0]["lnl"] == out[1]["lnl"]
    assert out[0]["site_lnl"] == out[1]["site_lnl"]
    assert out[0]["grad_t"] == out[1]["grad_t"]
    for k in ("grad_beta", "grad_class_w", "grad_theta", "grad_rate_w"):
        x, y = np.asarray(out[0][k], float), np.asarray(out[1][k], float)
        assert np.max(np.abs(x - y)) <= 1e-12 * max(1.0, float(np.max(np.abs(x)))), k
    assert abs(out[0]["grad_beta_bg"] - out[1]["grad_beta_bg"]) <= 1e-12 * max(1.0, abs(out[0]["grad_beta_bg"]))
