"""MG94 global fits on the device likelihood core (MG94Fitter, optimizer.hpp:857-1135).

The reference's own known answer: the full unconstrained MG94 fit of adh reaches
lnL = -4686.73 +- 5 (python/tests/test_python_autograd.py:46-55).  The fitted
point must also be a stationary point of the device gradient.
"""
import json
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def with_lengths(newick: str, length: float) -> str:
    """The same topology with every branch set to `length` (adh.nex's embedded tree has none)."""
    body = newick.strip().rstrip(";")
    return re.sub(r"([^(),:;]+|\))(?=[,)])", lambda m: m.group(1) + f":{length}", body) + ";"


@pytest.fixture(scope="module")
def adh_fit(golden_dir):
    import _hyphy3 as h3
    h3.set_precision("fp64")
    a = h3.Alignment.load(str(golden_dir / "adh.nex"))
    # the reference starts this fit from a nucleotide GTR fit; here every branch starts at 0.05
    t = h3.Tree.from_newick(with_lengths(a.embedded_tree_newick, 0.05))
    assert all(nd.branch_length == 0.05 for nd in t.nodes if nd.id != t.root_id)
    f = h3.MG94Fitter(t, a)
    quick = f.fit_omega_and_scale()
    full = f.fit_full_model()
    return h3, a, t, quick, full


def test_full_model_fit_matches_reference_adh(adh_fit, golden_dir):
    k = json.loads((golden_dir / "known_answers.json").read_text())["adh_global_fit"]
    h3, a, t, quick, full = adh_fit
    assert abs(full.log_likelihood - k["full_model_logl"]) <= k["delta"]
    assert full.log_likelihood >= quick.log_likelihood - 1e-6
    assert full.param_names[0] == "omega" and 0.01 < full.x_opt[0] < 10


def test_full_model_fit_is_stationary(adh_fit):
    h3, a, t, _, full = adh_fit
    ft = full.tree
    p = full.params
    bl = [nd.branch_length for nd in ft.nodes]
    r = h3.compute_joint_frechet_gradients(ft, a, p, bl)
    assert abs(r["log_likelihood"] - full.log_likelihood) < 1e-6 * abs(full.log_likelihood)
    # log-space gradients at the optimum: branches away from their lower bound, omega, thetas
    g = [b * gb for b, gb, nd in zip(bl, r["grad_branches"], ft.nodes) if nd.id != ft.root_id and b > 1e-6]
    th = [p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT]
    g += [p.beta * r["grad_omega"]] + [x * gx for x, gx in zip(th, r["grad_theta"])]
    assert np.max(np.abs(g)) < 0.05


def test_omega_and_scale_fit_improves_start(adh_fit):
    h3, a, t, quick, _ = adh_fit

    def lnl_at(omega, scale):
        p = h3.MG94Parameters()
        p.beta = omega
        conv = 3.0 / h3.mg94_eigensystem(a, p)["mu"]
        bl = [nd.branch_length * scale * conv for nd in t.nodes]
        return h3.compute_branch_length_gradients(t, a, p, bl)[0]

    omega, scale = quick.x_opt
    assert abs(lnl_at(omega, scale) - quick.log_likelihood) < 1e-9 * abs(quick.log_likelihood)
    assert quick.log_likelihood > lnl_at(1.0, 1.0)
