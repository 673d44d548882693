"""h3g_eval_from_P_noalloc against h3g_eval_from_P, through the C ABI.

The no-allocation entry point serves callers that may not allocate device
memory while they run (a process whose framework owns the whole device pool,
or a latency path that must not synchronise on an allocation).  It must give
the same lnL and per-pattern values as the allocating entry point on the same
inputs, on two calls in a row (the shared scratch keeps the previous call's
contents).  This file is collected last so a failure here leaves every other
test already run.
"""
import numpy as np
import pytest

from gpu_helpers import problem_from_oracle

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _inputs(oracle, golden_dir, which):
    if which == "cd2_reduced":
        import json
        known = json.loads((golden_dir / "known_answers.json").read_text())["cd2_reduced"]
        a = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
        t = oracle.Tree.parse(known["newick"])
        p = known["params"]
    else:
        from hyphy3.simulate import make_workload
        wl = make_workload(1, n_sites=150, n_taxa=24)
        a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
        t = oracle.Tree.parse(wl.newick)
        p = {"alpha": 1.0, "beta": 0.6, "theta": wl.theta}
    n = t.num_nodes()
    P = np.stack([np.eye(61) if i == t.root else oracle.transition_matrix(a, p, t.branch_lengths[i]) for i in range(n)])
    return t, a, P


@pytest.mark.parametrize("which", ["cd2_reduced", "synthetic"])
def test_noalloc_matches_allocating_entry_point(oracle, golden_dir, which):
    from hyphy3 import _capi
    t, a, P = _inputs(oracle, golden_dir, which)
    ctx = _capi.Context(0)
    pr = problem_from_oracle(ctx, oracle, t, a)
    ref_l, ref_site = pr.eval_from_P(P, a.pi)
    pr.close()
    ctx.close()
    l2t = oracle.leaf_map(t, a)
    leaf = np.array(t.is_leaf, dtype=np.uint8)
    taxon = np.array([l2t[i] if leaf[i] else -1 for i in range(t.num_nodes())], dtype=np.int32)
    for _ in range(2):
        lnl, site = _capi.eval_from_P_noalloc(np.array(t.parent, dtype=np.int32), leaf, taxon, a.states, a.masks,
                                              np.array(a.weights), P, a.pi)
        assert abs(lnl - ref_l) <= TOL * abs(ref_l)
        np.testing.assert_allclose(site, ref_site, rtol=TOL, atol=0)


def test_noalloc_rejects_problems_beyond_its_scratch(oracle):
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=1000, n_taxa=64)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    t = oracle.Tree.parse(wl.newick)
    n = t.num_nodes()
    P = np.zeros((n, 61, 61))
    l2t = oracle.leaf_map(t, a)
    leaf = np.array(t.is_leaf, dtype=np.uint8)
    taxon = np.array([l2t[i] if leaf[i] else -1 for i in range(n)], dtype=np.int32)
    with pytest.raises(_capi.H3GError, match="status 1"):
        _capi.eval_from_P_noalloc(np.array(t.parent, dtype=np.int32), leaf, taxon, a.states, a.masks,
                                  np.array(a.weights), P, a.pi)
