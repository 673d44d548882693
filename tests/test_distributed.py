"""Multi-rank host logic of hyphy3.distributed on CPU: gloo, world_size 2, the oracle as each rank's evaluator.

Pattern sharding must reproduce the unsharded evaluation (lnL, all gradients,
per-site lnL) to rounding; gene sharding must return every gene's result on
every rank; a rank whose evaluation fails must make every rank raise instead
of leaving the others waiting in the collective.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from hyphy3 import distributed as hd


def test_pattern_shards_cover_and_balance():
    for P in (0, 1, 7, 64, 1001):
        for W in (1, 2, 3, 8):
            sh = hd.pattern_shards(P, W)
            assert len(sh) == W and sh[0][0] == 0 and sh[-1][1] == P
            assert all(a[1] == b[0] for a, b in zip(sh, sh[1:]))
            sizes = [e - b for b, e in sh]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        hd.pattern_shards(10, 0)


def test_lpt_assign_partitions_and_bounds_makespan():
    rng = np.random.default_rng(7)
    costs = rng.integers(8, 512, size=50) * rng.integers(100, 3000, size=50)
    for W in (1, 2, 4, 8):
        bins = hd.lpt_assign(costs, W)
        flat = sorted(j for b in bins for j in b)
        assert flat == list(range(50))
        loads = [sum(costs[j] for j in b) for b in bins]
        # LPT is within 4/3 of optimal; the optimum is at least max(mean load, largest job)
        lower = max(costs.sum() / W, costs.max())
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-9


def test_pack_roundtrip():
    res = {"lnl": -12.5, "grad_t": np.arange(5.0), "grad_dir": np.array([1.0, 2.0]), "grad_class_w": np.array([3.0]),
           "grad_rate_w": np.array([4.0, 5.0])}
    v = hd.pack_result(res, 5, 2, 1, 2)
    assert v[-1] == 0.0
    back = hd.unpack_result(v, 5, 2, 1, 2)
    assert back["lnl"] == -12.5
    for k in ("grad_t", "grad_dir", "grad_class_w", "grad_rate_w"):
        np.testing.assert_array_equal(back[k], res[k])
    assert hd.pack_result(None, 5, 2, 1, 2, failed=True)[-1] == 1.0


class OracleShard:
    """The oracle on one pattern range, with the set_model / eval surface of a device Problem."""

    def __init__(self, tree, aln, begin, end, fail=False):
        self.tree, self.aln = tree, aln.subset_patterns(begin, end)
        self.fail = fail
        self.K = self.M = self.ndirs = 0

    def set_model(self, *, classes, class_w, rates=(), rate_w=()):
        self.classes, self.class_w, self.rates, self.rate_w = classes, list(class_w), list(rates), list(rate_w)
        self.K, self.M, self.ndirs = len(class_w), max(1, len(rates)), len(class_w) + 5

    def eval(self, bl, want):
        if self.fail:
            raise RuntimeError("planted failure")
        import h3oracle as o
        r = o.mixture_eval(self.tree, self.aln, self.classes, self.class_w, None, [], self.rates, self.rate_w,
                           list(bl), False, True, False)
        gr = list(r["grad_rate_w"]) if self.rates else [0.0]
        return {"lnl": r["lnl"], "grad_t": np.array(r["grad_t"]), "grad_dir": np.r_[r["grad_beta"], r["grad_theta"]],
                "grad_class_w": np.array(r["grad_class_w"]), "grad_rate_w": np.array(gr),
                "site_lnl": np.array(r["site_lnl"])}


def _case():
    import h3oracle as o
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=90, n_taxa=12)
    aln = o.Alignment.from_sequences(wl.names, wl.seqs)
    tree = o.Tree.parse(wl.newick)
    classes = [{"alpha": 1.0, "beta": om, "theta": wl.theta} for om in wl.omegas]
    model = {"classes": classes, "class_w": wl.omega_w, "rates": [0.4, 1.6], "rate_w": [0.5, 0.5]}
    return tree, aln, model


def _worker(rank, world, port, mode, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        tree, aln, model = _case()
        n = tree.num_nodes()
        fail_rank = 1 if mode == "fail" else -1
        factory = (lambda *a, pattern_range: OracleShard(tree, aln, *pattern_range, fail=(rank == fail_rank)))
        sp = hd.ShardedProblem(None, [0] * n, [0] * n, [0] * n, np.zeros((aln.num_patterns, 1)), np.zeros((aln.num_patterns, 1)),
                               np.zeros(aln.num_patterns), problem_factory=factory)
        sp.set_model(**model)
        from hyphy3 import _capi
        want = _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL | _capi.WANT_SITE_LNL
        if mode == "fail":
            try:
                sp.eval(list(tree.branch_lengths), want)
                q.put((rank, "no error"))
            except RuntimeError as ex:
                q.put((rank, str(ex)))
        elif mode == "genes":
            import h3oracle as o
            from hyphy3.simulate import make_workload
            sizes = [(6, 40), (9, 25), (5, 60), (12, 30), (7, 45)]
            costs = [nt * ns for nt, ns in sizes]
            mine = hd.lpt_assign(costs, world)[rank]
            local = {}
            for g in mine:
                wl = make_workload(0, n_taxa=sizes[g][0], n_sites=sizes[g][1])
                a = o.Alignment.from_sequences(wl.names, wl.seqs)
                t = o.Tree.parse(wl.newick)
                r = o.branch_length_gradients(t, a, {"alpha": 1.0, "beta": 0.5, "theta": wl.theta}, [])
                local[g] = {"lnl": r[0] if isinstance(r, tuple) else r["lnl"]}
            q.put((rank, hd.gather_gene_results(local)))
        else:
            q.put((rank, sp.eval(list(tree.branch_lengths), want)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(mode, world=2):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def test_pattern_sharded_matches_unsharded(oracle):
    tree, aln, model = _case()
    full = OracleShard(tree, aln, 0, aln.num_patterns)
    full.set_model(**model)
    ref = full.eval(list(tree.branch_lengths), 0)
    out = _run("patterns")
    for rank in (0, 1):
        r = out[rank]
        assert abs(r["lnl"] - ref["lnl"]) <= 1e-12 * abs(ref["lnl"])
        for k in ("grad_t", "grad_dir", "grad_class_w", "grad_rate_w"):
            np.testing.assert_allclose(r[k], ref[k], rtol=1e-11, atol=1e-11 * np.abs(ref[k]).max())
        np.testing.assert_allclose(r["site_lnl"], ref["site_lnl"], rtol=0, atol=0)


def test_failed_rank_raises_on_every_rank(oracle):
    out = _run("fail")
    assert out[1] == "planted failure"
    assert "failed on 1 rank" in out[0]


def test_gene_sharding_gathers_every_gene(oracle):
    out = _run("genes")
    assert sorted(out[0]) == list(range(5))
    assert out[0] == out[1]
