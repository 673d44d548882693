"""The NCCL data plane of pattern sharding, on one GPU (world size 1).

ShardedProblem with the NCCL backend keeps the evaluation on the device: the result vector is
assembled there (h3g_pack_result_device) and all-reduced in device memory.  With one rank the
all-reduce is the identity, so the sharded result must equal the single problem's h3g_eval (the
directional gradient is assembled on the device instead of the host: equal to rounding).  The
multi-rank logic (shard ranges, failure propagation, gathering) is covered by the gloo tests.
"""
import socket

import numpy as np
import pytest

from gpu_helpers import dq_beta, dq_theta, eigensystems, problem_from_oracle

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_nccl_world1_equals_single_problem(oracle):
    import datetime

    import torch
    import torch.distributed as dist
    from hyphy3 import _capi
    from hyphy3.distributed import ShardedProblem
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=250, n_taxa=30)
    t = oracle.Tree.parse(wl.newick)
    a = oracle.Alignment.from_sequences(wl.names, wl.seqs)
    models = [{"alpha": 1.0, "beta": om, "theta": list(wl.theta)} for om in wl.omegas]
    Q, lam, U, V, mu = eigensystems(oracle, a, models)
    nm = len(models)
    dirs = []
    for k in range(nm):
        d = np.zeros((nm, 61, 61))
        d[k] = dq_beta(a, models[k])
        dirs.append(d)
    dirs.append(np.stack([dq_theta(a, 3, m) for m in models]))
    dirs = np.stack(dirs)
    kw = dict(pi=a.pi, Q=Q, lam=lam, U=U, V=V, mu=mu, class_w=list(wl.omega_w), rates=[0.5, 1.5], rate_w=[0.4, 0.6],
              dQ=dirs, time_mode=_capi.TIME_NORMALIZED)
    want = _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL | _capi.WANT_SITE_LNL
    bl = np.array(t.branch_lengths)
    ctx = _capi.Context(0)
    single = problem_from_oracle(ctx, oracle, t, a)
    single.set_model(**kw)
    ref = single.eval(bl, want)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        l2t = oracle.leaf_map(t, a)
        leaf = np.array(t.is_leaf, dtype=np.uint8)
        taxon = np.array([l2t[i] if leaf[i] else -1 for i in range(t.num_nodes())], dtype=np.int32)
        sp = ShardedProblem(ctx, np.array(t.parent, dtype=np.int32), leaf, taxon, a.states, a.masks, np.array(a.weights))
        sp.set_model(**kw)
        for _ in range(2):
            out = sp.eval(bl, want)
            assert out["lnl"] == ref["lnl"]
            assert np.array_equal(out["grad_t"], ref["grad_t"])
            assert np.array_equal(out["grad_class_w"], ref["grad_class_w"])
            assert np.array_equal(out["grad_rate_w"], ref["grad_rate_w"])
            assert np.allclose(out["grad_dir"], ref["grad_dir"][: sp.ndirs], rtol=1e-13, atol=1e-12)
            assert np.array_equal(out["site_lnl"], ref["site_lnl"])
        sp.close()
    finally:
        dist.destroy_process_group()
    single.close()
    ctx.close()
