"""Multi-GPU sharding of the likelihood core: one process per GPU, torch.distributed plumbing.

Two partitions, both exact:

* Pattern sharding of one alignment.  Site patterns are independent given the
  tree and model (the reference evaluates them in self-contained tiles,
  likelihood.hpp:794-803, and sums per-pattern terms with weights), so every
  rank evaluates a contiguous range of patterns on its own device and one
  FP64 all-reduce (sum) of [lnL, dlnL/dt (n), dlnL/d(directions),
  dlnL/d(class weights), dlnL/d(rate weights)] gives the full result.  This is
  the only collective on the path; it moves (n + ~20) doubles per evaluation.
* Gene sharding of many independent alignments (longest-processing-time
  bin packing on cost ~ nodes x patterns x classes).  No collective on the
  data path; per-gene results may be gathered once at the end.

Errors do not desynchronise the ranks: a rank whose local evaluation fails
still joins the all-reduce with a failure flag set, and every rank then raises.

Data plane: with the NCCL backend and the library's problems, each rank's result
vector is assembled on its device (h3g_pack_result_device) and all-reduced in
device memory; with gloo (CPU tests) or substitute problems the vector is packed
on the host.

The evaluator on each rank is a `hyphy3._capi.Problem` (one device per
process); `problem_factory(parent, is_leaf, leaf_taxon, states, masks, weights,
pattern_range=(begin, end))` lets a caller substitute any object with the same
`set_model` / `eval` methods and `K`, `M`, `ndirs` attributes.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence

import numpy as np

from . import _capi

_FIELDS = ("grad_t", "grad_dir", "grad_class_w", "grad_rate_w")


def pattern_shards(n_patterns: int, world_size: int) -> list[tuple[int, int]]:
    """Contiguous [begin, end) pattern ranges, one per rank, sizes differing by at most one.

    The work per pattern does not depend on its weight (the weight only scales
    the pattern's terms), so ranges are balanced by pattern count.
    """
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    base, extra = divmod(int(n_patterns), world_size)
    out, b = [], 0
    for r in range(world_size):
        e = b + base + (1 if r < extra else 0)
        out.append((b, e))
        b = e
    return out


def lpt_assign(costs: Sequence[float], world_size: int) -> list[list[int]]:
    """Longest-processing-time assignment of independent jobs (genes, site fits) to ranks.

    Jobs are taken in decreasing cost and each goes to the currently least
    loaded rank (ties to the lower rank); the returned lists keep each rank's
    jobs in increasing index order.
    """
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    heap = [(0.0, r) for r in range(world_size)]
    bins: list[list[int]] = [[] for _ in range(world_size)]
    for j in sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i)):
        load, r = heapq.heappop(heap)
        bins[r].append(j)
        heapq.heappush(heap, (load + float(costs[j]), r))
    return [sorted(b) for b in bins]


def pack_result(res: dict | None, n: int, ndirs: int, K: int, M: int, failed: bool = False) -> np.ndarray:
    """[lnl, grad_t (n), grad_dir (ndirs), grad_class_w (K), grad_rate_w (M), failed] as one FP64 vector."""
    v = np.zeros(1 + n + ndirs + K + M + 1)
    if res is not None and not failed:
        v[0] = res["lnl"]
        o = 1
        for key, size in zip(_FIELDS, (n, ndirs, K, M)):
            if size:
                v[o:o + size] = np.asarray(res[key], dtype=np.float64)[:size]
            o += size
    v[-1] = 1.0 if failed else 0.0
    return v


def unpack_result(v: np.ndarray, n: int, ndirs: int, K: int, M: int) -> dict:
    out = {"lnl": float(v[0])}
    o = 1
    for key, size in zip(_FIELDS, (n, ndirs, K, M)):
        out[key] = np.array(v[o:o + size])
        o += size
    return out


def _allreduce_sum(vec: np.ndarray, group) -> np.ndarray:
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    t = torch.from_numpy(vec)
    if backend == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


class ShardedProblem:
    """One alignment's patterns split over the ranks of a process group.

    Every rank constructs it with the FULL pattern arrays (states [P, T],
    masks [P, T], weights [P]) and keeps only its own range; `eval` returns the
    full-alignment lnL and gradients on every rank.  Per-site log-likelihoods
    (WANT_SITE_LNL) are all-gathered into pattern order.
    """

    def __init__(self, ctx, parent, is_leaf, leaf_taxon, states, masks, weights, group=None,
                 problem_factory: Callable | None = None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        states = np.asarray(states)
        self.P_total = int(states.shape[0])
        self.shards = pattern_shards(self.P_total, self.world)
        b, e = self.shards[self.rank]
        self.begin, self.end = b, e
        factory = problem_factory or (lambda *a, pattern_range: _capi.Problem(ctx, *a))
        self.local = factory(parent, is_leaf, leaf_taxon, states[b:e], np.asarray(masks)[b:e], np.asarray(weights)[b:e],
                             pattern_range=(b, e))
        self.n = int(np.asarray(parent).size)
        self.K = self.M = self.ndirs = 0

    def set_model(self, **kw) -> None:
        self.local.set_model(**kw)
        self.K, self.M, self.ndirs = int(self.local.K), int(self.local.M), int(self.local.ndirs)

    def eval(self, bl, want=_capi.WANT_LNL | _capi.WANT_GRAD_T) -> dict:
        import torch.distributed as dist
        if dist.get_backend(self.group) == "nccl" and hasattr(self.local, "pack_device"):
            return self._eval_device(bl, want)
        return self._eval_host(bl, want)

    def _eval_device(self, bl, want) -> dict:
        """NCCL data plane: the local evaluation stays on the device, its result vector is assembled
        there (h3g_pack_result_device), summed across ranks by one NCCL all-reduce on device memory,
        and copied to the host once."""
        import torch
        import torch.distributed as dist
        width = 1 + self.n + self.ndirs + self.K + self.M + 1
        vec = torch.zeros(width, dtype=torch.float64, device="cuda")
        err = None
        try:
            if self.end > self.begin:
                self.local.stage_branch_lengths(bl)
                self.local.eval_resident(want)
                self.local.pack_device(want, vec.data_ptr())
                # the all-reduce (torch's current stream) runs after the library's stream has packed
                torch.cuda.current_stream().wait_stream(torch.cuda.ExternalStream(self.local.ctx.stream_handle))
        except Exception as ex:  # joined below so that no rank is left waiting in the collective
            err = ex
            vec.zero_()
            vec[-1] = 1.0
        dist.all_reduce(vec, op=dist.ReduceOp.SUM, group=self.group)
        host = vec.cpu().numpy()
        if host[-1] != 0.0:
            if err is not None:
                raise err
            raise RuntimeError(f"sharded evaluation failed on {int(host[-1])} rank(s)")
        out = unpack_result(host, self.n, self.ndirs, self.K, self.M)
        if want & _capi.WANT_SITE_LNL:
            local = self.local.read_result(want)["site_lnl"] if self.end > self.begin else np.zeros(0)
            out["site_lnl"] = self._gather_sites(np.asarray(local, dtype=np.float64)[: self.end - self.begin])
        return out

    def _eval_host(self, bl, want) -> dict:
        failed, err = False, None
        res = None
        try:
            if self.end > self.begin:
                res = self.local.eval(bl, want)
            else:
                res = {"lnl": 0.0, "site_lnl": np.zeros(0), "grad_t": np.zeros(self.n),
                       "grad_dir": np.zeros(self.ndirs), "grad_class_w": np.zeros(self.K), "grad_rate_w": np.zeros(self.M)}
        except Exception as ex:  # joined below so that no rank is left waiting in the collective
            failed, err = True, ex
        vec = _allreduce_sum(pack_result(res, self.n, self.ndirs, self.K, self.M, failed), self.group)
        if vec[-1] != 0.0:
            if err is not None:
                raise err
            raise RuntimeError(f"sharded evaluation failed on {int(vec[-1])} rank(s)")
        out = unpack_result(vec, self.n, self.ndirs, self.K, self.M)
        if want & _capi.WANT_SITE_LNL:
            out["site_lnl"] = self._gather_sites(np.asarray(res["site_lnl"], dtype=np.float64)[: self.end - self.begin])
        return out

    def _gather_sites(self, local: np.ndarray) -> np.ndarray:
        import torch
        import torch.distributed as dist
        width = max(e - b for b, e in self.shards)
        buf = np.zeros(width)
        buf[: local.size] = local
        t = torch.from_numpy(buf)
        if dist.get_backend(self.group) == "nccl":
            t = t.cuda()
        parts = [torch.empty_like(t) for _ in range(self.world)]
        dist.all_gather(parts, t, group=self.group)
        return np.concatenate([p.cpu().numpy()[: e - b] for p, (b, e) in zip(parts, self.shards)])

    def close(self) -> None:
        if hasattr(self.local, "close"):
            self.local.close()


def gather_gene_results(local: dict[int, dict], group=None) -> dict[int, dict]:
    """All-gather per-gene result dicts (gene index -> result) after a gene-sharded run."""
    import torch.distributed as dist
    parts: list = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    merged: dict[int, dict] = {}
    for p in parts:
        merged.update(p)
    return merged
