"""Benchmark: codon site-branch lnL+gradient evaluations per second on one B200.

Workload (one step = one lnL + full-gradient evaluation), default --config 3, the largest
single-GPU configuration:
  1024-taxon Yule tree (2045 branches), 5000 simulated codons, MG94xREV with omegas
  {0.2, 2} (weights {0.8, 0.2}) mixed at the P level and 4 discrete-gamma synonymous-rate
  classes as separate pruning passes combined by a root log-sum-exp; lnL plus the gradient
  w.r.t. every branch length, both omegas, both class weights, the 5 exchangeabilities and the
  4 rate weights.  Unit: alignment sites x branches per completed evaluation (5000 x 2045).
  --config 1: the 64-taxon, 1000-codon, 3-omega mixture; 2: FEL per-site fits; 4: 500 uneven
  genes in one batch.

value  device-resident throughput: branch lengths already on the device, each
       step timed with CUDA events on the library's stream, L2 flushed (256 MiB
       write) before every timed step.
e2e    the same evaluation through the public API (_hyphy3.compute_mixture_gradients)
       with host inputs and host results, host wall clock around the
       synchronous calls.
--impl reference  times the CPU restatement of the reference engine (the
       reference itself needs Eigen, which this image lacks) on the host cores.
Multi-GPU (torchrun): one process per GPU.  Default (--mode sharded): the
workload's site patterns split over the ranks, one NCCL all-reduce of the
device-assembled result vector per step (strong scaling); --mode replicas: each
rank evaluates its own replica gene with no collective (weak scaling).  value =
all ranks' units / max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
for _p in (ROOT / "hyphy-3_b200" / "python", ROOT / "oracle" / "_build"):
    sys.path.insert(0, str(_p))

import numpy as np  # noqa: E402

METRIC = "codon site*branch lnL+grad evals/s: mixed vs FP64 on 1 B200 at |dlnL|/|lnL|<=1e-7"
UNIT = "site*branch/s"
WORKLOAD = ("BUSTED-style 3-omega MG94xREV: 64-taxon random unrooted tree (125 branches), 1000 codons "
            "(3% gaps, 1% ambiguous), omegas {0.1,1,5} w {0.6,0.3,0.1}; lnL + grads wrt 125 t, 3 omega, 3 w, 5 theta")


WORKLOADS = {
    1: WORKLOAD,
    3: ("large mixed MG94xREV: 1024-taxon Yule tree (2045 branches), 5000 codons, omegas {0.2,2} w {0.8,0.2} "
        "mixed at the P level x 4 discrete-gamma synonymous-rate passes (root log-sum-exp); lnL + grads wrt 2045 t, "
        "2 omega, 2 w, 5 theta, 4 rate weights"),
}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of each pruning stage per evaluation,
# summed over the stage's launches in the ncu launch list of `bench.py --profile` (one evaluation,
# --clock-control none).  The 1024-taxon workload is captured on its 512-codon prefix and scaled by
# the padded pattern count (5120 / 512): these stages stream per-pattern partials, so their traffic is
# proportional to the patterns processed.
MEASURED_TRAFFIC = {
    (1, "mixed"): {"inside": 19.5e6, "outside": 36.2e6, "accum_A": 49.4e6},
    (1, "fp64"): {"inside": 36.5e6, "outside": 68.7e6, "accum_A": 98.3e6},
    (3, "mixed"): {"inside": 14.724e9, "outside": 28.220e9, "accum_A": 18.835e9},
    (3, "fp64"): {"inside": 29.259e9, "outside": 48.234e9, "accum_A": 34.790e9},
    # alignment compression, 1024 taxa x 100000 codons, captured at full size (one pass:
    # dram__bytes_read.sum + dram__bytes_write.sum of the call's launch)
    ("compress", "translate"): 479.30e6,
    ("compress", "rounds"): 207.80e6,
}


def build_inputs(seed_offset: int = 0, config: int = 1, sites: int | None = None):
    import _hyphy3 as h
    from hyphy3.simulate import make_workload
    wl = make_workload(config, n_sites=sites)
    if seed_offset:
        # independent replica gene for another rank: same shapes, different draw
        import hyphy3.simulate as sim
        rng = np.random.default_rng(sim.SEED_BASE + 1 + 1000 * seed_offset)
        noisy = config == 1
        names, seqs = sim.simulate_alignment(wl.tree, wl.n_sites, rng, theta=wl.theta,
                                             pos_freq=rng.dirichlet(np.ones(4), size=3), omegas=wl.omegas,
                                             omega_w=wl.omega_w, rates=wl.rates, rate_w=wl.rate_w,
                                             gap_frac=0.03 if noisy else 0.0, ambig_frac=0.01 if noisy else 0.0)
        wl.names, wl.seqs = names, seqs
    aln = h.Alignment.from_sequences(wl.names, wl.seqs)
    tree = h.Tree.from_newick(wl.newick)
    return h, wl, aln, tree


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
            # nvidia-smi takes a moment to start: wait (bounded) for its first sample, then drop it,
            # so the samples kept are the ones taken while the timed region runs
            t_end = time.time() + 3.0
            while not self.lines and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
            self.lines.clear()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def fp64_dgemm_peak() -> float:
    """Measured FP64 matmul throughput (cuBLAS DGEMM, 8192^3) in TFLOP/s, best of 5."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def stage_work(aln_P: int, tree, M: int, elem_bytes: int = 8) -> dict:
    """Algorithmic bytes and flops per stage for one evaluation (61 states, not padded).

    elem_bytes is the storage width of a partial entry: 8 on the FP64 path, 4 on
    the mixed path (FP32 partials; the per-pattern int32 exponent is counted as
    4 more bytes per stored vector).
    Partials are counted as one HBM round trip each way: the inside stage
    reads the messages of internal children, writes D and (non-root) the
    message P*D; the outside stage reads U of the parent and the sibling
    messages, writes the scaled outside vector of every child and U of
    internal children; accum_A reads V and D of every branch.
    """
    S = 61
    nodes = tree.nodes
    root = tree.root_id
    internal = [nd for nd in nodes if not nd.is_leaf]
    cols = aln_P * M
    vec = elem_bytes * S + (4 if elem_bytes == 4 else 0)
    ins_b = ins_f = out_b = out_f = acc_b = acc_f = 0
    for nd in internal:
        int_kids = [c for c in nd.children if not nodes[c].is_leaf]
        ins_b += vec * (len(int_kids) + 1 + (nd.id != root))
        ins_f += 2 * S * S * (nd.id != root)
        k = len(nd.children)
        out_b += vec * (1 + k)
        for c in nd.children:
            out_b += vec * sum(1 for s in nd.children if s != c and not nodes[s].is_leaf)
            if not nodes[c].is_leaf:
                out_b += vec
                out_f += 2 * S * S
    for nd in nodes:
        if nd.id == root:
            continue
        acc_b += vec * (2 if not nd.is_leaf else 1)
        acc_f += 2 * S * S
    return {"inside": (ins_b * cols, ins_f * cols), "outside": (out_b * cols, out_f * cols),
            "accum_A": (acc_b * cols, acc_f * cols)}


def load_simulate():
    """hyphy3/simulate.py loaded by file path: the workload generator is plain numpy, and loading it
    this way keeps the hyphy3 package (and with it the CUDA library) out of the CPU-only legs."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("h3_simulate", ROOT / "hyphy-3_b200" / "python" / "hyphy3" / "simulate.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["h3_simulate"] = mod
    spec.loader.exec_module(mod)
    return mod


# patterns per CPU step: the whole 64-taxon alignment; a 384-pattern slice of the 1024-taxon one
# (about 3 s per evaluation on 16 host threads)
CPU_SAMPLE_PATTERNS = {1: None, 3: 384}


class CpuEngine:
    """The CPU restatement of the reference engine (oracle/, FP64, OpenMP on every host thread) in the
    reference's batched shape: 64-pattern tiles, S x 64 products per branch (likelihood.hpp:1151-1197),
    on the workload's tree and classes and a bounded slice of its site patterns."""

    def __init__(self, wl, max_patterns: int | None):
        import h3oracle as o
        self.o = o
        a = o.Alignment.from_sequences(wl.names, wl.seqs)
        self.full_patterns = a.num_patterns
        if max_patterns is not None and max_patterns < self.full_patterns:
            a = a.subset_patterns(0, max_patterns)
        self.a = a
        self.t = o.Tree.parse(wl.newick)
        self.cls = [{"alpha": 1.0, "beta": om, "theta": list(wl.theta)} for om in wl.omegas]
        self.w = list(wl.omega_w)
        self.rates, self.rw = (list(wl.rates), list(wl.rate_w)) if len(wl.rates) > 1 else ([], [])
        self.threads = o.max_threads()
        o.set_threads(self.threads)
        self.bl = list(self.t.branch_lengths)
        self.sites = float(np.sum(a.weights))
        self.branches = self.t.num_nodes() - 1
        self.patterns = len(a.weights)

    def step(self) -> float:
        return self.o.mixture_eval(self.t, self.a, self.cls, self.w, None, [], self.rates, self.rw, self.bl,
                                   False, True, False, True)["lnl"]

    def sample_text(self, n_steps: int, what: str) -> str:
        return (f"{n_steps} {what}: lnL + gradients w.r.t. every branch length, omega, class weight, theta and rate "
                f"weight over {self.patterns} of {self.full_patterns} site patterns ({self.sites:.0f} sites) x "
                f"{self.branches} branches, oracle/ CPU restatement in 64-pattern tiles (the reference itself needs "
                f"Eigen 3.4, absent from this image)")


def cpu_baseline(wl, config: int, reps: int = 3) -> dict:
    """The CPU restatement on the host cores (all threads), a bounded sample of the workload."""
    eng = CpuEngine(wl, CPU_SAMPLE_PATTERNS.get(config))
    eng.step()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        eng.step()
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return {"value": eng.sites * eng.branches / med, "unit": UNIT, "cores": eng.threads, "kind": "port",
            "sample": eng.sample_text(reps, f"evaluations after 1 warm-up, median {med:.3f} s")}


def run_reference(args) -> None:
    """The reference arm: the CPU restatement of the reference engine on every host thread (rank 0 only),
    exactly --warmup untimed and --steps timed evaluations of the configured workload's sample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sim = load_simulate()
    if args.config == 4:
        run_reference_genes(args, sim)
        return
    wl = sim.make_workload(args.config)
    eng = CpuEngine(wl, CPU_SAMPLE_PATTERNS.get(args.config))
    for _ in range(args.warmup):
        eng.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.step()
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    v = eng.sites * eng.branches / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.config], "sites": wl.n_sites, "branches": eng.branches},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": eng.threads, "kind": "port",
                             "sample": eng.sample_text(args.steps, "timed evaluations")},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_genes(args, sim) -> None:
    """Reference arm of the multi-gene workload: each step evaluates a fixed sample of 4 of its genes
    (lnL + branch gradients) with the CPU restatement on every host thread."""
    import h3oracle as o
    G = args.genes or 500
    genes = sim.make_gene_batch(G)
    sample = sorted(np.random.default_rng(1).choice(G, size=4, replace=False).tolist())
    threads = o.max_threads()
    o.set_threads(threads)
    work = []
    for gi in sample:
        g = genes[gi]
        oa = o.Alignment.from_sequences(g.names, g.seqs)
        ot = o.Tree.parse(g.newick)
        work.append((ot, oa, [{"alpha": 1.0, "beta": g.omega, "theta": list(g.theta)}]))
    units = sum(oa.num_codons * (ot.num_nodes() - 1) for ot, oa, _ in work)

    def step():
        for ot, oa, cls in work:
            o.mixture_eval(ot, oa, cls, [1.0], None, [], [], [], list(ot.branch_lengths), False, False, False, True)
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    v = units / dt
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": BATCH_WORKLOAD.format(G=G, S=args.slots), "genes": G},
                      "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                       "sample": f"genes {sample} per step, lnL + branch gradients, oracle/ CPU restatement"},
                      "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def run_sharded(args) -> None:
    """N GPUs, one process each: the workload's site patterns split into N contiguous ranges
    (hyphy3.distributed.ShardedProblem); per step every rank evaluates its range on its device, the
    result vectors are assembled on the devices and summed by one NCCL all-reduce in device memory,
    and the full-alignment result is copied to the host.  Strong scaling (one alignment, fixed)."""
    import datetime

    import torch
    import torch.distributed as dist
    from hyphy3 import _capi
    from hyphy3.distributed import ShardedProblem
    world = int(os.environ["WORLD_SIZE"])
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    h, wl, aln, tree = build_inputs(config=args.config)
    stream = torch.cuda.current_stream()
    ctx = _capi.Context(local, stream=stream.cuda_stream)
    states, masks, weights = aln.pattern_arrays()
    l2t = h.build_leaf_to_taxon_map(tree, aln)
    n = tree.num_nodes()
    is_leaf = np.array([nd.is_leaf for nd in tree.nodes], dtype=np.uint8)
    sp = ShardedProblem(ctx, np.array(tree.parents, dtype=np.int32), is_leaf,
                        np.array([l2t[i] if is_leaf[i] else -1 for i in range(n)], dtype=np.int32), states, masks, weights)
    es = []
    for om in wl.omegas:
        p = h.MG94Parameters()
        p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = wl.theta
        p.beta = om
        es.append(h.mg94_eigensystem(aln, p))
    sp.set_model(pi=aln.codon_frequencies, Q=np.stack([e["Q"] for e in es]), lam=np.stack([e["lam"] for e in es]),
                 U=np.stack([e["U"] for e in es]), V=np.stack([e["V"] for e in es]), mu=np.array([e["mu"] for e in es]),
                 class_w=wl.omega_w, rates=list(wl.rates), rate_w=list(wl.rate_w), dQ=_directions(aln, wl, es),
                 precision=_capi.PREC_MIXED)
    want = _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL
    bl = np.array(tree.get_branch_lengths())
    units = wl.n_sites * (n - 1)
    for _ in range(max(args.warmup, 3)):
        sp.eval(bl, want)
    dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t0 = time.perf_counter()
    for e0, e1 in evs:
        e0.record()
        out = sp.eval(bl, want)
        e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clocks = sampler.stop() if sampler else None
    dist.barrier()
    t = torch.tensor([sum(a.elapsed_time(b) for a, b in evs) / 1e3, wall], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    secs, wall_max = float(t[0].item()), float(t[1].item())
    if rank == 0:
        line = {"metric": METRIC, "value": units * args.steps / secs, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "bf16x3/f32", "data": "synthetic",
                "config": {"workload": WORKLOADS[args.config], "sites": wl.n_sites, "branches": n - 1,
                           "patterns": aln.num_patterns, "precision": "mixed",
                           "l2": "inputs far larger than L2 (partials stream through HBM every step)",
                           "parallelism": f"pattern-shards{world} (one NCCL all-reduce of the result vector per step)"},
                "e2e": {"value": units * args.steps / wall_max, "unit": UNIT, "h2d_bytes_per_step": 8 * n,
                        "d2h_bytes_per_step": 8 * (2 + n + sp.ndirs + sp.K + sp.M),
                        "api": "hyphy3.distributed.ShardedProblem.eval", "timing": "host wall clock, max over ranks"},
                "gpu_launches": None, "clocks": clocks, "lnl": out["lnl"]}
        print(json.dumps(line), flush=True)
    sp.close()
    ctx.close()
    dist.destroy_process_group()


def run_ours(args) -> None:
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and args.mode == "sharded":
        run_sharded(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    h, wl, aln, tree = build_inputs(seed_offset=rank, config=args.config)
    from hyphy3 import _capi
    precision = args.precision
    if precision == "auto":
        precision = "mixed" if _mixed_available() else "fp64"
    prec_code = _capi.PREC_MIXED if precision == "mixed" else _capi.PREC_FP64
    stream = torch.cuda.Stream()
    ctx = _capi.Context(local, stream=stream.cuda_stream)
    states, masks, weights = aln.pattern_arrays()
    l2t = h.build_leaf_to_taxon_map(tree, aln)
    n = tree.num_nodes()
    is_leaf = np.array([nd.is_leaf for nd in tree.nodes], dtype=np.uint8)
    pr = _capi.Problem(ctx, np.array(tree.parents, dtype=np.int32), is_leaf,
                       np.array([l2t[i] if is_leaf[i] else -1 for i in range(n)], dtype=np.int32),
                       states, masks, weights)
    base = h.MG94Parameters()
    base.theta_AC, base.theta_AT, base.theta_CG, base.theta_CT, base.theta_GT = wl.theta

    def model_arrays():
        es = []
        for om in wl.omegas:
            p = h.MG94Parameters()
            p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = wl.theta
            p.beta = om
            es.append(h.mg94_eigensystem(aln, p))
        return es

    es = model_arrays()
    # directions: 3 omegas (dQ/dbeta of one class) + 5 thetas, built like the public API does
    dirs = _directions(aln, wl, es)
    want = _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL
    bl = np.array(tree.get_branch_lengths())
    units = wl.n_sites * (n - 1)

    def install(prec):
        pr.set_model(pi=aln.codon_frequencies, Q=np.stack([e["Q"] for e in es]), lam=np.stack([e["lam"] for e in es]),
                     U=np.stack([e["U"] for e in es]), V=np.stack([e["V"] for e in es]),
                     mu=np.array([e["mu"] for e in es]), class_w=wl.omega_w, rates=list(wl.rates),
                     rate_w=list(wl.rate_w), dQ=dirs, precision=prec)
        if args.memory_budget:
            # subtree checkpointing: the workspace is held under the budget, partials recomputed per block
            pr.set_memory_budget(int(args.memory_budget * 1e9))
        pr.stage_branch_lengths(bl)

    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def device_timed(steps, warmup, sampler=None):
        for _ in range(warmup):
            pr.eval_resident(want)
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for e0, e1 in evs:
                flush.zero_()
                e0.record(stream)
                pr.eval_resident(want)
                e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        return sum(e0.elapsed_time(e1) for e0, e1 in evs) / 1e3

    results = {}
    for prec_name, code in ([("fp64", _capi.PREC_FP64)] + ([("mixed", _capi.PREC_MIXED)] if precision == "mixed" else [])):
        install(code)
        # launch shapes from the autotuner (h3g_autotune: coordinate descent over the A-accumulation chunk,
        # the persistent passes' CTAs per SM and the Frechet branch groups), part of setup, not timed
        tuning, _ = pr.autotune(bl, want, reps=2) if not args.no_tune else (pr.get_tuning(), 0.0)
        pr.stage_branch_lengths(bl)
        sampler = ClockSampler(local) if prec_name == precision else None
        secs = device_timed(args.steps, max(args.warmup, 3), sampler)
        clocks = sampler.stop() if sampler else None
        t = torch.tensor([secs], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        res = pr.read_result(want)
        stages = pr.profile_stages(want, reps=3)
        results[prec_name] = {"secs": float(t.item()), "lnl": res["lnl"], "grad_t": res["grad_t"].copy(),
                              "grad_dir": res["grad_dir"].copy(), "clocks": clocks, "stages": stages, "tuning": tuning,
                              "checkpoint": pr.checkpoint_info()}
    head = results[precision]
    ms_per_step = head["secs"] / args.steps * 1e3
    value = units * world * args.steps / head["secs"]
    _, launches = pr.last_stats()
    launches_per_eval = sum(v[1] for v in head["stages"].values())

    # end to end through the public API, host buffers in and out
    h.set_precision(precision)
    if args.memory_budget:
        h.set_memory_budget(int(args.memory_budget * 1e9))
    bl_list = list(bl)
    api_args = (tree, aln, base, bl_list, wl.omegas, wl.omega_w, list(wl.rates), list(wl.rate_w))
    for _ in range(max(args.warmup, 3)):
        r_api = h.compute_mixture_gradients(*api_args)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r_api = h.compute_mixture_gradients(*api_args)
    e2e_secs = time.perf_counter() - t0
    et = torch.tensor([e2e_secs], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e_value = units * world * args.steps / float(et.item())
    h2d = int(n * 8)
    d2h = int((2 + n + len(wl.omegas) + len(wl.omegas) + 1) * 8 + dirs.shape[0] * len(es) * 8 + aln.num_patterns * 8)

    # accuracy of the headline path against the FP64 path on the same inputs
    acc = None
    if precision == "mixed":
        f, m = results["fp64"], results["mixed"]
        acc = {"rel_dlnl": abs(m["lnl"] - f["lnl"]) / abs(f["lnl"]),
               "grad_rel_err": float(np.linalg.norm(np.r_[m["grad_t"], m["grad_dir"]] - np.r_[f["grad_t"], f["grad_dir"]]) /
                                     np.linalg.norm(np.r_[f["grad_t"], f["grad_dir"]]))}

    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    work = stage_work(aln.num_patterns, tree, len(wl.rates), 4 if precision == "mixed" else 8)
    work64 = stage_work(aln.num_patterns, tree, len(wl.rates), 8)
    stg = head["stages"]
    dom = max(("inside", "outside", "accum_A"), key=lambda k: stg.get(k, (0.0, 0))[0])
    dom_ms, dom_launches = stg[dom]
    dom_bytes, dom_flops = work[dom]
    traffic = MEASURED_TRAFFIC.get((args.config, precision), {}).get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": dom_bytes / (dom_ms * 1e-3) / 1e9, "peak": hbm_peak,
                "unit": "GB/s", "frac": dom_bytes / (dom_ms * 1e-3) / 1e9 / hbm_peak, "traffic": traffic,
                "traffic_unit": "bytes per evaluation (all launches of the stage), from ncu",
                "peak_source": "measured" if peaks else "fallback",
                "algorithmic_bytes_per_eval": dom_bytes, "stage_ms": dom_ms, "launches_per_eval": dom_launches}
    fp64_peak = fp64_dgemm_peak() if rank == 0 else None
    f_st = results["fp64"]["stages"]
    fp64_pipe = {}
    for k in ("inside", "outside", "accum_A"):
        if k in f_st and f_st[k][0] > 0:
            fl = work64[k][1] / (f_st[k][0] * 1e-3) / 1e12
            fp64_pipe[k] = {"tflops": fl, "frac_of_dgemm": fl / fp64_peak if fp64_peak else None, "ms": f_st[k][0]}

    cpu = cpu_baseline(wl, args.config) if (rank == 0 and world == 1 and not args.no_cpu) else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if precision == "fp64" else "bf16x3/f32", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.config], "sites": wl.n_sites, "branches": n - 1, "patterns": aln.num_patterns,
                       "precision": precision, "l2": "flushed (256 MiB write) before every timed step",
                       "parallelism": f"replicas{world}" if world > 1 else "single", "tuning": head["tuning"],
                       "workspace_gb": head["checkpoint"]["workspace_bytes"] / 1e9,
                       **({"checkpoint": head["checkpoint"]} if head["checkpoint"]["active"] else {})},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "api": "_hyphy3.compute_mixture_gradients", "timing": "host wall clock around synchronous calls"},
            "gpu_launches": launches_per_eval * args.steps,
            "roofline": roofline,
            "fp64_pipe": {"dgemm_peak_tflops": fp64_peak, "stages": fp64_pipe},
            "stage_ms": {k: v[0] for k, v in stg.items()},
            "clocks": head["clocks"],
            "cpu_baseline": cpu,
            "fp64_value": units * world * args.steps / results["fp64"]["secs"],
            "accuracy_vs_fp64": acc,
            "lnl": head["lnl"], "api_lnl": r_api["log_likelihood"],
        }
        print(json.dumps(line), flush=True)
    pr.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()


BATCH_WORKLOAD = ("uneven multi-gene batch: {G} simulated genes, taxa ~ U{{8..512}}, codons ~ U{{100..3000}}, each with "
                  "its own random unrooted tree and MG94xREV parameters (one omega); per step lnL + the gradient w.r.t. "
                  "every branch length of every gene, all genes in one CUDA-graph launch over {S} slot workspaces")


def _gene_problems(h, _capi, ctx, genes):
    """One device problem per gene (no model yet: models go in once the problems belong to a batch,
    whose slot workspaces they use); the genes' host objects."""
    probs, hosts = [], []
    for g in genes:
        aln = h.Alignment.from_sequences(g.names, g.seqs)
        tree = h.Tree.from_newick(g.newick)
        states, masks, weights = aln.pattern_arrays()
        l2t = h.build_leaf_to_taxon_map(tree, aln)
        n = tree.num_nodes()
        is_leaf = np.array([nd.is_leaf for nd in tree.nodes], dtype=np.uint8)
        pr = _capi.Problem(ctx, np.array(tree.parents, dtype=np.int32), is_leaf,
                           np.array([l2t[i] if is_leaf[i] else -1 for i in range(n)], dtype=np.int32), states, masks, weights)
        p = h.MG94Parameters()
        p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = g.theta
        p.beta = g.omega
        probs.append(pr)
        hosts.append((aln, tree, p))
    return probs, hosts


def _install_gene_models(h, probs, hosts, precision):
    """Each gene's MG94 generator, diagonalised on the device."""
    for pr, (aln, tree, p) in zip(probs, hosts):
        e = h.mg94_eigensystem(aln, p)
        pr.set_model(pi=aln.codon_frequencies, Q=e["Q"], mu=[e["mu"]], precision=precision)


def run_batch(args) -> None:
    """The uneven multi-gene workload through h3g_batch_* (one graph launch per step), FP64 and mixed,
    a short joint branch-length fit, and the CPU restatement on a sample of the genes."""
    import torch
    import _hyphy3 as h
    from hyphy3 import _capi
    from hyphy3.batch import fit_branch_lengths
    from hyphy3.simulate import make_gene_batch
    G = args.genes or 500
    genes = make_gene_batch(G)
    ctx = _capi.Context(0)
    want = _capi.WANT_LNL | _capi.WANT_GRAD_T
    results, units, batch = {}, 0, None
    steps, warm = args.steps, max(args.warmup, 3)
    for prec_name, prec in (("fp64", _capi.PREC_FP64), ("mixed", _capi.PREC_MIXED)):
        if batch is None:
            probs, hosts = _gene_problems(h, _capi, ctx, genes)
            batch = _capi.Batch(ctx, probs, n_slots=args.slots)
            bls = [np.array(tr.get_branch_lengths()) for _, tr, _ in hosts]
            units = sum(aln.num_sites * (tr.num_nodes() - 1) for aln, tr, _ in hosts)
        _install_gene_models(h, probs, hosts, prec)
        for _ in range(warm):
            batch.eval(bls, want)
        sampler = ClockSampler(0) if prec_name == "mixed" else None
        if sampler:
            sampler.start()
        dev, t0 = [], time.perf_counter()
        for _ in range(steps):
            out = batch.eval(bls, want)
            dev.append(batch.last_stats()[0])
        wall = time.perf_counter() - t0
        clocks = sampler.stop() if sampler else None
        results[prec_name] = {"dev_s": sum(dev) / 1e3, "wall_s": wall, "launches": batch.last_stats()[1], "clocks": clocks,
                              "lnl": [o["lnl"] for o in out], "grad": np.concatenate([o["grad_t"] for o in out])}
    m, f = results["mixed"], results["fp64"]
    acc = {"rel_dlnl": abs(sum(m["lnl"]) - sum(f["lnl"])) / abs(sum(f["lnl"])),
           "max_gene_rel_dlnl": max(abs(a - b) / abs(b) for a, b in zip(m["lnl"], f["lnl"])),
           "grad_rel_err": float(np.linalg.norm(m["grad"] - f["grad"]) / np.linalg.norm(f["grad"]))}
    # joint fit of every gene's branch lengths (mixed): objective = one batch evaluation
    t0 = time.perf_counter()
    fit = fit_branch_lengths(batch, bls, max_iter=args.fit_iters)
    fit_s = time.perf_counter() - t0
    # algorithmic bytes of the three pruning stages summed over the genes (FP32 partials)
    alg = 0.0
    for aln, tree, _ in hosts:
        w = stage_work(aln.num_patterns, tree, 1, 4)
        alg += sum(w[k][0] for k in ("inside", "outside", "accum_A"))
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    per_step = m["dev_s"] / steps
    cpu = None
    if not args.no_cpu:
        import h3oracle as o
        rng = np.random.default_rng(1)
        sample = sorted(rng.choice(G, size=4, replace=False).tolist())
        threads = o.max_threads()
        o.set_threads(threads)
        cu, ct = 0, 0.0
        for gi in sample:
            g = genes[gi]
            oa = o.Alignment.from_sequences(g.names, g.seqs)
            ot = o.Tree.parse(g.newick)
            cls = [{"alpha": 1.0, "beta": g.omega, "theta": list(g.theta)}]
            t1 = time.perf_counter()
            o.mixture_eval(ot, oa, cls, [1.0], None, [], [], [], list(ot.branch_lengths), False, False, False, True)
            ct += time.perf_counter() - t1
            cu += oa.num_codons * (ot.num_nodes() - 1)
        cpu = {"value": cu / ct, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"genes {sample}: one lnL + branch-gradient evaluation each, oracle/ CPU restatement in 64-pattern tiles"}
    line = {
        "metric": METRIC, "value": units * steps / m["dev_s"], "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": warm,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16x3/f32", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD.format(G=G, S=args.slots), "genes": G,
                   "sites": int(sum(aln.num_sites for aln, _, _ in hosts)), "branches": int(sum(t.num_nodes() - 1 for _, t, _ in hosts)),
                   "site_branch_units": int(units), "precision": "mixed", "slots": args.slots,
                   "l2": "inputs far larger than L2 (every gene's partials stream through HBM)", "parallelism": "single"},
        "e2e": {"value": units * steps / m["wall_s"], "unit": UNIT, "h2d_bytes_per_step": int(sum(8 * t.num_nodes() for _, t, _ in hosts)),
                "d2h_bytes_per_step": int(sum(8 * (4 + 2 * t.num_nodes()) for _, t, _ in hosts)),
                "api": "hyphy3._capi.Batch.eval (h3g_batch_eval)", "timing": "host wall clock around synchronous calls"},
        "gpu_launches": m["launches"] * steps,
        "roofline": {"bound": "hbm", "kernel": "batch graph (inside + outside + accum_A of every gene)",
                     "achieved": alg / per_step / 1e9, "peak": hbm, "unit": "GB/s", "frac": alg / per_step / 1e9 / hbm,
                     "traffic": None, "peak_source": "measured" if peaks else "fallback",
                     "algorithmic_bytes_per_eval": alg, "note": "whole graph time, H2D/D2H copies included"},
        "clocks": m["clocks"], "cpu_baseline": cpu,
        "fp64_value": units * steps / f["dev_s"], "accuracy_vs_fp64": acc,
        "joint_fit": {"iterations": fit["iterations"], "evaluations": fit["evaluations"], "seconds": fit_s,
                      "lnl_start": float(sum(m["lnl"])), "lnl_end": fit["log_likelihood"]},
    }
    print(json.dumps(line), flush=True)
    batch.close()
    for pr in probs:
        pr.close()
    ctx.close()


MEME_METRIC = "MEME per-site fits/s (FEL baseline + MEME alternative, null and branch EBFs per codon site)"
MEME_WORKLOAD = ("MEME per-site fits: 256-taxon random unrooted tree (509 branches), 2000 simulated codons, every "
                 "branch tested; per site the FEL fit, the reference's 4-D Nelder-Mead of (alpha, omega1, p1, beta+) "
                 "from its start grid, the 3-D null and warm refit where beta+ > alpha, LRT, p-value and the "
                 "empirical Bayes factor of every branch")
FEL_METRIC = "FEL per-site fits/s (alternative + null model per codon site)"
FEL_WORKLOAD = ("FEL per-site fits: 256-taxon random unrooted tree (509 branches), 2000 simulated codons, "
                "every branch tested; per site the reference's 12-point grid, bounded Nelder-Mead on (alpha, beta), "
                "null grid + Brent on alpha = beta, LRT and p-value")


def _fel_inputs(h, aln, p):
    """pi, Qs (alpha=1, beta=0) and Qn (alpha=0, beta=1) rate matrices of the base model, zero diagonals."""
    ps, pn = h.MG94Parameters(), h.MG94Parameters()
    for q in (ps, pn):
        q.theta_AC, q.theta_AT, q.theta_CG, q.theta_CT, q.theta_GT = p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT
    ps.alpha, ps.beta, pn.alpha, pn.beta = 1.0, 0.0, 0.0, 1.0
    qs = np.array(h.mg94_eigensystem(aln, ps)["Q"])
    qn = np.array(h.mg94_eigensystem(aln, pn)["Q"])
    np.fill_diagonal(qs, 0.0)
    np.fill_diagonal(qn, 0.0)
    return np.asarray(aln.codon_frequencies), qs, qn


def run_fel(args) -> None:
    """FEL (or, with --analysis meme, MEME) per-site fits of the 256-taxon / 2000-codon workload through
    h3g_fel_run / h3g_meme_run (FP64)."""
    meme = args.analysis == "meme"
    import torch
    import _hyphy3 as h
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    wl = make_workload(2, n_sites=args.sites)
    aln = h.Alignment.from_sequences(wl.names, wl.seqs)
    tree = h.Tree.from_newick(wl.newick)
    p = h.MG94Parameters()
    p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = wl.theta
    p.beta = float(np.dot(wl.omegas, wl.omega_w))
    fel = h.FELAnalyzer(tree, aln, p)
    conv = fel.conversion_factor
    ctx = _capi.Context(0)
    states, masks, weights = aln.pattern_arrays()
    l2t = h.build_leaf_to_taxon_map(tree, aln)
    n = tree.num_nodes()
    is_leaf = np.array([nd.is_leaf for nd in tree.nodes], dtype=np.uint8)
    pr = _capi.Problem(ctx, np.array(tree.parents, dtype=np.int32), is_leaf,
                       np.array([l2t[i] if is_leaf[i] else -1 for i in range(n)], dtype=np.int32), states, masks, weights)
    pi, qs, qn = _fel_inputs(h, aln, p)
    bl = np.array(tree.get_branch_lengths()) * conv
    steps = max(3, min(args.steps, 5))
    fit = (lambda: pr.meme_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=bl)) if meme else \
          (lambda: pr.fel_run(pi=pi, Qs=qs, Qn=qn, branch_lengths=bl))
    out = fit()                                                          # warm-up
    if args.profile:                                                     # one more run, nothing else (for ncu)
        out = fit()
        ms, launches = pr.last_stats()
        print(json.dumps({"profile": args.analysis, "sites": wl.n_sites, "ms": ms, "gpu_launches": launches}), flush=True)
        pr.close()
        ctx.close()
        return
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        out = fit()
        times.append(time.perf_counter() - t0)
    clocks = sampler.stop()
    h2d, d2h = pr.last_transfer()
    launches = pr.last_stats()[1]
    secs = statistics.median(times)
    sites = wl.n_sites
    evals = float(np.dot(out["evaluations"], weights))
    branches = n - 1
    value = sites / secs
    t0 = time.perf_counter()
    res = h.MEMEAnalyzer(tree, aln, p).run() if meme else fel.run()
    e2e_secs = time.perf_counter() - t0
    cpu = None
    if not args.no_cpu:
        import h3oracle as o
        oa = o.Alignment.from_sequences(wl.names, wl.seqs)
        ot = o.Tree.parse(wl.newick)
        cls = {"alpha": 1.0, "beta": p.beta, "theta": list(wl.theta)}
        threads = o.max_threads()
        o.set_threads(threads)
        # a MEME site costs the oracle ~100x a FEL site: one pattern per thread, a few threads
        k = min(threads, 4) if meme else max(threads, 16)
        run_cpu = o.meme_run if meme else o.fel_run
        o.fel_run(ot, oa, cls, 2)
        t0 = time.perf_counter()
        r = run_cpu(ot, oa, cls, k)
        cs = time.perf_counter() - t0
        fitted = int(np.sum(np.array(r["evals"]) > 0))
        cpu = {"value": k / cs, "unit": "sites/s", "cores": min(threads, k) if meme else threads, "kind": "port",
               "sample": f"the first {k} patterns ({fitted} fitted, the rest invariant) of the same alignment, "
                         f"{cs:.1f} s (oracle restatement of {'meme.hpp' if meme else 'fel.hpp'} with the "
                         f"reference's optimisers)"}
    line = {
        "metric": MEME_METRIC if meme else FEL_METRIC, "value": value, "unit": "sites/s", "n_gpus": 1, "steps": steps,
        "warmup": 1,
        "ms_per_step": secs * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": MEME_WORKLOAD if meme else FEL_WORKLOAD, "sites": sites, "patterns": aln.num_patterns,
                   "branches": branches},
        "site_branch_lnl_evals_per_s": evals * branches / secs,
        "evaluations_per_site": evals / sites,
        "e2e": {"value": sites / e2e_secs, "unit": "sites/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "api": f"hyphy3.{'MEMEAnalyzer' if meme else 'FELAnalyzer'}(tree, aln, params).run()"},
        "cpu_baseline": cpu,
        "significant_at_0.1": int(sum(1 for r in res if r.p_value <= 0.1)),
        "clocks": clocks, "gpu_launches": int(launches),
        "timing": f"host wall clock around each blocking {'h3g_meme_run' if meme else 'h3g_fel_run'} (median of steps)",
    }
    print(json.dumps(line), flush=True)
    pr.close()
    ctx.close()


COMPRESS_METRIC = "alignment cells (taxon x codon) translated and compressed to site patterns per second"
COMPRESS_WORKLOAD = ("Alignment::finalize on the device: 1024 taxa x 100000 codons, columns resampled with replacement "
                     "from a simulated 1024-taxon Yule alignment of 5000 codons; codon translation, positional nucleotide "
                     "counts, site patterns in first-occurrence order")


def _compress_rows(n_codons: int):
    """[1024, 3 n_codons] uint8 rows: columns of the 1024-taxon simulated alignment drawn with replacement."""
    from hyphy3.simulate import make_workload
    wl = make_workload(3)
    T = len(wl.seqs)
    base = np.frombuffer(b"".join(x.encode() for x in wl.seqs), np.uint8).reshape(T, -1, 3)
    cols = np.random.default_rng(SEED_COMPRESS).integers(0, base.shape[1], n_codons)
    return np.ascontiguousarray(base[:, cols, :].reshape(T, -1))


SEED_COMPRESS = 20261204


def run_compress(args) -> None:
    """h3g_alignment_compress_device on device-resident rows (value) and h3g_alignment_compress from
    pinned host rows (e2e); the oracle's finalize on the same rows as the CPU baseline."""
    import ctypes as C
    import torch
    from hyphy3 import _capi
    n_codons = args.sites or 100000
    rows = _compress_rows(n_codons)
    T, L = rows.shape
    cells = T * n_codons
    stream = torch.cuda.current_stream()
    ctx = _capi.Context(0, stream=stream.cuda_stream)
    lib = ctx.lib
    sense = np.full(64, -1, np.int8)
    from hyphy3.simulate import universal_code
    codons, _ = universal_code()
    for i, cod in enumerate(codons):
        sense[16 * cod[0] + 4 * cod[1] + cod[2]] = i
    code = _capi.GeneticCodeDesc(S=len(codons), codon_to_sense=sense.ctypes.data_as(C.POINTER(C.c_int8)))
    d_rows = torch.from_numpy(rows).cuda()
    d_s2p = torch.empty(n_codons, dtype=torch.int32, device="cuda")
    d_w = torch.empty(n_codons, dtype=torch.int32, device="cuda")
    d_first = torch.empty(n_codons, dtype=torch.int32, device="cuda")
    d_st = torch.empty(n_codons * T, dtype=torch.int8, device="cuda")
    d_mk = torch.empty(n_codons * T, dtype=torch.int64, device="cuda")
    info = _capi.CompressInfo()
    vp = C.c_void_p

    def dev_call(profile=0):
        info.profile = profile
        ctx.check(lib.h3g_alignment_compress_device(ctx.h, T, L, vp(d_rows.data_ptr()), L, C.byref(code), vp(d_s2p.data_ptr()),
                                                    vp(d_w.data_ptr()), vp(d_first.data_ptr()), vp(d_st.data_ptr()),
                                                    vp(d_mk.data_ptr()), C.byref(info)))

    warm = max(3, args.warmup)
    for _ in range(warm):
        dev_call()
    torch.cuda.synchronize()
    if args.profile:                                                     # one more call, nothing else (for ncu)
        dev_call()
        torch.cuda.synchronize()
        print(json.dumps({"profile": "compress", "codons": n_codons, "patterns": int(info.n_patterns),
                          "gpu_launches": int(info.launches)}), flush=True)
        ctx.close()
        return
    steps = max(3, min(args.steps, 50))
    # stage times of the library's own events (one profiled call per step, outside the timed loop)
    stage = np.zeros(4)
    for _ in range(steps):
        dev_call(profile=1)
        stage += np.array(info.stage_ms[:])
    stage /= steps
    sampler = ClockSampler(0)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        dev_call()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1) / steps
    P = int(info.n_patterns)
    launches = int(info.launches)
    # e2e: the C ABI with host buffers (pinned), copies in the timed region
    h_rows = torch.from_numpy(rows).pin_memory()
    h_s2p = torch.empty(n_codons, dtype=torch.int32).pin_memory()
    h_w = torch.empty(n_codons, dtype=torch.int32).pin_memory()
    h_first = torch.empty(n_codons, dtype=torch.int32).pin_memory()
    h_st = torch.empty(n_codons * T, dtype=torch.int8).pin_memory()
    h_mk = torch.empty(n_codons * T, dtype=torch.int64).pin_memory()
    i32 = C.POINTER(C.c_int32)

    def host_call():
        ctx.check(lib.h3g_alignment_compress(ctx.h, T, L, vp(h_rows.data_ptr()), L, C.byref(code), C.cast(h_s2p.data_ptr(), i32),
                                             C.cast(h_w.data_ptr(), i32), C.cast(h_first.data_ptr(), i32),
                                             C.cast(h_st.data_ptr(), C.POINTER(C.c_int8)),
                                             C.cast(h_mk.data_ptr(), C.POINTER(C.c_uint64)), C.byref(info)))

    host_call()
    e2e = []
    for _ in range(steps):
        t0 = time.perf_counter()
        host_call()
        e2e.append(time.perf_counter() - t0)
    e2e_s = statistics.median(e2e)
    assert np.array_equal(h_s2p.numpy(), d_s2p.cpu().numpy()) and int(info.n_patterns) == P
    # roofline of the dominant stage: algorithmic bytes per call
    dup_cells = T * (n_codons - P)
    algo = {"translate": 5 * cells,                                      # 3 B read, 2 B key written per cell
            "rounds": 4 * dup_cells + 24 * n_codons,                    # keys of a duplicate and of its first column; hash/table
            "numbering": 16 * n_codons,
            "output": 16 * n_codons + 11 * P * T}                       # site map, weights; 2 B read + 9 B written per pattern cell
    names = ["translate", "rounds", "numbering", "output"]
    k = int(np.argmax(stage))
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = algo[names[k]] / (stage[k] * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu:
        import h3oracle as o
        seqs = [bytes(r).decode("latin-1") for r in rows]
        t0 = time.perf_counter()
        ref = o.Alignment.from_sequences([f"t{i}" for i in range(T)], seqs, "Universal")
        cs = time.perf_counter() - t0
        ok = ref.num_patterns == P and np.array_equal(np.asarray(ref.site_pattern), h_s2p.numpy())
        cpu = {"value": cells / cs, "unit": "cells/s", "cores": 1, "kind": "port",
               "sample": f"the whole workload ({cells} cells), {cs:.1f} s, one thread: the oracle's restatement of "
                         f"alignment.hpp:665-722, 1021-1078 (std::map of translated columns); same patterns: {ok}"}
    line = {
        "metric": COMPRESS_METRIC, "value": cells / (ms * 1e-3), "unit": "cells/s", "n_gpus": 1, "steps": steps,
        "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/u64",
        "data": "synthetic",
        "config": {"workload": COMPRESS_WORKLOAD, "taxa": T, "codons": n_codons, "patterns": P,
                   "l2": "inputs (307 MB) and keys (205 MB) larger than L2, no flush"},
        "e2e": {"value": cells / e2e_s, "unit": "cells/s", "h2d_bytes_per_step": int(rows.nbytes),
                "d2h_bytes_per_step": int(4 * n_codons + 8 * P + 9 * P * T),
                "api": "h3g_alignment_compress (C ABI, pinned host buffers)", "timing": "host wall clock, median"},
        "gpu_launches": launches * steps,
        "stage_ms": dict(zip(names, map(float, stage))),
        "roofline": {"bound": "hbm", "kernel": names[k], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None, "traffic": MEASURED_TRAFFIC.get(("compress", names[k])),
                     "traffic_unit": "bytes per call (the stage's launches), from ncu",
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                     "algorithmic_bytes": algo[names[k]]},
        "cpu_baseline": cpu, "clocks": clocks,
        "timing": "CUDA events on the launching stream around the timed calls (each call reads its round count back)",
    }
    print(json.dumps(line), flush=True)
    ctx.close()


GTR_METRIC = "nucleotide GTR pattern x branch log-likelihood evaluations per second"
GTR_WORKLOAD = ("LikelihoodEngine::compute_gtr_log_likelihood: the simulated 1024-taxon Yule alignment (5000 codons = "
                "15000 nucleotide sites), its nucleotide patterns, GTR at the simulation's exchangeabilities")


def run_gtr(args) -> None:
    """h3g_nuc_eval_from_P on the nucleotide patterns of the 1024-taxon workload (value), the public
    compute_gtr_log_likelihood from host objects (e2e), the oracle on the host's threads (CPU baseline)."""
    import ctypes as C
    import torch
    import _hyphy3 as h
    from hyphy3 import _capi
    from hyphy3.simulate import make_workload
    wl = make_workload(3)
    aln = h.Alignment.from_sequences(wl.names, wl.seqs)
    nuc = aln.to_nucleotide_alignment()
    tree = h.Tree.from_newick(wl.newick)
    gp = h.GTRParameters()
    gp.theta_AC, gp.theta_AT, gp.theta_CG, gp.theta_CT, gp.theta_GT = wl.theta
    g = h.GTRMatrix()
    g.update(gp, list(nuc.nuc_frequencies))
    stream = torch.cuda.current_stream()
    ctx = _capi.Context(0, stream=stream.cuda_stream)
    states, masks, weights = nuc.pattern_arrays()
    l2t = h.build_leaf_to_taxon_map(tree, nuc)
    n = tree.num_nodes()
    is_leaf = np.array([nd.is_leaf for nd in tree.nodes], dtype=np.uint8)
    pr = _capi.Problem(ctx, np.array(tree.parents, dtype=np.int32), is_leaf,
                       np.array([l2t[i] if is_leaf[i] else -1 for i in range(n)], dtype=np.int32), states, masks, weights)
    bl = tree.get_branch_lengths()
    P = np.zeros((n, 4, 4))
    for i in range(n):
        if i != tree.root_id:
            P[i] = g.transition_matrix(bl[i])
    pi = np.ascontiguousarray(g.pi, dtype=np.float64)
    lnl = C.c_double()
    dp = C.POINTER(C.c_double)

    def call():
        ctx.check(ctx.lib.h3g_nuc_eval_from_P(pr.h, P.ctypes.data_as(dp), pi.ctypes.data_as(dp), C.byref(lnl), None))

    warm = max(3, args.warmup)
    for _ in range(warm):
        call()
    if args.profile:
        call()
        print(json.dumps({"profile": "gtr", "patterns": int(nuc.num_patterns), "lnl": lnl.value}), flush=True)
        pr.close()
        ctx.close()
        return
    steps = max(3, min(args.steps, 200))
    sampler = ClockSampler(0)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        call()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1) / steps
    Pn, T, branches = int(nuc.num_patterns), int(nuc.num_taxa), n - 1
    units = Pn * branches
    # e2e: the public API from host objects (transition matrices built on the host, cached device problem)
    e2e = []
    for _ in range(min(steps, 10)):
        t0 = time.perf_counter()
        l_api, _site = h.compute_gtr_log_likelihood(tree, nuc, g)
        e2e.append(time.perf_counter() - t0)
    e2e_s = statistics.median(e2e)
    internal = sum(1 for nd in tree.nodes if not nd.is_leaf)
    algo = Pn * (T * 1 + 2 * 36 * (internal - 1) + 8)                   # leaf states; partials parked and restored; site
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = algo / (ms * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu:
        import h3oracle as o
        threads = o.max_threads()
        o.set_threads(threads)
        onuc = o.nucleotide_patterns(o.Alignment.from_sequences(wl.names, wl.seqs))
        ot = o.Tree.parse(wl.newick)
        t0 = time.perf_counter()
        l_ref, _ = o.gtr_loglik(ot, onuc, list(wl.theta), list(nuc.nuc_frequencies))
        cs = time.perf_counter() - t0
        cpu = {"value": units / cs, "unit": "pattern*branch/s", "cores": threads, "kind": "port",
               "sample": f"the whole workload, {cs:.2f} s on {threads} threads (oracle restatement of likelihood.hpp:181-254); "
                         f"lnL {l_ref:.6f} vs device {lnl.value:.6f}"}
    line = {
        "metric": GTR_METRIC, "value": units / (ms * 1e-3), "unit": "pattern*branch/s", "n_gpus": 1, "steps": steps,
        "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": GTR_WORKLOAD, "taxa": T, "nucleotide_sites": int(nuc.num_nucleotides), "patterns": Pn,
                   "branches": branches, "l2": "partial stack L2-resident; no flush"},
        "e2e": {"value": units / e2e_s, "unit": "pattern*branch/s", "h2d_bytes_per_step": int(P.nbytes + 32),
                "d2h_bytes_per_step": int(8 + 8 * Pn), "api": "_hyphy3.compute_gtr_log_likelihood(tree, nuc_aln, gtr)",
                "timing": "host wall clock, median"},
        "gpu_launches": 2 * steps, "lnl": lnl.value, "api_lnl": l_api,
        "roofline": {"bound": "hbm", "kernel": "k_nuc_lnl", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": MEASURED_TRAFFIC.get(("gtr", "k_nuc_lnl")),
                     "traffic_unit": "bytes per launch, from ncu", "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                     "algorithmic_bytes": algo, "note": "the call (P upload, two kernels, lnL read back) timed as a whole"},
        "cpu_baseline": cpu, "clocks": clocks,
        "timing": "CUDA events on the launching stream around the timed calls",
    }
    print(json.dumps(line), flush=True)
    pr.close()
    ctx.close()


def _mixed_available() -> bool:
    return os.environ.get("H3G_BENCH_PRECISION", "mixed") == "mixed"


def _directions(aln, wl, es):
    """dQ/d omega_k (one class each) and dQ/d theta_x (all classes), shape [8, K, S, S]."""
    from hyphy3.simulate import universal_code
    codons, aas = universal_code()
    pos = np.asarray(aln.pos_nuc_frequencies)
    S = len(codons)
    AC, AT, CG, CT, GT = wl.theta
    r = np.array([[0, AC, 1, AT], [AC, 0, CG, CT], [1, CG, 0, GT], [AT, CT, GT, 0]], dtype=float)
    single = np.zeros((S, S), dtype=bool)
    frm = np.zeros((S, S), dtype=int)
    to = np.zeros((S, S), dtype=int)
    ps = np.zeros((S, S), dtype=int)
    syn = np.zeros((S, S), dtype=bool)
    for i, ci in enumerate(codons):
        for j, cj in enumerate(codons):
            d = [q for q in range(3) if ci[q] != cj[q]]
            if len(d) == 1:
                single[i, j] = True
                ps[i, j], frm[i, j], to[i, j] = d[0], ci[d[0]], cj[d[0]]
                syn[i, j] = aas[i] == aas[j]
    K = len(es)
    out = []
    for k in range(K):
        dq = np.zeros((K, S, S))
        m = single & ~syn
        dq[k][m] = r[frm[m], to[m]] * pos[ps[m], to[m]]
        dq[k][np.diag_indices(S)] = -dq[k].sum(1)
        out.append(dq)
    pairs = [(0, 1), (0, 3), (1, 2), (1, 3), (2, 3)]
    for (u, v) in pairs:
        dq = np.zeros((K, S, S))
        m = single & (((frm == u) & (to == v)) | ((frm == v) & (to == u)))
        for k, om in enumerate(wl.omegas):
            rate = np.where(syn, 1.0, om)
            dq[k][m] = rate[m] * pos[ps[m], to[m]]
            dq[k][np.diag_indices(S)] = -dq[k].sum(1)
        out.append(dq)
    return np.stack(out)


def run_profile(args) -> None:
    """Evaluations only (no CPU leg, no API leg, no clock sampling): the command ncu captures."""
    import torch
    h, wl, aln, tree = build_inputs(config=args.config, sites=args.sites)
    from hyphy3 import _capi
    ctx = _capi.Context(0)
    states, masks, weights = aln.pattern_arrays()
    l2t = h.build_leaf_to_taxon_map(tree, aln)
    n = tree.num_nodes()
    is_leaf = np.array([nd.is_leaf for nd in tree.nodes], dtype=np.uint8)
    pr = _capi.Problem(ctx, np.array(tree.parents, dtype=np.int32), is_leaf,
                       np.array([l2t[i] if is_leaf[i] else -1 for i in range(n)], dtype=np.int32), states, masks, weights)
    es = []
    for om in wl.omegas:
        p = h.MG94Parameters()
        p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT = wl.theta
        p.beta = om
        es.append(h.mg94_eigensystem(aln, p))
    prec = _capi.PREC_FP64 if args.precision == "fp64" else _capi.PREC_MIXED
    pr.set_model(pi=aln.codon_frequencies, Q=np.stack([e["Q"] for e in es]), lam=np.stack([e["lam"] for e in es]),
                 U=np.stack([e["U"] for e in es]), V=np.stack([e["V"] for e in es]), mu=np.array([e["mu"] for e in es]),
                 class_w=wl.omega_w, rates=list(wl.rates), rate_w=list(wl.rate_w), dQ=_directions(aln, wl, es),
                 precision=prec)
    pr.stage_branch_lengths(np.array(tree.get_branch_lengths()))
    want = _capi.WANT_LNL | _capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL
    for _ in range(args.warmup + args.steps):
        pr.eval_resident(want)
    r = pr.read_result(want)
    torch.cuda.synchronize()
    print(f"profile run: precision={args.precision} lnL={r['lnl']:.6f} launches/eval={pr.last_stats()[1]}")
    pr.close()
    ctx.close()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["auto", "fp64", "mixed"], default="auto")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--profile", action="store_true", help="device evaluations only (for ncu)")
    ap.add_argument("--sites", type=int, default=None, help="shrink the alignment to this many codons (--profile; --config 2)")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (heuristic launch shapes)")
    ap.add_argument("--memory-budget", type=float, default=0.0,
                    help="GB one evaluation workspace may take (subtree checkpointing below the full size)")
    ap.add_argument("--mode", choices=["sharded", "replicas"], default="sharded",
                    help="N > 1 GPUs: split one alignment's patterns over the ranks (NCCL all-reduce per step), or "
                         "run an independent replica per rank (no collective)")
    ap.add_argument("--genes", type=int, default=None, help="--config 4: number of genes (default 500)")
    ap.add_argument("--slots", type=int, default=8, help="--config 4: batch slot workspaces (concurrent streams)")
    ap.add_argument("--fit-iters", type=int, default=20, help="--config 4: L-BFGS iterations of the joint fit")
    ap.add_argument("--config", type=int, choices=[1, 2, 3, 4], default=3,
                    help="1: 64-taxon 3-omega mixture; 2: FEL per-site fits, 256 taxa x 2000 codons; "
                         "3: 1024-taxon, 4 rate x 2 omega classes (headline: the largest single-GPU workload); "
                         "4: 500 uneven genes in one batch")
    ap.add_argument("--analysis", choices=["fel", "meme", "compress", "gtr"], default="fel",
                    help="--config 2: which per-site analysis; compress: alignment finalize on the device; "
                         "gtr: nucleotide GTR likelihood (both any config)")
    args = ap.parse_args()
    if args.analysis == "compress" and args.impl == "ours":
        run_compress(args)
    elif args.analysis == "gtr" and args.impl == "ours":
        run_gtr(args)
    elif args.config == 2 and args.impl == "ours":
        run_fel(args)
    elif args.config == 4 and args.impl == "ours":
        run_batch(args)
    elif args.profile:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
