"""Seeded synthetic workloads: random trees and codon alignments simulated under MG94xREV.

The benchmark and parity workloads are synthetic stand-ins shaped like the
reference's use of its likelihood core: a random unrooted binary tree (or a
Yule tree), codon sites simulated down it under MG94xREV with omega and
synonymous-rate site classes, F3x4 generator frequencies drawn from
Dirichlet(1) per codon position, GTR exchangeabilities ~ U(0.5, 2), and a
fraction of gap and single-nucleotide-ambiguity codons.  The alignment text
is then compressed by the library's own loader (CF3x4 frequencies and
patterns, as alignment.hpp:893-1078 does).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

NUC = "ACGT"
# NCBI table 1 amino acids in T,C,A,G-major codon order, the order it is usually printed in
_TCAG_TABLE = "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG"
_TCAG_POS = {0: 2, 1: 1, 2: 3, 3: 0}  # A C G T -> index in T C A G


def universal_code():
    """Sense codons (ACGT-major order) and their amino acids."""
    codons, aas = [], []
    for c in range(64):
        a, b, d = c >> 4, (c >> 2) & 3, c & 3
        aa = _TCAG_TABLE[16 * _TCAG_POS[a] + 4 * _TCAG_POS[b] + _TCAG_POS[d]]
        if aa != "*":
            codons.append((a, b, d))
            aas.append(aa)
    return codons, aas


def mg94_generator(theta, omega, pos_freq, alpha=1.0):
    """MG94xREV generator with single-nucleotide changes (rate_matrix.hpp:165-227)."""
    codons, aas = universal_code()
    S = len(codons)
    AC, AT, CG, CT, GT = theta
    r = np.array([[0, AC, 1, AT], [AC, 0, CG, CT], [1, CG, 0, GT], [AT, CT, GT, 0]], dtype=float)
    Q = np.zeros((S, S))
    for i, ci in enumerate(codons):
        for j, cj in enumerate(codons):
            diff = [p for p in range(3) if ci[p] != cj[p]]
            if len(diff) != 1:
                continue
            p = diff[0]
            w = alpha if aas[i] == aas[j] else omega
            Q[i, j] = w * r[ci[p], cj[p]] * pos_freq[p][cj[p]]
    Q[np.diag_indices(S)] = -Q.sum(1)
    pi = np.array([pos_freq[0][c[0]] * pos_freq[1][c[1]] * pos_freq[2][c[2]] for c in codons])
    return Q, pi / pi.sum()


class ReversibleExp:
    """exp(Q t) for a reversible Q via one symmetrised eigendecomposition."""

    def __init__(self, Q, pi):
        s = np.sqrt(np.maximum(pi, 1e-12))
        A = (s[:, None] * Q) / s[None, :]
        lam, E = np.linalg.eigh(0.5 * (A + A.T))
        self.lam = np.minimum(lam, 0.0)
        self.L = E / s[:, None]
        self.R = E.T * s[None, :]

    def __call__(self, t):
        return np.maximum(self.L @ (np.exp(self.lam * t)[:, None] * self.R), 0.0)


def expm_sym(Q, pi, t):
    """exp(Q t) for a reversible Q via the symmetrised eigenproblem."""
    return ReversibleExp(Q, pi)(t)


@dataclasses.dataclass
class TreeSpec:
    parent: list[int]
    length: list[float]
    names: list[str]          # leaf names ('' for internal nodes)

    def newick(self) -> str:
        kids = [[] for _ in self.parent]
        root = -1
        for i, p in enumerate(self.parent):
            if p < 0:
                root = i
            else:
                kids[p].append(i)

        def rec(u):
            if not kids[u]:
                s = self.names[u]
            else:
                s = "(" + ",".join(rec(c) for c in kids[u]) + ")"
            if u != root:
                s += f":{self.length[u]:.10g}"
            return s
        return rec(root) + ";"


def random_unrooted_tree(n_taxa: int, rng: np.random.Generator, mean_bl: float) -> TreeSpec:
    """Uniform random unrooted binary topology by sequential edge insertion, trifurcating root."""
    if n_taxa < 3:
        raise ValueError("need at least 3 taxa")
    parent = [-1, 0, 0, 0]
    names = ["", "T1", "T2", "T3"]
    for k in range(4, n_taxa + 1):
        edges = [i for i, p in enumerate(parent) if p >= 0]
        e = edges[int(rng.integers(len(edges)))]
        mid = len(parent)
        parent.append(parent[e])
        names.append("")
        parent[e] = mid
        parent.append(mid)
        names.append(f"T{k}")
    length = [0.0 if p < 0 else float(rng.exponential(mean_bl)) for p in parent]
    return TreeSpec(parent, length, names)


def yule_tree(n_taxa: int, rng: np.random.Generator, mean_bl: float) -> TreeSpec:
    """Pure-birth topology (random leaf splits), then the root collapsed to a trifurcation."""
    parent = [-1, 0, 0]
    leaves = [1, 2]
    while len(leaves) < n_taxa:
        i = int(rng.integers(len(leaves)))
        u = leaves.pop(i)
        a, b = len(parent), len(parent) + 1
        parent += [u, u]
        leaves += [a, b]
    # unroot: absorb an internal child of the root
    kids0 = [i for i, p in enumerate(parent) if p == 0]
    absorb = next((c for c in kids0 if any(p == c for p in parent)), None)
    if absorb is not None:
        for i, p in enumerate(parent):
            if p == absorb:
                parent[i] = 0
        parent[absorb] = -2  # removed
    keep = [i for i, p in enumerate(parent) if p != -2]
    remap = {old: new for new, old in enumerate(keep)}
    new_parent = [-1 if parent[o] < 0 else remap[parent[o]] for o in keep]
    is_leaf = [not any(p == i for p in new_parent) for i in range(len(new_parent))]
    names, k = [], 0
    for i in range(len(new_parent)):
        if is_leaf[i]:
            k += 1
            names.append(f"T{k}")
        else:
            names.append("")
    length = [0.0 if p < 0 else float(rng.exponential(mean_bl)) for p in new_parent]
    return TreeSpec(new_parent, length, names)


def simulate_alignment(tree: TreeSpec, n_sites: int, rng: np.random.Generator, *, theta, pos_freq,
                       omegas=(0.5,), omega_w=(1.0,), rates=(1.0,), rate_w=(1.0,),
                       gap_frac=0.0, ambig_frac=0.0) -> tuple[list[str], list[str]]:
    """Codon sequences for the leaves of `tree` (names, sequences)."""
    codons, _ = universal_code()
    n = len(tree.parent)
    kids = [[] for _ in range(n)]
    root = -1
    for i, p in enumerate(tree.parent):
        if p < 0:
            root = i
        else:
            kids[p].append(i)
    order = [root]
    for u in order:
        order.extend(kids[u])
    site_om = rng.choice(len(omegas), size=n_sites, p=np.asarray(omega_w) / np.sum(omega_w))
    site_rt = rng.choice(len(rates), size=n_sites, p=np.asarray(rate_w) / np.sum(rate_w))
    gens = [mg94_generator(theta, om, pos_freq) for om in omegas]
    exps = [ReversibleExp(Q, pik) for Q, pik in gens]
    pi = gens[0][1]
    states = np.zeros((n, n_sites), dtype=np.int64)
    states[root] = rng.choice(len(pi), size=n_sites, p=pi)
    for u in order[1:]:
        par = tree.parent[u]
        u_rand = rng.random(n_sites)
        for k, (Q, pik) in enumerate(gens):
            for m, r in enumerate(rates):
                sel = np.flatnonzero((site_om == k) & (site_rt == m))
                if sel.size == 0:
                    continue
                cum = np.cumsum(exps[k](r * tree.length[u]), axis=1)
                cum /= cum[:, -1:]
                rows = cum[states[par, sel]]
                states[u, sel] = np.minimum((rows < u_rand[sel, None]).sum(1), len(pi) - 1)
    names, seqs = [], []
    if ambig_frac == 0.0:
        # vectorised text: one uniform draw per (leaf, site) in the same order as the loop below,
        # so the sequences are identical to it
        table = np.array([NUC[a] + NUC[b] + NUC[c] for a, b, c in codons] + ["---"], dtype="S3")
        for u in range(n):
            if kids[u]:
                continue
            idx = states[u].copy()
            x = rng.random(n_sites)
            idx[x < gap_frac] = len(codons)
            names.append(tree.names[u])
            seqs.append(table[idx].tobytes().decode("ascii"))
        return names, seqs
    iupac_one = {0: "MRW", 1: "MSY", 2: "RSK", 3: "WYK"}  # codes containing the true base
    for u in range(n):
        if kids[u]:
            continue
        chars = []
        for s in range(n_sites):
            a, b, c = codons[states[u, s]]
            trip = [NUC[a], NUC[b], NUC[c]]
            x = rng.random()
            if x < gap_frac:
                trip = ["-", "-", "-"]
            elif x < gap_frac + ambig_frac:
                pos = int(rng.integers(3))
                nuc = "ACGT".index(trip[pos])
                trip[pos] = iupac_one[nuc][int(rng.integers(3))]
            chars.append("".join(trip))
        names.append(tree.names[u])
        seqs.append("".join(chars))
    return names, seqs


def gamma_rates(shape: float, k: int) -> np.ndarray:
    """Mean-one discrete gamma rates (category medians, renormalised)."""
    from scipy.stats import gamma
    q = (np.arange(k) + 0.5) / k
    r = gamma.ppf(q, a=shape, scale=1.0 / shape)
    return r / r.mean()


@dataclasses.dataclass
class Workload:
    name: str
    tree: TreeSpec
    names: list[str]
    seqs: list[str]
    theta: list[float]
    omegas: list[float]
    omega_w: list[float]
    rates: list[float]
    rate_w: list[float]

    @property
    def newick(self) -> str:
        return self.tree.newick()

    @property
    def n_sites(self) -> int:
        return len(self.seqs[0]) // 3


SEED_BASE = 20261203


def simulate_gene(tree: TreeSpec, n_sites: int, rng: np.random.Generator, *, theta, pos_freq, omega) -> tuple[list[str], list[str]]:
    """One-class MG94xREV codon sequences for the leaves of `tree`, sampled fast.

    Same model as simulate_alignment with one omega class and no gaps or ambiguity codes, but
    every node's states are drawn with one inverse-CDF search: the transition rows are laid end
    to end, row s shifted by s, so the child state of a site whose parent is in state s is found by
    searching s + u in the flattened cumulative table."""
    codons, _ = universal_code()
    n = len(tree.parent)
    kids = [[] for _ in range(n)]
    root = -1
    for i, p in enumerate(tree.parent):
        if p < 0:
            root = i
        else:
            kids[p].append(i)
    order = [root]
    for u in order:
        order.extend(kids[u])
    Q, pi = mg94_generator(theta, omega, pos_freq)
    expm = ReversibleExp(Q, pi)
    S = len(pi)
    shift = np.arange(S, dtype=float)[:, None]
    states = np.zeros((n, n_sites), dtype=np.int64)
    states[root] = rng.choice(S, size=n_sites, p=pi)
    for u in order[1:]:
        cum = np.cumsum(expm(tree.length[u]), axis=1)
        cum /= cum[:, -1:]
        flat = (cum + shift).ravel()
        par = states[tree.parent[u]]
        idx = np.searchsorted(flat, par + rng.random(n_sites), side="left")
        states[u] = np.clip(idx - par * S, 0, S - 1)
    table = np.array([NUC[a] + NUC[b] + NUC[c] for a, b, c in codons], dtype="S3")
    names, seqs = [], []
    for u in range(n):
        if not kids[u]:
            names.append(tree.names[u])
            seqs.append(table[states[u]].tobytes().decode("ascii"))
    return names, seqs


@dataclasses.dataclass
class Gene:
    tree: TreeSpec
    names: list[str]
    seqs: list[str]
    theta: list[float]
    omega: float

    @property
    def newick(self) -> str:
        return self.tree.newick()

    @property
    def n_sites(self) -> int:
        return len(self.seqs[0]) // 3


def make_gene_batch(n_genes: int = 500, *, taxa=(8, 512), sites=(100, 3000), seed: int | None = None) -> list[Gene]:
    """The uneven multi-gene workload: n_genes alignments with taxa ~ U{taxa}, codons ~ U{sites},
    each with its own random unrooted tree (branch lengths ~ Exp(mean 0.1)), GTR exchangeabilities
    ~ U(0.5, 2), F3x4 generator frequencies ~ Dirichlet(1) per position and omega ~ U(0.1, 1)."""
    rng = np.random.default_rng(SEED_BASE + 4 if seed is None else seed)
    out = []
    for _ in range(n_genes):
        nt = int(rng.integers(taxa[0], taxa[1] + 1))
        ns = int(rng.integers(sites[0], sites[1] + 1))
        theta = list(rng.uniform(0.5, 2.0, size=5))
        pos_freq = rng.dirichlet(np.ones(4), size=3)
        omega = float(rng.uniform(0.1, 1.0))
        tree = random_unrooted_tree(nt, rng, 0.1)
        names, seqs = simulate_gene(tree, ns, rng, theta=theta, pos_freq=pos_freq, omega=omega)
        out.append(Gene(tree, names, seqs, theta, omega))
    return out


def make_workload(config: int, *, n_sites: int | None = None, n_taxa: int | None = None) -> Workload:
    """Synthetic stand-ins for the five benchmark configurations (index 0..4); sizes may be shrunk for tests."""
    rng = np.random.default_rng(SEED_BASE + config)
    theta = list(rng.uniform(0.5, 2.0, size=5))
    pos_freq = rng.dirichlet(np.ones(4), size=3)
    if config == 0:
        nt, ns, mean, kind = 8, 300, 0.1, "random"
        omegas, ow, rates, rw, gap, amb = [0.5], [1.0], [1.0], [1.0], 0.0, 0.0
    elif config == 1:
        nt, ns, mean, kind = 64, 1000, 0.1, "random"
        omegas, ow, rates, rw, gap, amb = [0.1, 1.0, 5.0], [0.6, 0.3, 0.1], [1.0], [1.0], 0.03, 0.01
    elif config == 2:
        nt, ns, mean, kind = 256, 2000, 0.1, "random"
        omegas, ow, rates, rw, gap, amb = [0.3, 1.5], [0.7, 0.3], [1.0], [1.0], 0.0, 0.0
    elif config == 3:
        nt, ns, mean, kind = 1024, 5000, 0.05, "yule"
        omegas, ow = [0.2, 2.0], [0.8, 0.2]
        rates, rw = list(gamma_rates(0.5, 4)), [0.25] * 4
        gap, amb = 0.0, 0.0
    else:
        raise ValueError("config must be 0..3 (multi-gene batches are built by callers)")
    nt = n_taxa or nt
    ns = n_sites or ns
    tree = random_unrooted_tree(nt, rng, mean) if kind == "random" else yule_tree(nt, rng, mean)
    names, seqs = simulate_alignment(tree, ns, rng, theta=theta, pos_freq=pos_freq, omegas=omegas, omega_w=ow,
                                     rates=rates, rate_w=rw, gap_frac=gap, ambig_frac=amb)
    return Workload(f"config{config}", tree, names, seqs, theta, omegas, ow, rates, rw)
