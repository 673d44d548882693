"""Shared helpers for the device parity tests: feed the oracle's inputs through the C ABI."""
import numpy as np


def problem_from_oracle(ctx, oracle, tree, aln):
    from hyphy3 import _capi
    l2t = oracle.leaf_map(tree, aln)
    n = tree.num_nodes()
    leaf = np.array(tree.is_leaf, dtype=np.uint8)
    taxon = np.array([l2t[i] if leaf[i] else -1 for i in range(n)], dtype=np.int32)
    return _capi.Problem(ctx, np.array(tree.parent, dtype=np.int32), leaf, taxon, aln.states, aln.masks,
                         np.array(aln.weights))


def eigensystems(oracle, aln, params_list):
    es = [oracle.mg94(aln, p) for p in params_list]
    return (np.stack([e["Q"] for e in es]), np.stack([e["lam"] for e in es]), np.stack([e["U"] for e in es]),
            np.stack([e["V"] for e in es]), np.array([e["mu"] for e in es]))


def dq_beta(oracle_code_aln, p):
    """dQ/dbeta for a MG94 model (single-nucleotide non-synonymous changes)."""
    from hyphy3.simulate import universal_code
    codons, aas = universal_code()
    pos = np.asarray(oracle_code_aln.pos_freq)
    AC, AT, CG, CT, GT = p["theta"]
    r = np.array([[0, AC, 1, AT], [AC, 0, CG, CT], [1, CG, 0, GT], [AT, CT, GT, 0]], dtype=float)
    S = len(codons)
    d = np.zeros((S, S))
    for i, ci in enumerate(codons):
        for j, cj in enumerate(codons):
            diff = [q for q in range(3) if ci[q] != cj[q]]
            if len(diff) == 1 and aas[i] != aas[j]:
                q = diff[0]
                d[i, j] = r[ci[q], cj[q]] * pos[q][cj[q]]
    d[np.diag_indices(S)] = -d.sum(1)
    return d


def dq_theta(aln, x, p):
    from hyphy3.simulate import universal_code
    pairs = [(0, 1), (0, 3), (1, 2), (1, 3), (2, 3)]
    u, v = pairs[x]
    codons, aas = universal_code()
    pos = np.asarray(aln.pos_freq)
    S = len(codons)
    d = np.zeros((S, S))
    for i, ci in enumerate(codons):
        for j, cj in enumerate(codons):
            diff = [q for q in range(3) if ci[q] != cj[q]]
            if len(diff) != 1:
                continue
            q = diff[0]
            f, t = ci[q], cj[q]
            if (f, t) in ((u, v), (v, u)):
                d[i, j] = (p["alpha"] if aas[i] == aas[j] else p["beta"]) * pos[q][t]
    d[np.diag_indices(S)] = -d.sum(1)
    return d


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def ranks(v):
    """Average ranks with ties closer than 1e-12 (tests/test_fel_multi_dataset.cpp:22-44)."""
    order = np.argsort(v, kind="stable")
    r = np.empty(len(v))
    i = 0
    while i < len(v):
        j = i + 1
        while j < len(v) and abs(v[order[j]] - v[order[i]]) < 1e-12:
            j += 1
        r[order[i:j]] = 0.5 * (i + j - 1) + 1.0
        i = j
    return r
