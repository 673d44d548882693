"""aBSREL (adaptive branch-site random effects likelihood) on the device.

The reference's analysis (include/hyphy/analyses/absrel.hpp, run() :1355-2330): a nucleotide
GTR fit; a baseline MG94xREV model with one omega per branch (:812-1027); a step-up search that
gives each branch, longest first, as many omega classes (up to max_rate_classes) as the AICc
supports (:1400-1495); the full adaptive model; and per tested branch a likelihood-ratio test of
its largest omega against omega = 1, with the mixture p-value 0.2 erfc(sqrt(LRT/2)) +
0.3 exp(-LRT/2) (:433-435, stats.hpp:101-107) and Holm-Bonferroni correction (stats.hpp:157-181).

Every likelihood here is one device evaluation of the whole tree with per-branch omega mixtures
(h3g_model_desc.branch_classes: P_b = sum_k w_bk exp(t_b Q(omega_bk)), absrel.hpp:262-276),
whose gradients -- branch lengths, each class's omega (one per-class direction, dQ_model) and
weight, the five exchangeabilities -- drive bounded L-BFGS fits.  The reference fits the same
models by coordinate-wise refinements over cavity vectors of single branches; here each fit is
joint over its free parameters, so the path differs and the models and criteria are the same.
"""
from __future__ import annotations

import math

import numpy as np

from . import _capi
from .simulate import universal_code

# nucleotide pairs of the five free exchangeabilities (AC AT CG CT GT) and AG (fixed at 1)
_PAIR = {(0, 1): 0, (0, 3): 1, (1, 2): 2, (1, 3): 3, (2, 3): 4, (0, 2): 5}


class MG94Structure:
    """MG94xREV (alpha = 1) as linear combinations of fixed matrices of the universal code:
    Q(theta, omega) = sum_x theta_x (Syn_x + omega Non_x) off the diagonal, rows summing to 0, where
    Syn_x / Non_x hold pi^pos_to for the synonymous / non-synonymous single-nucleotide changes of
    pair x (rate_matrix.hpp:165-227).  dQ/domega and dQ/dtheta_x follow directly."""

    def __init__(self, pos_freq):
        codons, aas = universal_code()
        S = len(codons)
        pos = np.asarray(pos_freq, dtype=float)
        self.syn = np.zeros((6, S, S))
        self.non = np.zeros((6, S, S))
        for i, ci in enumerate(codons):
            for j, cj in enumerate(codons):
                d = [q for q in range(3) if ci[q] != cj[q]]
                if len(d) != 1:
                    continue
                q = d[0]
                f, t = ci[q], cj[q]
                x = _PAIR[(min(f, t), max(f, t))]
                (self.syn if aas[i] == aas[j] else self.non)[x, i, j] = pos[q, t]
        self.S = S

    @staticmethod
    def _rows(M):
        np.fill_diagonal(M, 0.0)
        np.fill_diagonal(M, -M.sum(1))
        return M

    def Q(self, theta, omega):
        th = np.append(np.asarray(theta, dtype=float), 1.0)
        return self._rows(np.tensordot(th, self.syn + omega * self.non, axes=1))

    def dQ_domega(self, theta):
        th = np.append(np.asarray(theta, dtype=float), 1.0)
        return self._rows(np.tensordot(th, self.non, axes=1))

    def dQ_dtheta(self, x, omega):
        return self._rows(self.syn[x] + omega * self.non[x])


class BranchMixtures:
    """Per-branch omega distributions (omegas, weights), raw-time branch lengths t and the five
    exchangeabilities; the root entries are unused."""

    def __init__(self, n, root, t, theta, omega0):
        self.n, self.root = n, root
        self.t = np.asarray(t, dtype=float).copy()
        self.theta = np.asarray(theta, dtype=float).copy()
        self.omegas = [[] if b == root else [float(omega0[b])] for b in range(n)]
        self.weights = [[] if b == root else [1.0] for b in range(n)]

    def copy(self):
        c = BranchMixtures.__new__(BranchMixtures)
        c.n, c.root, c.t, c.theta = self.n, self.root, self.t.copy(), self.theta.copy()
        c.omegas = [list(o) for o in self.omegas]
        c.weights = [list(w) for w in self.weights]
        return c

    def offsets(self):
        return np.concatenate([[0], np.cumsum([len(o) for o in self.omegas])]).astype(np.int32)

    def classes(self):
        return sum(len(o) for o in self.omegas)


def mixture_p_value(lrt: float) -> float:
    """0.2 erfc(sqrt(LRT / 2)) + 0.3 exp(-LRT / 2), 1 for LRT <= 0 (stats.hpp:101-107 with absrel.hpp:433-435)."""
    if not math.isfinite(lrt) or lrt <= 0.0:
        return 1.0
    v = 0.2 * math.erfc(math.sqrt(lrt / 2.0)) + 0.3 * math.exp(-lrt / 2.0)
    return min(max(v, 0.0), 1.0) if math.isfinite(v) else 1.0


def aicc(log_l: float, k: int, n_obs: int) -> float:
    """-2 lnL + 2 k n / (n - k - 1), or AIC when n <= k + 1 (stats.hpp:114-121)."""
    if n_obs > k + 1:
        return -2.0 * log_l + 2.0 * k * n_obs / (n_obs - k - 1.0)
    return -2.0 * log_l + 2.0 * k


def holm_bonferroni(p_values):
    """Holm's step-down adjusted p-values in input order (stats.hpp:157-181)."""
    p = [min(max(x, 0.0), 1.0) if math.isfinite(x) else 1.0 for x in p_values]
    m = len(p)
    order = sorted(range(m), key=lambda i: p[i])
    out = [1.0] * m
    run = 0.0
    for rank, i in enumerate(order):
        run = min(max(run, p[i] * (m - rank)), 1.0)
        out[i] = run
    return out


class ABSRELAnalyzer:
    """aBSREL on one alignment and tree (ABSRELAnalyzer, absrel.hpp:140-2339).

    tree, aln: _hyphy3.Tree and _hyphy3.Alignment.  Every branch is tested ("All", the reference's
    default); max_rate_classes and p_threshold as in ABSRELSettings (absrel.hpp:66-71)."""

    def __init__(self, tree, aln, *, max_rate_classes: int = 3, p_threshold: float = 0.05,
                 precision: str = "fp64", device: int = 0, max_iter: int = 300):
        import _hyphy3 as h
        self.h, self.tree, self.aln = h, tree, aln
        self.max_rate_classes, self.p_threshold, self.max_iter = max_rate_classes, p_threshold, max_iter
        self.prec = _capi.PREC_MIXED if precision == "mixed" else _capi.PREC_FP64
        states, masks, weights = aln.pattern_arrays()
        l2t = h.build_leaf_to_taxon_map(tree, aln)
        self.n = tree.num_nodes()
        self.root = tree.root_id
        is_leaf = np.array([nd.is_leaf for nd in tree.nodes], dtype=np.uint8)
        self.ctx = _capi.Context(device)
        self.pr = _capi.Problem(self.ctx, np.array(tree.parents, dtype=np.int32), is_leaf,
                                np.array([l2t[i] if is_leaf[i] else -1 for i in range(self.n)], dtype=np.int32),
                                states, masks, weights)
        self.struct = MG94Structure(np.asarray(aln.pos_nuc_frequencies))
        self.pi = np.asarray(aln.codon_frequencies)
        self.n_obs = int(aln.num_taxa) * int(aln.num_codons)
        self.branches = [b for b in range(self.n) if b != self.root]
        self.evaluations = 0

    def close(self):
        self.pr.close()
        self.ctx.close()

    # ---------------------------------------------------------------- likelihood
    def evaluate(self, m: BranchMixtures, grads: bool = True) -> dict:
        """lnL and, with grads, d lnL / d t (per node), d / d omega and d / d weight (per class in
        branch order) and d / d theta (5) -- one device evaluation."""
        omegas = [o for b in range(self.n) for o in m.omegas[b]]
        weights = [w for b in range(self.n) for w in m.weights[b]]
        Q = np.stack([self.struct.Q(m.theta, o) for o in omegas])
        kw = dict(pi=self.pi, Q=Q, class_w=np.asarray(weights), branch_classes=m.offsets(), precision=self.prec)
        if grads:
            kw["dQ"] = np.stack([np.stack([self.struct.dQ_dtheta(x, o) for o in omegas]) for x in range(5)])
            dq_om = self.struct.dQ_domega(m.theta)
            kw["dQ_model"] = np.broadcast_to(dq_om, (len(omegas),) + dq_om.shape)
        self.pr.set_model(**kw)
        want = _capi.WANT_LNL | ((_capi.WANT_GRAD_T | _capi.WANT_GRAD_GLOBAL) if grads else 0)
        out = self.pr.eval(m.t, want)
        self.evaluations += 1
        res = {"lnl": out["lnl"]}
        if grads:
            K = len(omegas)
            res.update(grad_t=np.array(out["grad_t"]), grad_theta=np.array(out["grad_dir"][:5]),
                       grad_omega=np.array(out["grad_dir"][5:5 + K]), grad_w=np.array(out["grad_class_w"][:K]))
        return res

    # ---------------------------------------------------------------------- fits
    def fit(self, m: BranchMixtures, *, t_nodes=(), mix_nodes=(), theta=False, fixed=None, max_iter=None) -> float:
        """Maximise lnL over the branch lengths of t_nodes, the omegas and weights of mix_nodes and, with
        theta, the exchangeabilities (log scales; weights by softmax logits), the rest held; fixed maps
        (node, class) -> an omega held at that value.  Updates m in place; returns its lnL."""
        from scipy.optimize import minimize
        fixed = dict(fixed or {})
        t_nodes, mix_nodes = list(t_nodes), list(mix_nodes)
        om_free = [(b, k) for b in mix_nodes for k in range(len(m.omegas[b])) if (b, k) not in fixed]
        wt_free = [b for b in mix_nodes if len(m.omegas[b]) > 1]
        for (b, k), v in fixed.items():
            m.omegas[b][k] = v
        starts = {}
        x0, lo, hi = [], [], []

        def seg(name, vals, lb, ub):
            starts[name] = len(x0)
            x0.extend(vals)
            lo.extend([lb] * len(vals))
            hi.extend([ub] * len(vals))
        seg("t", [math.log(max(m.t[b], 1e-8)) for b in t_nodes], math.log(1e-8), math.log(50.0))
        seg("om", [math.log(min(max(m.omegas[b][k], 1e-4), 1e4)) for b, k in om_free], math.log(1e-4), math.log(1e4))
        logits = []
        for b in wt_free:
            w = np.maximum(np.asarray(m.weights[b]), 1e-10)
            logits.extend(list(np.clip(np.log(w[1:] / w[0]), -20, 20)))
        seg("wt", logits, -20.0, 20.0)
        seg("th", [math.log(x) for x in m.theta] if theta else [], math.log(1e-3), math.log(1e3))
        if not x0:
            return self.evaluate(m, grads=False)["lnl"]
        cls_off = m.offsets()

        def apply(x):
            for i, b in enumerate(t_nodes):
                m.t[b] = math.exp(x[starts["t"] + i])
            for i, (b, k) in enumerate(om_free):
                m.omegas[b][k] = math.exp(x[starts["om"] + i])
            o = starts["wt"]
            for b in wt_free:
                K = len(m.omegas[b])
                z = np.concatenate([[0.0], x[o:o + K - 1]])
                e = np.exp(z - z.max())
                m.weights[b] = list(e / e.sum())
                o += K - 1
            if theta:
                m.theta = np.exp(x[starts["th"]:starts["th"] + 5])

        best = {"f": math.inf, "x": np.array(x0)}

        def objective(x):
            apply(x)
            r = self.evaluate(m)
            if not math.isfinite(r["lnl"]):
                return 1e30, np.zeros_like(x)
            g = np.zeros_like(x)
            for i, b in enumerate(t_nodes):
                g[starts["t"] + i] = r["grad_t"][b] * m.t[b]
            for i, (b, k) in enumerate(om_free):
                g[starts["om"] + i] = r["grad_omega"][cls_off[b] + k] * m.omegas[b][k]
            o = starts["wt"]
            for b in wt_free:
                K = len(m.omegas[b])
                w = np.asarray(m.weights[b])
                gw = r["grad_w"][cls_off[b]:cls_off[b] + K]
                gz = w * (gw - np.dot(w, gw))                  # softmax chain rule
                g[o:o + K - 1] = gz[1:]
                o += K - 1
            if theta:
                g[starts["th"]:starts["th"] + 5] = r["grad_theta"] * m.theta
            if -r["lnl"] < best["f"]:
                best["f"], best["x"] = -r["lnl"], np.array(x)
            return -r["lnl"], -g

        minimize(objective, np.array(x0), jac=True, method="L-BFGS-B", bounds=list(zip(lo, hi)),
                 options={"maxiter": max_iter or self.max_iter, "ftol": 1e-10, "gtol": 1e-5})
        apply(best["x"])
        return -best["f"]

    # ------------------------------------------------------------------ analysis
    def expected_length(self, m: BranchMixtures, b: int) -> float:
        """Expected substitutions per codon on branch b: t_b sum_k w_k mu(omega_k)."""
        return float(m.t[b] * sum(w * -np.dot(self.pi, np.diag(self.struct.Q(m.theta, o)))
                                  for o, w in zip(m.omegas[b], m.weights[b])))

    def run(self) -> dict:
        h = self.h
        nb = len(self.branches)
        # Phase 1: nucleotide GTR fit (absrel.hpp:780-795), the starting branch lengths and rates
        gtr = h.GTRFitter(self.tree, self.aln).fit()
        gp = gtr.params
        theta = np.array([gp.theta_AC, gp.theta_AT, gp.theta_CG, gp.theta_CT, gp.theta_GT])
        gtr_len = np.array(gtr.tree.get_branch_lengths())
        omega0 = 0.25
        mu0 = -np.dot(self.pi, np.diag(self.struct.Q(theta, omega0)))
        t0 = np.where(np.arange(self.n) == self.root, 0.0, np.maximum(3.0 * gtr_len / mu0, 1e-6))
        n_gtr = sum(1 for b in self.branches)
        result = {"gtr_fit": {"log_likelihood": gtr.log_likelihood, "parameters": 5 + 3 + n_gtr, "aicc": gtr.aicc}}
        # Phase 2: baseline MG94xREV, one omega per branch (absrel.hpp:812-1027)
        m = BranchMixtures(self.n, self.root, t0, theta, [omega0] * self.n)
        base_ll = self.fit(m, t_nodes=self.branches, mix_nodes=self.branches, theta=True)
        params = 5 + 9 + 2 * nb
        best_aicc = aicc(base_ll, params, self.n_obs)
        result["baseline_fit"] = {"log_likelihood": base_ll, "parameters": params, "aicc": best_aicc}
        names = {nd.id: nd.name for nd in self.tree.nodes}
        branches = {}
        for b in self.branches:
            branches[names[b]] = {"node": b, "baseline_omega": m.omegas[b][0],
                                  "baseline_branch_length": self.expected_length(m, b), "rate_classes": 1}
        # Phase 3: step-up complexity, longest baseline branches first (absrel.hpp:1400-1495)
        order = sorted(self.branches, key=lambda b: (-branches[names[b]]["baseline_branch_length"], b))
        cur_ll = base_ll
        for b in order:
            for K in range(2, self.max_rate_classes + 1):
                cand = None
                w_top = m.omegas[b]
                for new_om, new_w in ((max(w_top) * 4.0 + 1.0, 0.1), (min(w_top) * 0.2, 0.3)):
                    c = m.copy()
                    base_w = [x * (1.0 - new_w) for x in m.weights[b]]
                    pairs = sorted(zip(w_top + [new_om], base_w + [new_w]))
                    c.omegas[b] = [p[0] for p in pairs]
                    c.weights[b] = [p[1] for p in pairs]
                    ll = self.fit(c, t_nodes=[b], mix_nodes=[b])
                    if cand is None or ll > cand[0]:
                        cand = (ll, c)
                cand_params = params + 2
                cand_aicc = aicc(cand[0], cand_params, self.n_obs)
                if cand_aicc < best_aicc:
                    best_aicc, params, m, cur_ll = cand_aicc, cand_params, cand[1], cand[0]
                    branches[names[b]]["rate_classes"] = K
                else:
                    break
        # Phase 4: the full adaptive model, every parameter at once
        full_ll = self.fit(m, t_nodes=self.branches, mix_nodes=self.branches, theta=True)
        if full_ll < cur_ll:
            full_ll = cur_ll
        result["full_adaptive_fit"] = {"log_likelihood": full_ll, "parameters": params, "aicc": aicc(full_ll, params, self.n_obs)}
        # Phase 5: per branch, its largest omega against omega = 1 (absrel.hpp:2050-2240)
        raw_p, tested = [], []
        for b in self.branches:
            br = branches[names[b]]
            om, w = m.omegas[b], m.weights[b]
            kmax = int(np.argmax(om))
            br.update(is_tested=True, omegas=list(om), weights=list(w))
            if om[kmax] <= 1.0:
                lrt, p = 0.0, 1.0
            else:
                null = m.copy()
                null_ll = self.fit(null, t_nodes=self.branches, mix_nodes=[b], fixed={(b, kmax): 1.0})
                lrt = 2.0 * (full_ll - null_ll)
                if not (lrt > 0.0 and math.isfinite(lrt)):
                    lrt, p = 0.0, 0.5
                else:
                    p = mixture_p_value(lrt)
            br.update(lrt=lrt, uncorrected_p_value=p)
            raw_p.append(p)
            tested.append(names[b])
        for nm, q in zip(tested, holm_bonferroni(raw_p)):
            branches[nm]["corrected_p_value"] = q
        result["branches"] = branches
        result["tested_branches"] = tested
        result["positive_branches"] = [nm for nm in tested if branches[nm]["corrected_p_value"] <= self.p_threshold]
        result["evaluations"] = self.evaluations
        return result
