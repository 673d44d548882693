"""ctypes binding of the C ABI in include/h3g.h (libh3g.so).

This is the thin layer a Python caller (or a test) uses to reach the device
library without the pybind11 module: plain pointers, sizes and status codes.
Loading fails loudly when the shared library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import weakref

import numpy as np

_PKG = pathlib.Path(__file__).resolve().parent.parent.parent  # hyphy-3_b200/
LIB_PATH = pathlib.Path(os.environ.get("H3G_LIBRARY", _PKG / "lib" / "libh3g.so"))

H3G_OK, H3G_ERR_ARG, H3G_ERR_OOM, H3G_ERR_CUDA, H3G_ERR_NUMERIC, H3G_ERR_TIMEOUT, H3G_ERR_STATE = range(7)
PREC_FP64, PREC_MIXED = 0, 1
TIME_RAW, TIME_NORMALIZED = 0, 1
WANT_LNL, WANT_SITE_LNL, WANT_GRAD_T, WANT_GRAD_GLOBAL = 1, 2, 4, 8

EXPORTED = [
    "h3g_ctx_create", "h3g_ctx_destroy", "h3g_last_error", "h3g_version", "h3g_problem_create",
    "h3g_problem_destroy", "h3g_model_set", "h3g_eval", "h3g_eval_from_P", "h3g_branch_length_gradients",
    "h3g_last_eval_stats", "h3g_last_eval_transfer", "h3g_stage_branch_lengths", "h3g_eval_resident",
    "h3g_read_result", "h3g_profile_stages", "h3g_eval_from_P_noalloc", "h3g_fel_run", "h3g_meme_run",
    "h3g_fel_run_tested", "h3g_meme_run_tested", "h3g_alignment_compress", "h3g_alignment_compress_device",
    "h3g_nuc_eval_from_P", "h3g_problem_set_wait_limit", "h3g_batch_create", "h3g_batch_destroy", "h3g_batch_eval",
    "h3g_batch_last_stats", "h3g_pack_result_device", "h3g_ctx_stream", "h3g_problem_set_tuning",
    "h3g_problem_get_tuning", "h3g_autotune", "h3g_model_get_eigensystem", "h3g_problem_set_memory_budget",
    "h3g_problem_checkpoint_info", "h3g_checkpoint_plan",
]
STAGE_NAMES = "build_P,prep_mixed,inside,root,outside,accum_A,frechet,hsum,small,dir".split(",")

_dp = C.POINTER(C.c_double)


class Tuning(C.Structure):
    _fields_ = [("a_chunk", C.c_int), ("ctas_per_sm", C.c_int), ("frechet_groups", C.c_int)]


class CheckpointInfo(C.Structure):
    _fields_ = [("active", C.c_int32), ("n_blocks", C.c_int32), ("target", C.c_int32), ("n_persistent", C.c_int32),
                ("scratch_internal", C.c_int32), ("scratch_nodes", C.c_int32), ("workspace_bytes", C.c_uint64),
                ("full_bytes", C.c_uint64)]


class ModelDesc(C.Structure):
    _fields_ = [
        ("S", C.c_int), ("pi", _dp), ("n_models", C.c_int), ("Q", _dp), ("lam", _dp), ("U", _dp), ("V", _dp),
        ("mu", _dp), ("K", C.c_int), ("class_w", _dp), ("has_bg", C.c_int), ("is_test", C.POINTER(C.c_uint8)),
        ("M", C.c_int), ("rates", _dp), ("rate_w", _dp), ("time_mode", C.c_int), ("n_dirs", C.c_int),
        ("dQ", _dp), ("precision", C.c_int), ("zero_l_sentinel", C.c_int), ("bg_w", _dp),
        ("branch_classes", C.POINTER(C.c_int32)), ("dQ_model", _dp),
    ]


class FelModel(C.Structure):
    _fields_ = [("S", C.c_int), ("pi", _dp), ("Qs", _dp), ("Qn", _dp)]


class FelResult(C.Structure):
    _fields_ = [("alpha", C.c_double), ("beta", C.c_double), ("alpha_null", C.c_double), ("log_l_alt", C.c_double),
                ("log_l_null", C.c_double), ("lrt", C.c_double), ("p_value", C.c_double), ("evaluations", C.c_int),
                ("beta_nuisance", C.c_double)]


class GeneticCodeDesc(C.Structure):
    _fields_ = [("S", C.c_int), ("codon_to_sense", C.POINTER(C.c_int8))]


class CompressInfo(C.Structure):
    _fields_ = [("n_patterns", C.c_int64), ("pos_counts", C.c_int64 * 12), ("rounds", C.c_int), ("hash_bits", C.c_int),
                ("profile", C.c_int), ("stage_ms", C.c_double * 4), ("launches", C.c_int)]


class MemeResult(C.Structure):
    _fields_ = [("alpha", C.c_double), ("beta1", C.c_double), ("p1", C.c_double), ("beta_plus", C.c_double),
                ("p_plus", C.c_double), ("lrt", C.c_double), ("p_value", C.c_double),
                ("branches_under_selection", C.c_int), ("total_branch_length", C.c_double),
                ("log_l_meme", C.c_double), ("log_l_fel", C.c_double), ("p_value_meme_vs_fel", C.c_double),
                ("fel_alpha", C.c_double), ("fel_beta", C.c_double), ("evaluations", C.c_int), ("beta_bg", C.c_double)]


class Result(C.Structure):
    _fields_ = [("lnl", C.c_double), ("site_lnl", _dp), ("grad_t", _dp), ("grad_dir", _dp),
                ("grad_class_w", _dp), ("grad_rate_w", _dp), ("grad_bg_w", _dp)]


_lib = None


def load() -> C.CDLL:
    """Load libh3g.so once; raises if it is missing (there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"libh3g.so not built at {LIB_PATH}; run __graft_entry__.build()")
        lib = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        lib.h3g_version.restype = C.c_char_p
        lib.h3g_last_error.restype = C.c_char_p
        lib.h3g_last_error.argtypes = [vp]
        lib.h3g_ctx_create.argtypes = [C.c_int, vp, C.POINTER(vp)]
        lib.h3g_ctx_destroy.argtypes = [vp]
        lib.h3g_problem_create.argtypes = [vp, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_uint8), C.POINTER(C.c_int32),
                                           C.c_int, C.c_int, C.POINTER(C.c_int8), C.POINTER(C.c_uint64), _dp, C.POINTER(vp)]
        lib.h3g_problem_destroy.argtypes = [vp]
        lib.h3g_model_set.argtypes = [vp, C.POINTER(ModelDesc)]
        lib.h3g_eval.argtypes = [vp, _dp, C.c_uint, C.POINTER(Result)]
        lib.h3g_eval_from_P.argtypes = [vp, C.c_int, _dp, _dp, _dp, _dp]
        lib.h3g_branch_length_gradients.argtypes = [vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp]
        lib.h3g_last_eval_stats.argtypes = [vp, _dp, C.POINTER(C.c_int)]
        lib.h3g_last_eval_transfer.argtypes = [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
        lib.h3g_stage_branch_lengths.argtypes = [vp, _dp]
        lib.h3g_eval_resident.argtypes = [vp, C.c_uint]
        lib.h3g_read_result.argtypes = [vp, C.c_uint, C.POINTER(Result)]
        lib.h3g_profile_stages.argtypes = [vp, C.c_uint, C.c_int, _dp, C.POINTER(C.c_int)]
        lib.h3g_eval_from_P_noalloc.argtypes = [C.c_int, vp, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_uint8),
                                                C.POINTER(C.c_int32), C.c_int, C.c_int, C.POINTER(C.c_int8),
                                                C.POINTER(C.c_uint64), _dp, C.c_int, _dp, _dp, _dp, _dp]
        lib.h3g_fel_run.argtypes = [vp, C.POINTER(FelModel), _dp, C.POINTER(FelResult)]
        lib.h3g_nuc_eval_from_P.argtypes = [vp, _dp, _dp, _dp, _dp]
        lib.h3g_problem_set_wait_limit.argtypes = [vp, C.c_uint32, C.c_int]
        lib.h3g_batch_create.argtypes = [vp, C.c_int, C.POINTER(vp), C.c_int, C.POINTER(vp)]
        lib.h3g_batch_destroy.argtypes = [vp]
        lib.h3g_batch_eval.argtypes = [vp, C.POINTER(_dp), C.c_uint, C.POINTER(Result)]
        lib.h3g_batch_last_stats.argtypes = [vp, _dp, C.POINTER(C.c_int)]
        lib.h3g_pack_result_device.argtypes = [vp, C.c_uint, vp]
        lib.h3g_ctx_stream.argtypes = [vp, C.POINTER(vp)]
        lib.h3g_problem_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
        lib.h3g_problem_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
        lib.h3g_autotune.argtypes = [vp, _dp, C.c_uint, C.c_int, C.POINTER(Tuning), _dp]
        lib.h3g_model_get_eigensystem.argtypes = [vp, C.c_int, _dp, _dp, _dp]
        lib.h3g_problem_set_memory_budget.argtypes = [vp, C.c_uint64, C.c_int]
        lib.h3g_problem_checkpoint_info.argtypes = [vp, C.POINTER(CheckpointInfo)]
        _i32 = C.POINTER(C.c_int32)
        lib.h3g_checkpoint_plan.argtypes = [C.c_int, _i32, C.POINTER(C.c_uint8), C.c_int, _i32, _i32, _i32, _i32, _i32]
        lib.h3g_fel_run_tested.argtypes = [vp, C.POINTER(FelModel), _dp, C.POINTER(C.c_uint8), C.POINTER(FelResult)]
        lib.h3g_meme_run.argtypes = [vp, C.POINTER(FelModel), _dp, C.POINTER(MemeResult), _dp]
        _i32p = C.POINTER(C.c_int32)
        lib.h3g_alignment_compress.argtypes = [vp, C.c_int, C.c_int64, C.c_void_p, C.c_size_t, C.POINTER(GeneticCodeDesc), _i32p,
                                               _i32p, _i32p, C.POINTER(C.c_int8), C.POINTER(C.c_uint64), C.POINTER(CompressInfo)]
        lib.h3g_alignment_compress_device.argtypes = [vp, C.c_int, C.c_int64, C.c_void_p, C.c_size_t, C.POINTER(GeneticCodeDesc),
                                                      vp, vp, vp, vp, vp, C.POINTER(CompressInfo)]
        lib.h3g_meme_run_tested.argtypes = [vp, C.POINTER(FelModel), _dp, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8),
                                            C.POINTER(MemeResult), _dp]
        for name in EXPORTED:
            getattr(lib, name).restype = getattr(lib, name).restype or C.c_int
        lib.h3g_version.restype = C.c_char_p
        lib.h3g_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def checkpoint_plan(parent, is_leaf, target: int) -> dict:
    """The subtree-checkpoint plan of a tree (host only, no device): per node is_checkpoint, block,
    slot_internal and slot_vf, and the counts {blocks, persistent, scratch_internal, scratch_nodes}."""
    lib = load()
    par = np.ascontiguousarray(parent, dtype=np.int32)
    lf = np.ascontiguousarray(is_leaf, dtype=np.uint8)
    n = len(par)
    out = {k: np.zeros(n, dtype=np.int32) for k in ("is_checkpoint", "block", "slot_internal", "slot_vf")}
    counts = np.zeros(4, dtype=np.int32)
    i32 = C.POINTER(C.c_int32)
    st = lib.h3g_checkpoint_plan(n, par.ctypes.data_as(i32), lf.ctypes.data_as(C.POINTER(C.c_uint8)), int(target),
                                 *(out[k].ctypes.data_as(i32) for k in ("is_checkpoint", "block", "slot_internal", "slot_vf")),
                                 counts.ctypes.data_as(i32))
    if st != 0:
        raise H3GError(f"h3g_checkpoint_plan failed with status {st}", st)
    out.update(blocks=int(counts[0]), persistent=int(counts[1]), scratch_internal=int(counts[2]),
               scratch_nodes=int(counts[3]))
    return out


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a: np.ndarray | None, ct=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


class H3GError(RuntimeError):
    """A C ABI call failed; .status is its h3g_status."""

    def __init__(self, msg: str, status: int = -1):
        super().__init__(msg)
        self.status = status


class Context:
    def __init__(self, device: int = 0, stream: int | None = None):
        self.lib = load()
        self.h = C.c_void_p()
        self._problems = weakref.WeakSet()
        st = self.lib.h3g_ctx_create(device, C.c_void_p(stream) if stream else None, C.byref(self.h))
        if st != H3G_OK:
            raise H3GError(f"h3g_ctx_create failed with status {st}")

    def check(self, st: int) -> None:
        if st != H3G_OK:
            raise H3GError(f"status {st}: {self.lib.h3g_last_error(self.h).decode()}", st)

    @property
    def stream_handle(self) -> int:
        """The cudaStream_t this context enqueues on (h3g_ctx_stream), as an integer handle."""
        sp = C.c_void_p()
        self.check(self.lib.h3g_ctx_stream(self.h, C.byref(sp)))
        return int(sp.value or 0)

    def alignment_compress(self, rows, codon_to_sense, hash_bits: int = 0) -> dict:
        """Codon translation, nucleotide counts and site-pattern compression of an in-frame alignment
        (h3g_alignment_compress).  rows: [n_taxa, n_nuc] uint8 array (or equal-length strings);
        codon_to_sense: 64 sense indices (-1 for stops) in A, C, G, T order.  Returns the patterns in
        first-site order: "site_to_pattern", "weight", "first_site", "states" [P, T], "masks" [P, T],
        "pos_counts" [3, 4], "rounds"."""
        if not isinstance(rows, np.ndarray):
            rows = np.frombuffer(b"".join(r.encode("latin-1") for r in rows), dtype=np.uint8).reshape(len(rows), -1)
        rows = np.ascontiguousarray(rows, dtype=np.uint8)
        T, L = rows.shape
        sense = np.ascontiguousarray(codon_to_sense, dtype=np.int8)
        code = GeneticCodeDesc(S=int((sense >= 0).sum()), codon_to_sense=sense.ctypes.data_as(C.POINTER(C.c_int8)))
        Cn = L // 3
        s2p = np.zeros(max(Cn, 1), np.int32)
        w = np.zeros(max(Cn, 1), np.int32)
        first = np.zeros(max(Cn, 1), np.int32)
        st = np.zeros((max(Cn, 1), T), np.int8)
        mk = np.zeros((max(Cn, 1), T), np.uint64)
        info = CompressInfo(hash_bits=hash_bits)
        i32 = C.POINTER(C.c_int32)
        self.check(self.lib.h3g_alignment_compress(
            self.h, T, L, rows.ctypes.data_as(C.c_void_p), L, C.byref(code), s2p.ctypes.data_as(i32), w.ctypes.data_as(i32),
            first.ctypes.data_as(i32), st.ctypes.data_as(C.POINTER(C.c_int8)), mk.ctypes.data_as(C.POINTER(C.c_uint64)),
            C.byref(info)))
        P = int(info.n_patterns)
        return {"site_to_pattern": s2p[:Cn], "weight": w[:P], "first_site": first[:P], "states": st[:P], "masks": mk[:P],
                "pos_counts": np.array(info.pos_counts[:], dtype=np.int64).reshape(3, 4), "rounds": int(info.rounds)}

    def close(self) -> None:
        """Destroy the context after every batch and problem still alive on it."""
        for b in list(getattr(self, "_batches", ())):
            b.close()
        for p in list(self._problems):
            p.close()
        if self.h:
            self.lib.h3g_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Problem:
    """One tree + compressed alignment resident on the device."""

    def __init__(self, ctx: Context, parent, is_leaf, leaf_taxon, states, masks, weights):
        self.ctx = ctx
        self.parent = np.ascontiguousarray(parent, dtype=np.int32)
        self.is_leaf = np.ascontiguousarray(is_leaf, dtype=np.uint8)
        self.leaf_taxon = np.ascontiguousarray(leaf_taxon, dtype=np.int32)
        self.states = np.ascontiguousarray(states, dtype=np.int8)
        self.masks = np.ascontiguousarray(masks, dtype=np.uint64)
        self.weights = _f64(weights)
        self.n = int(self.parent.size)
        self.P, self.T = (int(self.states.shape[0]), int(self.states.shape[1])) if self.states.ndim == 2 else (0, 0)
        self.root = int(np.flatnonzero(self.parent < 0)[0])
        self.h = C.c_void_p()
        ctx.check(ctx.lib.h3g_problem_create(
            ctx.h, self.n, _ptr(self.parent, C.c_int32), _ptr(self.is_leaf, C.c_uint8), _ptr(self.leaf_taxon, C.c_int32),
            self.T, self.P, _ptr(self.states, C.c_int8), _ptr(self.masks, C.c_uint64), _ptr(self.weights), C.byref(self.h)))
        ctx._problems.add(self)
        self.K = self.M = self.ndirs = 0

    def close(self) -> None:
        if self.h and self.ctx.h:
            self.ctx.lib.h3g_problem_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_model(self, *, pi, Q, lam=None, U=None, V=None, mu=None, class_w=(1.0,), has_bg=False, is_test=None, rates=(1.0,),
                  rate_w=(1.0,), time_mode=TIME_RAW, dQ=None, precision=PREC_FP64, zero_l_sentinel=False,
                  bg_w=None, branch_classes=None, dQ_model=None) -> None:
        """Q, U, V: [n_models, S, S]; lam: [n_models, S]; dQ: [n_dirs, n_models, S, S].  bg_w: weights of
        len(bg_w) background classes (models K ..), or None with has_bg for one background model.
        lam, U and V all None: the device diagonalises each Q (and mu defaults to -sum pi_i Q_ii)."""
        Q = _f64(Q)
        if Q.ndim == 2:
            Q = Q[None]
        dev_eig = U is None and V is None and lam is None       # the device diagonalises every Q_k
        if not dev_eig:
            U = _f64(U); V = _f64(V); lam = _f64(lam)
            if U.ndim == 2:
                U, V, lam = U[None], V[None], lam[None]
        nm, S = Q.shape[0], Q.shape[1]
        pi = _f64(pi)
        mu_a = None if (mu is None and dev_eig) else _f64(mu if mu is not None else np.ones(nm))
        cw = _f64(class_w); rt = _f64(rates); rw = _f64(rate_w)
        it = None if is_test is None else np.ascontiguousarray(is_test, dtype=np.uint8)
        dq = None if dQ is None else _f64(dQ)
        nd = 0 if dq is None else int(dq.shape[0])
        bw = None if bg_w is None else _f64(bg_w)
        bc = None if branch_classes is None else np.ascontiguousarray(branch_classes, dtype=np.int32)
        dqm = None if dQ_model is None else _f64(dQ_model)          # [n_models, S, S], one direction per model
        self._bc = bc                                    # kept alive while the model is installed
        if bw is not None:
            nbg = int(bw.size)
        else:
            nbg = int(has_bg) if isinstance(has_bg, int) and not isinstance(has_bg, bool) else int(bool(has_bg))
        d = ModelDesc(S=S, pi=_ptr(pi), n_models=nm, Q=_ptr(Q), lam=_ptr(lam), U=_ptr(U), V=_ptr(V), mu=_ptr(mu_a),
                      K=len(cw), class_w=_ptr(cw), has_bg=nbg, is_test=_ptr(it, C.c_uint8), M=len(rt),
                      rates=_ptr(rt), rate_w=_ptr(rw), time_mode=time_mode, n_dirs=nd, dQ=_ptr(dq),
                      precision=precision, zero_l_sentinel=int(bool(zero_l_sentinel)), bg_w=_ptr(bw),
                      branch_classes=_ptr(bc, C.c_int32), dQ_model=_ptr(dqm))
        self.ctx.check(self.ctx.lib.h3g_model_set(self.h, C.byref(d)))
        self.K, self.M, self.ndirs, self.nmod, self.S = len(cw), len(rt), nd + (nm if dqm is not None else 0), nm, S

    def eval(self, bl, want=WANT_LNL | WANT_GRAD_T, out=None) -> dict:
        bl = _f64(bl)
        if bl.size != self.n:
            raise ValueError("branch lengths must have one entry per node")
        if out is None:
            out = {"site_lnl": np.zeros(self.P), "grad_t": np.zeros(self.n), "grad_dir": np.zeros(max(self.ndirs, 1)),
                   "grad_class_w": np.zeros(self.K), "grad_rate_w": np.zeros(self.M),
                   "grad_bg_w": np.zeros(max(self.nmod - self.K, 1))}
        r = Result(site_lnl=_ptr(out["site_lnl"]), grad_t=_ptr(out["grad_t"]), grad_dir=_ptr(out["grad_dir"]),
                   grad_class_w=_ptr(out["grad_class_w"]), grad_rate_w=_ptr(out["grad_rate_w"]),
                   grad_bg_w=_ptr(out.get("grad_bg_w")))
        self.ctx.check(self.ctx.lib.h3g_eval(self.h, _ptr(bl), want, C.byref(r)))
        out["lnl"] = r.lnl
        return out

    def eval_from_P(self, P, pi) -> tuple[float, np.ndarray]:
        P = _f64(P); pi = _f64(pi)
        S = int(pi.size)
        lnl = C.c_double()
        site = np.zeros(self.P)
        self.ctx.check(self.ctx.lib.h3g_eval_from_P(self.h, S, _ptr(P), _ptr(pi), C.byref(lnl), _ptr(site)))
        return lnl.value, site

    def branch_length_gradients(self, *, pi, Q, lam=None, U=None, V=None, bl, precision=PREC_FP64) -> tuple[float, np.ndarray]:
        """h3g_branch_length_gradients; lam, U, V all None: the device diagonalises Q."""
        pi, Q, bl = (_f64(x) for x in (pi, Q, bl))
        lam, U, V = (None if x is None else _f64(x) for x in (lam, U, V))
        lnl = C.c_double()
        g = np.zeros(self.n)
        self.ctx.check(self.ctx.lib.h3g_branch_length_gradients(
            self.h, int(pi.size), _ptr(pi), _ptr(Q), _ptr(lam), _ptr(U), _ptr(V), _ptr(bl), precision, C.byref(lnl), _ptr(g)))
        return lnl.value, g

    def fel_run(self, *, pi, Qs, Qn, branch_lengths, tested=None) -> dict:
        """FEL per-pattern fits (h3g_fel_run, or h3g_fel_run_tested when tested[n_nodes] is given);
        branch lengths in FEL time.  Returns arrays per pattern."""
        pi, Qs, Qn, bl = _f64(pi), _f64(Qs), _f64(Qn), _f64(branch_lengths)
        S = int(pi.size)
        if Qs.shape != (S, S) or Qn.shape != (S, S) or bl.size != self.n:
            raise ValueError("Qs, Qn must be S x S and branch_lengths one per node")
        m = FelModel(S=S, pi=_ptr(pi), Qs=_ptr(Qs), Qn=_ptr(Qn))
        res = (FelResult * max(self.P, 1))()
        if tested is None:
            self.ctx.check(self.ctx.lib.h3g_fel_run(self.h, C.byref(m), _ptr(bl), res))
        else:
            tv = np.ascontiguousarray(np.asarray(tested, dtype=bool), dtype=np.uint8)
            if tv.size != self.n:
                raise ValueError("tested needs one entry per node")
            self.ctx.check(self.ctx.lib.h3g_fel_run_tested(
                self.h, C.byref(m), _ptr(bl), tv.ctypes.data_as(C.POINTER(C.c_uint8)), res))
        names = [f[0] for f in FelResult._fields_]
        return {k: np.array([getattr(res[i], k) for i in range(self.P)]) for k in names}

    def meme_run(self, *, pi, Qs, Qn, branch_lengths, with_ebf: bool = True, tested=None, fel_tested=None) -> dict:
        """MEME per-pattern fits (h3g_meme_run, or h3g_meme_run_tested when tested[n_nodes] is given;
        fel_tested, the FEL baseline's set, defaults to tested); branch lengths in FEL time.  Returns
        arrays per pattern and, with with_ebf, "branch_ebf" [n_patterns, n_nodes]."""
        pi, Qs, Qn, bl = _f64(pi), _f64(Qs), _f64(Qn), _f64(branch_lengths)
        S = int(pi.size)
        if Qs.shape != (S, S) or Qn.shape != (S, S) or bl.size != self.n:
            raise ValueError("Qs, Qn must be S x S and branch_lengths one per node")
        m = FelModel(S=S, pi=_ptr(pi), Qs=_ptr(Qs), Qn=_ptr(Qn))
        res = (MemeResult * max(self.P, 1))()
        ebf = np.zeros((max(self.P, 1), self.n)) if with_ebf else None
        if tested is None:
            self.ctx.check(self.ctx.lib.h3g_meme_run(self.h, C.byref(m), _ptr(bl), res, _ptr(ebf) if with_ebf else None))
        else:
            def mask(x):
                v = np.ascontiguousarray(np.asarray(x, dtype=bool), dtype=np.uint8)
                if v.size != self.n:
                    raise ValueError("tested / fel_tested need one entry per node")
                return v
            tv = mask(tested)
            fv = mask(fel_tested) if fel_tested is not None else None
            u8 = C.POINTER(C.c_uint8)
            self.ctx.check(self.ctx.lib.h3g_meme_run_tested(
                self.h, C.byref(m), _ptr(bl), tv.ctypes.data_as(u8), fv.ctypes.data_as(u8) if fv is not None else None,
                res, _ptr(ebf) if with_ebf else None))
        names = [f[0] for f in MemeResult._fields_]
        out = {k: np.array([getattr(res[i], k) for i in range(self.P)]) for k in names}
        if with_ebf:
            out["branch_ebf"] = ebf[: self.P]
        return out

    def _result_struct(self, out):
        return Result(site_lnl=_ptr(out["site_lnl"]), grad_t=_ptr(out["grad_t"]), grad_dir=_ptr(out["grad_dir"]),
                      grad_class_w=_ptr(out["grad_class_w"]), grad_rate_w=_ptr(out["grad_rate_w"]))

    def empty_result(self) -> dict:
        return {"site_lnl": np.zeros(self.P), "grad_t": np.zeros(self.n), "grad_dir": np.zeros(max(self.ndirs, 1)),
                "grad_class_w": np.zeros(self.K), "grad_rate_w": np.zeros(self.M)}

    def set_wait_limit(self, polls: int = 0, unmatched: bool = False) -> None:
        """Polls before a persistent-pass flag wait gives up (0 = default); unmatched makes every such
        wait look for a value no item publishes (tests the H3G_ERR_TIMEOUT path)."""
        self.ctx.check(self.ctx.lib.h3g_problem_set_wait_limit(self.h, C.c_uint32(polls), C.c_int(int(unmatched))))

    def set_memory_budget(self, nbytes: int = 0, target: int = 0) -> None:
        """Device bytes the evaluation workspace may take (0 = no budget; a workspace larger than free
        device memory still checkpoints by itself); target > 0 forces the checkpoint block size."""
        self.ctx.check(self.ctx.lib.h3g_problem_set_memory_budget(self.h, C.c_uint64(int(nbytes)), C.c_int(int(target))))

    def checkpoint_info(self) -> dict:
        """The installed workspace's checkpoint plan: active, blocks, target, slots and bytes."""
        ci = CheckpointInfo()
        self.ctx.check(self.ctx.lib.h3g_problem_checkpoint_info(self.h, C.byref(ci)))
        return {f: int(getattr(ci, f)) for f, _ in CheckpointInfo._fields_}

    def get_eigensystem(self, k: int = 0) -> dict:
        """The installed eigensystem of model k (given, or solved on the device): {"lam", "U", "V"}."""
        S = self.S
        lam, U, V = np.zeros(S), np.zeros((S, S)), np.zeros((S, S))
        self.ctx.check(self.ctx.lib.h3g_model_get_eigensystem(self.h, k, _ptr(lam), _ptr(U), _ptr(V)))
        return {"lam": lam, "U": U, "V": V}

    def set_tuning(self, a_chunk: int = 0, ctas_per_sm: int = 0, frechet_groups: int = 0) -> None:
        """Launch shapes (h3g_problem_set_tuning); 0 = the recorded tuning or the heuristic."""
        self.ctx.check(self.ctx.lib.h3g_problem_set_tuning(self.h, C.byref(Tuning(a_chunk, ctas_per_sm, frechet_groups))))

    def get_tuning(self) -> dict:
        t = Tuning()
        self.ctx.check(self.ctx.lib.h3g_problem_get_tuning(self.h, C.byref(t)))
        return {"a_chunk": t.a_chunk, "ctas_per_sm": t.ctas_per_sm, "frechet_groups": t.frechet_groups}

    def autotune(self, bl, want=WANT_LNL | WANT_GRAD_T, reps: int = 3) -> tuple[dict, float]:
        """Time the launch-shape candidates (h3g_autotune), keep and record the fastest; (tuning, ms)."""
        bl = _f64(bl)
        t, ms = Tuning(), C.c_double()
        self.ctx.check(self.ctx.lib.h3g_autotune(self.h, _ptr(bl), want, reps, C.byref(t), C.byref(ms)))
        return {"a_chunk": t.a_chunk, "ctas_per_sm": t.ctas_per_sm, "frechet_groups": t.frechet_groups}, ms.value

    def pack_device(self, want, d_ptr: int) -> None:
        """Enqueue the assembly of the last resident evaluation's results into the device vector at d_ptr
        (1 + n + ndirs + K + M + 1 doubles, h3g_pack_result_device)."""
        self.ctx.check(self.ctx.lib.h3g_pack_result_device(self.h, want, C.c_void_p(d_ptr)))

    def stage_branch_lengths(self, bl) -> None:
        bl = _f64(bl)
        self.ctx.check(self.ctx.lib.h3g_stage_branch_lengths(self.h, _ptr(bl)))

    def eval_resident(self, want=WANT_LNL | WANT_GRAD_T) -> None:
        """Enqueue one evaluation on the context stream (inputs already on the device); returns at once."""
        self.ctx.check(self.ctx.lib.h3g_eval_resident(self.h, want))

    def read_result(self, want=WANT_LNL | WANT_GRAD_T, out=None) -> dict:
        out = out or self.empty_result()
        r = self._result_struct(out)
        self.ctx.check(self.ctx.lib.h3g_read_result(self.h, want, C.byref(r)))
        out["lnl"] = r.lnl
        return out

    def profile_stages(self, want=WANT_LNL | WANT_GRAD_T, reps=5) -> dict:
        ms = np.zeros(len(STAGE_NAMES))
        nl = (C.c_int * len(STAGE_NAMES))()
        self.ctx.check(self.ctx.lib.h3g_profile_stages(self.h, want, reps, _ptr(ms), nl))
        return {name: (float(ms[i]), int(nl[i])) for i, name in enumerate(STAGE_NAMES) if nl[i] > 0}

    def last_transfer(self) -> tuple[int, int]:
        a, b = C.c_size_t(), C.c_size_t()
        self.ctx.check(self.ctx.lib.h3g_last_eval_transfer(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def last_stats(self) -> tuple[float, int]:
        ms = C.c_double()
        nl = C.c_int()
        self.ctx.check(self.ctx.lib.h3g_last_eval_stats(self.h, C.byref(ms), C.byref(nl)))
        return ms.value, nl.value


class Batch:
    """Independent problems (genes) evaluated by one graph launch per call (h3g_batch_*).

    The problems keep their topology, patterns and models; their workspaces are the batch's
    n_slots slot workspaces.  Install models with Problem.set_model (one precision for all) before
    the first eval; after close() every problem needs set_model again to be used alone."""

    def __init__(self, ctx: Context, problems, n_slots: int = 8):
        self.ctx = ctx
        self.problems = list(problems)
        arr = (C.c_void_p * len(self.problems))(*[p.h.value for p in self.problems])
        self.h = C.c_void_p()
        ctx.check(ctx.lib.h3g_batch_create(ctx.h, len(self.problems), arr, n_slots, C.byref(self.h)))
        if not hasattr(ctx, "_batches"):
            ctx._batches = weakref.WeakSet()
        ctx._batches.add(self)

    def eval(self, branch_lengths, want=WANT_LNL | WANT_GRAD_T) -> list[dict]:
        G = len(self.problems)
        bls = [_f64(b) for b in branch_lengths]
        if len(bls) != G or any(b.size != p.n for b, p in zip(bls, self.problems)):
            raise ValueError("one branch-length vector (one entry per node) per problem")
        outs = []
        res = (Result * G)()
        for g, p in enumerate(self.problems):
            o = {"site_lnl": np.zeros(p.P), "grad_t": np.zeros(p.n), "grad_dir": np.zeros(max(p.ndirs, 1)),
                 "grad_class_w": np.zeros(p.K), "grad_rate_w": np.zeros(p.M), "grad_bg_w": np.zeros(max(p.nmod - p.K, 1))}
            outs.append(o)
            res[g] = Result(site_lnl=_ptr(o["site_lnl"]), grad_t=_ptr(o["grad_t"]), grad_dir=_ptr(o["grad_dir"]),
                            grad_class_w=_ptr(o["grad_class_w"]), grad_rate_w=_ptr(o["grad_rate_w"]),
                            grad_bg_w=_ptr(o["grad_bg_w"]))
        blp = (_dp * G)(*[_ptr(b) for b in bls])
        self.ctx.check(self.ctx.lib.h3g_batch_eval(self.h, blp, want, res))
        for g in range(G):
            outs[g]["lnl"] = res[g].lnl
        return outs

    def last_stats(self) -> tuple[float, int]:
        ms, nl = C.c_double(), C.c_int()
        self.ctx.check(self.ctx.lib.h3g_batch_last_stats(self.h, C.byref(ms), C.byref(nl)))
        return ms.value, nl.value

    def close(self) -> None:
        if self.h and self.ctx.h:
            self.ctx.lib.h3g_batch_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def eval_from_P_noalloc(parent, is_leaf, leaf_taxon, states, masks, weights, P, pi, device: int = 0,
                        stream: int | None = None) -> tuple[float, np.ndarray]:
    """h3g_eval_from_P_noalloc: lnL from given transition matrices with no device allocation.

    For callers that may not allocate device memory while running; the library
    uses its fixed 32 MiB per-device scratch array instead.  Raises H3GError
    with the status code (H3G_ERR_ARG when the problem is larger than that).
    """
    lib = load()
    parent = np.ascontiguousarray(parent, dtype=np.int32)
    is_leaf = np.ascontiguousarray(is_leaf, dtype=np.uint8)
    leaf_taxon = np.ascontiguousarray(leaf_taxon, dtype=np.int32)
    states = np.ascontiguousarray(states, dtype=np.int8)
    masks = np.ascontiguousarray(masks, dtype=np.uint64)
    weights = _f64(weights)
    P = _f64(P)
    pi = _f64(pi)
    nP, T = states.shape
    lnl = C.c_double()
    site = np.zeros(nP)
    st = lib.h3g_eval_from_P_noalloc(device, C.c_void_p(stream) if stream else None, int(parent.size),
                                     _ptr(parent, C.c_int32), _ptr(is_leaf, C.c_uint8), _ptr(leaf_taxon, C.c_int32),
                                     T, nP, _ptr(states, C.c_int8), _ptr(masks, C.c_uint64), _ptr(weights),
                                     int(pi.size), _ptr(P), _ptr(pi), C.byref(lnl), _ptr(site))
    if st != H3G_OK:
        raise H3GError(f"h3g_eval_from_P_noalloc failed with status {st}")
    return lnl.value, site
