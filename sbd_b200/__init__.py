"""sbd_b200: the tensor-product-basis Davidson path of r-ccs-cms/sbd on B200.

Python binding (ctypes) of the C ABI declared in include/sbdgpu.h, implemented
by the in-tree library sbd_b200/libsbdgpu.so.  There is no CPU fallback: if the
library is missing, or no CUDA device is present, every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsbdgpu.so")

FP64 = 0
MIXED = 1
MIXED_TC = 2

_u64p = ctypes.POINTER(ctypes.c_uint64)
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

EXPORTS = [
    "sbdgpu_create", "sbdgpu_build_tables", "sbdgpu_table_sizes", "sbdgpu_get_tables", "sbdgpu_diag",
    "sbdgpu_sigma", "sbdgpu_sigma_device", "sbdgpu_davidson", "sbdgpu_rdm", "sbdgpu_occupation",
    "sbdgpu_alpha_weights", "sbdgpu_last_sigma_ms", "sbdgpu_last_error", "sbdgpu_destroy",
    "sbdgpu_sigma_device_noalloc", "sbdgpu_store_hamiltonian", "sbdgpu_release_hamiltonian",
    "sbdgpu_davidson_roots", "sbdgpu_wait_selftest", "sbdgpu_davidson_batch", "sbdgpu_sigma_rows_device",
    "sbdgpu_precond_train", "sbdgpu_precond_get", "sbdgpu_precond_set", "sbdgpu_precond_apply",
    "sbdgpu_mlp_loss_grad", "sbdgpu_genop_create", "sbdgpu_genop_set_terms", "sbdgpu_genop_mult",
    "sbdgpu_genop_mult_device", "sbdgpu_genop_diagonal", "sbdgpu_genop_lanczos", "sbdgpu_genop_davidson",
    "sbdgpu_genop_last_error", "sbdgpu_genop_destroy", "sbdgpu_genop_set_fcidump", "sbdgpu_set_tuning", "sbdgpu_genop_ham_square", "sbdgpu_genop_expand", "sbdgpu_set_fp64_same_spin",
    "sbdgpu_autotune",
]

PRECOND_DIAGONAL = 0
PRECOND_LEARNED = 1
PRECOND_OLSEN = 2


class SbdGpuError(RuntimeError):
    pass


class Opts(ctypes.Structure):
    _fields_ = [("max_it", ctypes.c_int), ("max_nb", ctypes.c_int), ("eps", ctypes.c_double),
                ("max_time", ctypes.c_double), ("precision", ctypes.c_int), ("verbose", ctypes.c_int),
                ("restart_keep", ctypes.c_int), ("restart_prev", ctypes.c_int), ("precond", ctypes.c_int)]


class LearnOpts(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_int), ("cycle", ctypes.c_int), ("cg_iters", ctypes.c_int),
                ("samples", ctypes.c_int), ("steps", ctypes.c_int), ("lr", ctypes.c_float),
                ("seed", ctypes.c_uint)]


_lib = None


def lib():
    """Load libsbdgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SbdGpuError(f"{LIB_PATH} is missing: build it with sbd_b200.build.build_lib()")
        L = ctypes.CDLL(LIB_PATH)
        L.sbdgpu_create.restype = ctypes.c_int
        L.sbdgpu_create.argtypes = [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t, _u64p,
                                    _u64p, ctypes.c_double, _dp, _dp, ctypes.c_int]
        L.sbdgpu_build_tables.argtypes = [_vp]
        L.sbdgpu_table_sizes.argtypes = [_vp, ctypes.c_int, _u64p, _u64p]
        L.sbdgpu_get_tables.argtypes = [_vp, ctypes.c_int, _u64p, _u64p, _u64p, _u64p]
        L.sbdgpu_diag.argtypes = [_vp, _dp]
        L.sbdgpu_sigma.argtypes = [_vp, _dp, _dp, ctypes.c_int]
        L.sbdgpu_sigma_device.argtypes = [_vp, _vp, _vp, ctypes.c_int]
        L.sbdgpu_sigma_device_noalloc.argtypes = [_vp, _vp, _vp]
        L.sbdgpu_sigma_rows_device.argtypes = [_vp, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t]
        L.sbdgpu_davidson.argtypes = [_vp, ctypes.POINTER(Opts), _dp, _dp, _dp, _dp, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int)]
        L.sbdgpu_davidson_roots.argtypes = [_vp, ctypes.POINTER(Opts), ctypes.c_int, _dp, _dp, _dp,
                                            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.sbdgpu_wait_selftest.argtypes = [_vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int)]
        L.sbdgpu_davidson_batch.argtypes = [ctypes.c_int, ctypes.POINTER(_vp), ctypes.POINTER(Opts),
                                            ctypes.POINTER(_dp), _dp, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        _fp = ctypes.POINTER(ctypes.c_float)
        L.sbdgpu_precond_train.argtypes = [_vp, ctypes.POINTER(LearnOpts), _dp, _dp]
        L.sbdgpu_precond_get.argtypes = [_vp, _fp, ctypes.POINTER(ctypes.c_int)]
        L.sbdgpu_precond_set.argtypes = [_vp, _fp, ctypes.c_int]
        L.sbdgpu_precond_apply.argtypes = [_vp, _dp, ctypes.c_double, _dp]
        L.sbdgpu_mlp_loss_grad.argtypes = [ctypes.c_int, _fp, ctypes.c_int, _fp, _dp, _dp, _dp, _dp, _dp,
                                           ctypes.c_double, ctypes.c_double, _dp, _fp]
        L.sbdgpu_set_tuning.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
        L.sbdgpu_set_fp64_same_spin.argtypes = [_vp, ctypes.c_int]
        L.sbdgpu_autotune.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_float)]
        L.sbdgpu_store_hamiltonian.argtypes = [_vp, _u64p]
        L.sbdgpu_release_hamiltonian.argtypes = [_vp]
        L.sbdgpu_rdm.argtypes = [_vp, _dp, _dp, _dp]
        L.sbdgpu_occupation.argtypes = [_vp, _dp, _dp]
        L.sbdgpu_alpha_weights.argtypes = [_vp, _dp, _dp]
        L.sbdgpu_last_sigma_ms.argtypes = [_vp, ctypes.POINTER(ctypes.c_float)]
        L.sbdgpu_last_error.restype = ctypes.c_char_p
        L.sbdgpu_last_error.argtypes = [_vp]
        L.sbdgpu_destroy.argtypes = [_vp]
        _i64p, _i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
        L.sbdgpu_genop_create.argtypes = [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, ctypes.c_size_t, _u64p,
                                          ctypes.c_int]
        L.sbdgpu_genop_set_terms.argtypes = [_vp, ctypes.c_size_t, _i64p, _i32p, _i32p, _dp,
                                             ctypes.c_size_t, _i64p, _i32p, _i32p, _dp]
        L.sbdgpu_genop_set_fcidump.argtypes = [_vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int)]
        L.sbdgpu_genop_mult.argtypes = [_vp, _dp, _dp]
        L.sbdgpu_genop_ham_square.argtypes = [_vp, _dp, _dp]
        L.sbdgpu_genop_expand.argtypes = [_vp, _dp, ctypes.c_double, _u64p, ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_size_t)]
        L.sbdgpu_genop_mult_device.argtypes = [_vp, _vp, _vp]
        L.sbdgpu_genop_diagonal.argtypes = [_vp, _dp]
        L.sbdgpu_genop_lanczos.argtypes = [_vp, _dp, ctypes.c_int, ctypes.c_double, _dp,
                                           ctypes.POINTER(ctypes.c_int)]
        L.sbdgpu_genop_davidson.argtypes = [_vp, ctypes.POINTER(Opts), _dp, _dp, _dp, _dp, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int)]
        L.sbdgpu_genop_last_error.restype = ctypes.c_char_p
        L.sbdgpu_genop_last_error.argtypes = [_vp]
        L.sbdgpu_genop_destroy.argtypes = [_vp]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


class Context:
    """One alpha x beta product basis and Hamiltonian on one GPU."""

    def __init__(self, norb: int, astr, bstr, ecore: float, h1: np.ndarray, eri_packed: np.ndarray,
                 device: int = 0):
        self.norb = int(norb)
        self.astr = np.ascontiguousarray(astr, dtype=np.uint64)
        self.bstr = np.ascontiguousarray(bstr, dtype=np.uint64)
        self.na, self.nb = len(self.astr), len(self.bstr)
        self.n = self.na * self.nb
        h = np.ascontiguousarray(h1, dtype=np.float64)
        e = np.ascontiguousarray(eri_packed, dtype=np.float64)
        self._h = _vp()
        rc = lib().sbdgpu_create(ctypes.byref(self._h), self.norb, self.na, self.nb, _p(self.astr, _u64p),
                                 _p(self.bstr, _u64p), float(ecore), _p(h, _dp), _p(e, _dp), int(device))
        if rc != 0:
            raise SbdGpuError(f"sbdgpu_create failed with status {rc}")

    def _check(self, rc: int):
        if rc != 0:
            msg = lib().sbdgpu_last_error(self._h)
            raise SbdGpuError(f"status {rc}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "_h", None):
            lib().sbdgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self, spin: int):
        ns, nd = ctypes.c_uint64(0), ctypes.c_uint64(0)
        self._check(lib().sbdgpu_table_sizes(self._h, spin, ctypes.byref(ns), ctypes.byref(nd)))
        n = self.na if spin == 0 else self.nb
        so = np.zeros(n + 1, np.uint64)
        do = np.zeros(n + 1, np.uint64)
        si = np.zeros(max(ns.value, 1), np.uint64)
        di = np.zeros(max(nd.value, 1), np.uint64)
        self._check(lib().sbdgpu_get_tables(self._h, spin, _p(so, _u64p), _p(si, _u64p), _p(do, _u64p),
                                            _p(di, _u64p)))
        return so, si[:ns.value], do, di[:nd.value]

    def hii(self) -> np.ndarray:
        out = np.zeros(self.n)
        self._check(lib().sbdgpu_diag(self._h, _p(out, _dp)))
        return out

    def sigma(self, C: np.ndarray, precision: int = FP64) -> np.ndarray:
        C = np.ascontiguousarray(C, dtype=np.float64).ravel()
        out = np.zeros(self.n)
        self._check(lib().sbdgpu_sigma(self._h, _p(C, _dp), _p(out, _dp), precision))
        return out

    def sigma_device(self, dC_ptr: int, dS_ptr: int, precision: int = FP64) -> None:
        self._check(lib().sbdgpu_sigma_device(self._h, _vp(dC_ptr), _vp(dS_ptr), precision))

    def sigma_rows_device(self, dC_ptr: int, dS_ptr: int, r0: int, r1: int) -> None:
        """FP64 sigma rows [r0, r1) (alpha strings) of the full device vector C
        into a (r1 - r0) x nb device block: one rank's share of a sigma split
        into alpha-row blocks."""
        self._check(lib().sbdgpu_sigma_rows_device(self._h, _vp(dC_ptr), _vp(dS_ptr), int(r0), int(r1)))

    def sigma_device_noalloc(self, dC_ptr: int, dS_ptr: int) -> None:
        """FP64 sigma on device vectors that allocates nothing during the call
        (scratch in a fixed 12 MiB device array; at most 524,288 determinants;
        the set-up, tables() and hii(), must have run first)."""
        self._check(lib().sbdgpu_sigma_device_noalloc(self._h, _vp(dC_ptr), _vp(dS_ptr)))

    def davidson_roots(self, nroots: int, max_it: int, max_nb: int, eps: float, W0: np.ndarray | None = None,
                       max_time: float = 86400.0, verbose: int = 0):
        """Block Davidson for the nroots lowest roots (FP64).  Returns
        (energies[nroots], W[nroots, n], residual norms, cycles, sigma builds)."""
        W = np.zeros((nroots, self.n)) if W0 is None else np.ascontiguousarray(W0, dtype=np.float64).reshape(
            nroots, self.n).copy()
        o = Opts(max_it, max_nb, eps, max_time, FP64, verbose, 0, 0, PRECOND_DIAGONAL)
        e = np.zeros(nroots)
        r = np.zeros(nroots)
        it, ns = ctypes.c_int(0), ctypes.c_int(0)
        self._check(lib().sbdgpu_davidson_roots(self._h, ctypes.byref(o), nroots, _p(W, _dp), _p(e, _dp), _p(r, _dp),
                                                ctypes.byref(it), ctypes.byref(ns)))
        return e, W, r, it.value, ns.value

    def wait_selftest(self, spin_limit: int = 4096):
        """(first wait timed out, second wait timed out) of the bounded
        mbarrier-wait diagnostic; (1, 0) is the expected answer."""
        st = (ctypes.c_int * 2)()
        self._check(lib().sbdgpu_wait_selftest(self._h, int(spin_limit), st))
        return int(st[0]), int(st[1])

    def set_fp64_same_spin(self, method: int) -> None:
        """0 (the default): same-spin terms of the FP64 sigma as exact INT8
        tensor-core products where they fit; 1: the rows kernels."""
        self._check(lib().sbdgpu_set_fp64_same_spin(self._h, int(method)))

    def set_tuning(self, ab_group: int, ab_threads: int) -> None:
        """Launch shape of the FP64 alpha-beta kernel ((0, 0): the default)."""
        self._check(lib().sbdgpu_set_tuning(self._h, int(ab_group), int(ab_threads)))

    def autotune(self, reps: int = 3):
        """Time every alpha-beta shape that fits, keep the fastest:
        (ab_group, ab_threads, sigma ms)."""
        g, t, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0.0)
        self._check(lib().sbdgpu_autotune(self._h, int(reps), ctypes.byref(g), ctypes.byref(t), ctypes.byref(ms)))
        return g.value, t.value, ms.value

    def store_hamiltonian(self) -> int:
        """Method 1: keep the Hamiltonian's off-diagonal elements on the device
        (makeQCham, chemistry/tpb/qcham.h:10-312); later FP64 sigma builds,
        those of davidson() included, use them.  Returns the element count."""
        nnz = np.zeros(1, dtype=np.uint64)
        self._check(lib().sbdgpu_store_hamiltonian(self._h, _p(nnz, _u64p)))
        return int(nnz[0])

    def release_hamiltonian(self) -> None:
        self._check(lib().sbdgpu_release_hamiltonian(self._h))

    def last_sigma_ms(self):
        a = (ctypes.c_float * 5)()
        self._check(lib().sbdgpu_last_sigma_ms(self._h, a))
        return [float(x) for x in a]

    def davidson(self, W0: np.ndarray, max_it: int, max_nb: int, eps: float, max_time: float = 86400.0,
                 precision: int = FP64, verbose: int = 0, max_trace: int = 100000, restart_keep: int = 0,
                 restart_prev: int = 0, precond: int = PRECOND_DIAGONAL):
        W = np.ascontiguousarray(W0, dtype=np.float64).ravel().copy()
        o = Opts(max_it, max_nb, eps, max_time, precision, verbose, restart_keep, restart_prev, precond)
        e = ctypes.c_double(0.0)
        te = np.zeros(max_trace)
        tt = np.zeros(max_trace)
        ns = ctypes.c_int(0)
        self._check(lib().sbdgpu_davidson(self._h, ctypes.byref(o), _p(W, _dp), ctypes.byref(e), _p(te, _dp),
                                          _p(tt, _dp), max_trace, ctypes.byref(ns)))
        k = min(ns.value, max_trace)
        return e.value, W, te[:k], tt[:k]

    def precond_train(self, pairs: int = 12, cycle: int = 10, cg_iters: int = 40, samples: int = 65536,
                      steps: int = 600, lr: float = 1e-3, seed: int = 0):
        """Harvest (Ritz vector, residual, correction) triples on this system
        and train the learned preconditioner.  Returns (loss per step,
        [harvest s, training s])."""
        o = LearnOpts(pairs, cycle, cg_iters, samples, steps, lr, seed)
        tr = np.zeros(max(steps, 1))
        sec = np.zeros(2)
        self._check(lib().sbdgpu_precond_train(self._h, ctypes.byref(o), _p(tr, _dp), _p(sec, _dp)))
        return tr[:steps], sec

    def precond_get(self) -> np.ndarray:
        n = ctypes.c_int(0)
        self._check(lib().sbdgpu_precond_get(self._h, None, ctypes.byref(n)))
        w = np.zeros(n.value, dtype=np.float32)
        self._check(lib().sbdgpu_precond_get(self._h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                             ctypes.byref(n)))
        return w

    def precond_set(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(lib().sbdgpu_precond_set(self._h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(w)))

    def precond_apply(self, R: np.ndarray, e0: float) -> np.ndarray:
        R = np.ascontiguousarray(R, dtype=np.float64).ravel()
        out = np.zeros(self.n)
        self._check(lib().sbdgpu_precond_apply(self._h, _p(R, _dp), float(e0), _p(out, _dp)))
        return out

    def rdm(self, W: np.ndarray):
        W = np.ascontiguousarray(W, dtype=np.float64).ravel()
        L = self.norb
        one = np.zeros(2 * L * L)
        two = np.zeros(4 * L ** 4)
        self._check(lib().sbdgpu_rdm(self._h, _p(W, _dp), _p(one, _dp), _p(two, _dp)))
        return one, two

    def occupation(self, W: np.ndarray) -> np.ndarray:
        W = np.ascontiguousarray(W, dtype=np.float64).ravel()
        d = np.zeros(2 * self.norb)
        self._check(lib().sbdgpu_occupation(self._h, _p(W, _dp), _p(d, _dp)))
        return d

    def alpha_weights(self, W: np.ndarray) -> np.ndarray:
        W = np.ascontiguousarray(W, dtype=np.float64).ravel()
        d = np.zeros(self.na)
        self._check(lib().sbdgpu_alpha_weights(self._h, _p(W, _dp), _p(d, _dp)))
        return d


def davidson_batch(ctxs, W0s, max_it: int, max_nb: int, eps: float, precision: int = FP64,
                   max_time: float = 86400.0, restart_keep: int = 0, restart_prev: int = 0, max_threads: int = 0):
    """Lowest-root Davidson for several independent contexts at once
    (sbdgpu_davidson_batch).  Returns (energies, Ritz vectors, steps)."""
    n = len(ctxs)
    Ws = [np.ascontiguousarray(w, dtype=np.float64).ravel().copy() for w in W0s]
    hs = (_vp * n)(*[c._h for c in ctxs])
    wp = (_dp * n)(*[_p(w, _dp) for w in Ws])
    o = Opts(max_it, max_nb, eps, max_time, precision, 0, restart_keep, restart_prev, PRECOND_DIAGONAL)
    e = np.zeros(n)
    steps = (ctypes.c_int * n)()
    st = (ctypes.c_int * n)()
    rc = lib().sbdgpu_davidson_batch(n, hs, ctypes.byref(o), wp, _p(e, _dp), steps, st, int(max_threads))
    if rc == 1 and all(st[i] == 0 for i in range(n)):
        raise SbdGpuError("status 1: invalid arguments (null pointers or a context given twice)")
    if rc != 0:
        bad = [i for i in range(n) if st[i] != 0]
        msg = lib().sbdgpu_last_error(ctxs[bad[0]]._h) if bad else b""
        raise SbdGpuError(f"status {rc} (problems {bad}): {msg.decode() if msg else ''}")
    return e, Ws, [int(x) for x in steps]


def mlp_loss_grad(w, X, r, den, u, t, wt, S: float = 0.5, eps_reg: float = 1e-12, device: int = 0):
    """Loss and gradient of the learned preconditioner's training kernels
    (sbdgpu_mlp_loss_grad) for master weights w and features X [B, 48]."""
    fp = ctypes.POINTER(ctypes.c_float)
    w = np.ascontiguousarray(w, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    vs = [np.ascontiguousarray(v, dtype=np.float64) for v in (r, den, u, t, wt)]
    B = X.shape[0]
    loss = ctypes.c_double(0.0)
    g = np.zeros_like(w)
    rc = lib().sbdgpu_mlp_loss_grad(int(device), w.ctypes.data_as(fp), B, X.ctypes.data_as(fp),
                                    *[_p(v, _dp) for v in vs], float(S), float(eps_reg), ctypes.byref(loss),
                                    g.ctypes.data_as(fp))
    if rc != 0:
        raise SbdGpuError(f"sbdgpu_mlp_loss_grad failed with status {rc}")
    return loss.value, g


def context_from_integrals(ints, astr, bstr, device: int = 0) -> Context:
    """Context from an object with .norb, .ecore, .h [L,L] and .eri [L,L,L,L]."""
    from .synth import pack_eri
    return Context(ints.norb, astr, bstr, ints.ecore, ints.h, pack_eri(ints.eri), device)


class GenOp:
    """A second-quantised operator on a basis of bit strings on one GPU (the
    generic path: basic/generalop.h GeneralOp, basic/basis.h Basis,
    basic/out_of_place_func/mult.h, lanczos.h, davidson.h).

    states: uint64 array [n, nwords] (or [n] for nwords = 1), site q at bit
    q % 64 of word q // 64; vectors follow its order.  Terms are given per list
    (diagonal, off-diagonal) as sequences of (coef, ops) or (coef, ops, n_dag),
    ops a list of (dag, site) in the order written; n_dag defaults to the
    number of creation operators (ProductOp::n_dag)."""

    def __init__(self, states, sign: bool = True, device: int = 0):
        st = np.ascontiguousarray(states, dtype=np.uint64)
        if st.ndim == 1:
            st = st[:, None]
        self.n, self.nwords = st.shape
        self._states = st
        self._h = _vp()
        rc = lib().sbdgpu_genop_create(ctypes.byref(self._h), int(device), int(self.nwords), int(self.n),
                                       _p(st, _u64p), 1 if sign else 0)
        if rc != 0:
            self._h = _vp()
            raise SbdGpuError(f"sbdgpu_genop_create failed with status {rc}")

    def _check(self, rc: int):
        if rc != 0:
            msg = lib().sbdgpu_genop_last_error(self._h)
            raise SbdGpuError(f"status {rc}: {msg.decode() if msg else ''}")

    def close(self):
        if self._h:
            lib().sbdgpu_genop_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _flatten(terms):
        off, ops, ndag, coef = [0], [], [], []
        for t in terms:
            c, fops = t[0], t[1]
            nd = t[2] if len(t) > 2 else sum(1 for d, _ in fops if d)  # ProductOp::n_dag
            ops.extend(int(q) | (0x10000 if d else 0) for d, q in fops)
            off.append(len(ops))
            ndag.append(int(nd))
            coef.append(float(c))
        return (np.asarray(off, dtype=np.int64), np.asarray(ops if ops else [0], dtype=np.int32),
                np.asarray(ndag if ndag else [0], dtype=np.int32), np.asarray(coef if coef else [0.0]),
                len(coef))

    def set_terms(self, diag_terms, off_terms):
        i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
        d = self._flatten(diag_terms)
        o = self._flatten(off_terms)
        self._keep = (d, o)
        self._check(lib().sbdgpu_genop_set_terms(
            self._h, d[4], _p(d[0], i64p), _p(d[1], i32p), _p(d[2], i32p), _p(d[3], _dp),
            o[4], _p(o[0], i64p), _p(o[1], i32p), _p(o[2], i32p), _p(o[3], _dp)))

    def set_fcidump(self, path: str):
        """The FCIDUMP Hamiltonian as the operator; returns (norb, nelec)."""
        L, N = ctypes.c_int(0), ctypes.c_int(0)
        self._check(lib().sbdgpu_genop_set_fcidump(self._h, path.encode(), ctypes.byref(L), ctypes.byref(N)))
        return L.value, N.value

    def mult(self, C: np.ndarray, W: np.ndarray | None = None) -> np.ndarray:
        """W + H C (W = 0 when not given)."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        out = np.zeros(self.n) if W is None else np.array(W, dtype=np.float64)
        self._check(lib().sbdgpu_genop_mult(self._h, _p(C, _dp), _p(out, _dp)))
        return out

    def mult_device(self, dC_ptr: int, dW_ptr: int) -> None:
        self._check(lib().sbdgpu_genop_mult_device(self._h, _vp(dC_ptr), _vp(dW_ptr)))

    def ham_square(self, W: np.ndarray) -> float:
        """<W|H^2|W> over the expanded space (MeasHamSquare)."""
        W = np.ascontiguousarray(W, dtype=np.float64)
        r = ctypes.c_double(0.0)
        self._check(lib().sbdgpu_genop_ham_square(self._h, _p(W, _dp), ctypes.byref(r)))
        return r.value

    def expand(self, W: np.ndarray, eps_hb: float) -> np.ndarray:
        """The expanded basis (ExpandBasis): uint64 [m, nwords], ascending."""
        W = np.ascontiguousarray(W, dtype=np.float64)
        m = ctypes.c_size_t(0)
        self._check(lib().sbdgpu_genop_expand(self._h, _p(W, _dp), float(eps_hb), None, 0, ctypes.byref(m)))
        out = np.zeros((m.value, self.nwords), dtype=np.uint64)
        self._check(lib().sbdgpu_genop_expand(self._h, _p(W, _dp), float(eps_hb), _p(out, _u64p), m.value,
                                              ctypes.byref(m)))
        return out

    def diagonal(self) -> np.ndarray:
        out = np.empty(self.n)
        self._check(lib().sbdgpu_genop_diagonal(self._h, _p(out, _dp)))
        return out

    def lanczos(self, W0: np.ndarray, max_it: int, eps: float):
        """(energy, Ritz vector, Lanczos steps)."""
        W = np.array(W0, dtype=np.float64)
        e = ctypes.c_double(0.0)
        it = ctypes.c_int(0)
        self._check(lib().sbdgpu_genop_lanczos(self._h, _p(W, _dp), int(max_it), float(eps), ctypes.byref(e),
                                               ctypes.byref(it)))
        return e.value, W, it.value

    def davidson(self, W0: np.ndarray, max_it: int, max_nb: int, eps: float, verbose: bool = False):
        """(energy <W|HW>, W, energy trace, residual trace)."""
        o = Opts(max_it, max_nb, eps, 86400.0, FP64, 1 if verbose else 0, 0, 0, PRECOND_DIAGONAL)
        W = np.array(W0, dtype=np.float64)
        cap = max_it * max_nb
        te, tt = np.zeros(cap), np.zeros(cap)
        e = ctypes.c_double(0.0)
        steps = ctypes.c_int(0)
        self._check(lib().sbdgpu_genop_davidson(self._h, ctypes.byref(o), _p(W, _dp), ctypes.byref(e), _p(te, _dp),
                                                _p(tt, _dp), cap, ctypes.byref(steps)))
        k = min(steps.value, cap)
        return e.value, W, te[:k], tt[:k]
