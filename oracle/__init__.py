"""ctypes wrappers for the two parity checkers.  TEST INFRASTRUCTURE ONLY.

* ``Reference``: the unmodified reference headers behind oracle/ref_driver.cc
  (built into oracle/_ref/libsbdref.so).
* ``Oracle``: this repository's C restatement, oracle/sbd_oracle.c
  (oracle/_ref/libsbdoracle.so).

Only tests, the smoke check and the bench's CPU-baseline leg import this
package; the product path never does.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libsbdref.so")
ORACLE_SO = os.path.join(HERE, "_ref", "libsbdoracle.so")

_u64p = ctypes.POINTER(ctypes.c_uint64)
_dp = ctypes.POINTER(ctypes.c_double)


def build() -> None:
    """Compile the checkers (make in oracle/; the reference part only where the
    reference checkout exists)."""
    ref = "/root/reference"  # the reference checkout, where this machine has one
    args = ["make", "-s", "-C", HERE] + ([f"REF={ref}"] if os.path.exists(os.path.join(ref, "include")) else [])
    subprocess.run(args, check=True)


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def reference_available() -> bool:
    return os.path.exists(REF_SO)


class Reference:
    """The reference itself (r-ccs-cms/sbd) at MPI world size 1."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(REF_SO)
            vp = ctypes.c_void_p
            lib.sbdref_open.restype = vp
            lib.sbdref_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
            lib.sbdref_close.argtypes = [vp]
            lib.sbdref_norb.argtypes = [vp]
            lib.sbdref_count.restype = ctypes.c_size_t
            lib.sbdref_count.argtypes = [vp, ctypes.c_int]
            lib.sbdref_ecore.restype = ctypes.c_double
            lib.sbdref_ecore.argtypes = [vp]
            lib.sbdref_strings.argtypes = [vp, ctypes.c_int, _u64p]
            lib.sbdref_tables.restype = ctypes.c_size_t
            lib.sbdref_tables.argtypes = [vp, ctypes.c_int, ctypes.c_int, _u64p, _u64p]
            lib.sbdref_hii.argtypes = [vp, _dp]
            lib.sbdref_mult.argtypes = [vp, _dp, _dp, ctypes.c_size_t, ctypes.c_size_t]
            lib.sbdref_diag.restype = ctypes.c_double
            lib.sbdref_diag.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                        _dp, _dp, _dp, ctypes.c_char_p]
            lib.sbdref_last_output.restype = ctypes.c_size_t
            lib.sbdref_last_output.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
            lib.sbdref_correlation.argtypes = [vp, _dp, _dp, _dp]
            lib.sbdref_occupation.argtypes = [vp, _dp, _dp]
            lib.sbdref_carryover.restype = ctypes.c_size_t
            lib.sbdref_carryover.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_double, _u64p, _dp]
            lib.sbdref_max_threads.restype = ctypes.c_int
            lib.sbdref_save_wavefunction.argtypes = [vp, ctypes.c_char_p, _dp]
            lib.sbdref_load_wavefunction.argtypes = [vp, ctypes.c_char_p, _dp]
            cls._lib = lib
        return cls._lib

    def __init__(self, fcidump_path: str, adet_path: str, bit_length: int = 20, shuffle: int = 0):
        lib = self.lib()
        self.h = lib.sbdref_open(fcidump_path.encode(), adet_path.encode(), bit_length, shuffle)
        if not self.h:
            raise RuntimeError("reference failed to open inputs")
        self.norb = lib.sbdref_norb(self.h)
        self.na = lib.sbdref_count(self.h, 0)
        self.nb = lib.sbdref_count(self.h, 1)

    def close(self):
        if self.h:
            self.lib().sbdref_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def strings(self, spin: int) -> np.ndarray:
        n = self.na if spin == 0 else self.nb
        out = np.zeros(n, dtype=np.uint64)
        self.lib().sbdref_strings(self.h, spin, _ptr(out, _u64p))
        return out

    def table(self, spin: int, kind: int):
        lib = self.lib()
        n = self.na if spin == 0 else self.nb
        tot = lib.sbdref_tables(self.h, spin, kind, None, None)
        off = np.zeros(n + 1, dtype=np.uint64)
        idx = np.zeros(max(tot, 1), dtype=np.uint64)
        lib.sbdref_tables(self.h, spin, kind, _ptr(off, _u64p), _ptr(idx, _u64p))
        return off, idx[:tot]

    def hii(self) -> np.ndarray:
        out = np.zeros(self.na * self.nb)
        self.lib().sbdref_hii(self.h, _ptr(out, _dp))
        return out

    def sigma(self, C: np.ndarray, rows=None) -> np.ndarray:
        C = np.ascontiguousarray(C, dtype=np.float64).ravel()
        r0, r1 = (0, self.na) if rows is None else rows
        out = np.zeros((r1 - r0) * self.nb)
        self.lib().sbdref_mult(self.h, _ptr(C, _dp), _ptr(out, _dp), r0, r1)
        return out

    def diag(self, max_it: int, max_nb: int, eps: float, do_rdm: int = 0, savename: str | None = None):
        L = self.norb
        dens = np.zeros(2 * L)
        r1 = np.zeros(2 * L * L) if do_rdm else None
        r2 = np.zeros(4 * L ** 4) if do_rdm else None
        e = self.lib().sbdref_diag(self.h, max_it, max_nb, eps, do_rdm, _ptr(dens, _dp), _ptr(r1, _dp),
                                   _ptr(r2, _dp), savename.encode() if savename else None)
        return e, dens, r1, r2

    def last_output(self) -> str:
        lib = self.lib()
        n = lib.sbdref_last_output(self.h, None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        lib.sbdref_last_output(self.h, buf, n + 1)
        return buf.value.decode()

    def correlation(self, W: np.ndarray):
        L = self.norb
        W = np.ascontiguousarray(W, dtype=np.float64).ravel()
        r1 = np.zeros(2 * L * L)
        r2 = np.zeros(4 * L ** 4)
        self.lib().sbdref_correlation(self.h, _ptr(W, _dp), _ptr(r1, _dp), _ptr(r2, _dp))
        return r1, r2

    def occupation(self, W: np.ndarray) -> np.ndarray:
        W = np.ascontiguousarray(W, dtype=np.float64).ravel()
        d = np.zeros(2 * self.norb)
        self.lib().sbdref_occupation(self.h, _ptr(W, _dp), _ptr(d, _dp))
        return d

    def carryover(self, W: np.ndarray, ratio: float, threshold: float):
        W = np.ascontiguousarray(W, dtype=np.float64).ravel()
        out = np.zeros(self.na, dtype=np.uint64)
        w = np.zeros(1)
        n = self.lib().sbdref_carryover(self.h, _ptr(W, _dp), ratio, threshold, _ptr(out, _u64p), _ptr(w, _dp))
        return out[:n], float(w[0])

    def save_wavefunction(self, prefix: str, W: np.ndarray) -> None:
        """SaveWavefunction (restart.h:20-66): writes prefix + '000000'."""
        W = np.ascontiguousarray(W, dtype=np.float64).ravel()
        self.lib().sbdref_save_wavefunction(self.h, prefix.encode(), _ptr(W, _dp))

    def load_wavefunction(self, prefix: str) -> np.ndarray:
        """LoadWavefunction (restart.h:414-658) onto this handle's basis."""
        out = np.zeros(self.na * self.nb)
        self.lib().sbdref_load_wavefunction(self.h, prefix.encode(), _ptr(out, _dp))
        return out


_TRACE = re.compile(r"Davidson iteration (\d+)\.(\d+) \(tol=([^)]+)\):\s*(\S+)")


def parse_trace(text: str):
    """(it, ib, tol, E0) per Davidson step from the reference's log
    (chemistry/tpb/davidson.h:834-846)."""
    return [(int(m.group(1)), int(m.group(2)), float(m.group(3)), float(m.group(4)))
            for m in _TRACE.finditer(text)]


class Oracle:
    """C restatement of the reference algorithm (oracle/sbd_oracle.c)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(ORACLE_SO)
            vp = ctypes.c_void_p
            lib.orc_create.restype = vp
            lib.orc_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t, _u64p, _u64p,
                                       ctypes.c_double, _dp, _dp]
            lib.orc_destroy.argtypes = [vp]
            lib.orc_table.restype = ctypes.c_uint64
            lib.orc_table.argtypes = [vp, ctypes.c_int, ctypes.c_int, _u64p, _u64p]
            lib.orc_hij.restype = ctypes.c_double
            lib.orc_hij.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]
            lib.orc_hii.argtypes = [vp, _dp]
            lib.orc_sigma.argtypes = [vp, _dp, _dp, ctypes.c_size_t, ctypes.c_size_t]
            lib.orc_davidson.restype = ctypes.c_double
            lib.orc_davidson.argtypes = [vp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp,
                                         ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
            lib.orc_correlation.argtypes = [vp, _dp, _dp, _dp]
            lib.orc_occupation.argtypes = [vp, _dp, _dp]
            cls._lib = lib
        return cls._lib

    def __init__(self, norb: int, astr, bstr, ecore: float, h: np.ndarray, eri: np.ndarray):
        self.norb = norb
        self.astr = np.ascontiguousarray(astr, dtype=np.uint64)
        self.bstr = np.ascontiguousarray(bstr, dtype=np.uint64)
        self.na, self.nb = len(self.astr), len(self.bstr)
        hh = np.ascontiguousarray(h, dtype=np.float64)
        ee = np.ascontiguousarray(eri, dtype=np.float64)
        self.p = self.lib().orc_create(norb, self.na, self.nb, _ptr(self.astr, _u64p), _ptr(self.bstr, _u64p),
                                       ecore, _ptr(hh, _dp), _ptr(ee, _dp))

    def __del__(self):
        try:
            if self.p:
                self.lib().orc_destroy(self.p)
                self.p = None
        except Exception:
            pass

    def table(self, spin: int, kind: int):
        n = self.na if spin == 0 else self.nb
        tot = self.lib().orc_table(self.p, spin, kind, None, None)
        off = np.zeros(n + 1, dtype=np.uint64)
        idx = np.zeros(max(tot, 1), dtype=np.uint64)
        self.lib().orc_table(self.p, spin, kind, _ptr(off, _u64p), _ptr(idx, _u64p))
        return off, idx[:tot]

    def hij(self, ia, ib, ja, jb) -> float:
        return self.lib().orc_hij(self.p, int(ia), int(ib), int(ja), int(jb))

    def hii(self) -> np.ndarray:
        out = np.zeros(self.na * self.nb)
        self.lib().orc_hii(self.p, _ptr(out, _dp))
        return out

    def sigma(self, C: np.ndarray, rows=None) -> np.ndarray:
        C = np.ascontiguousarray(C, dtype=np.float64).ravel()
        r0, r1 = (0, self.na) if rows is None else rows
        out = np.zeros((r1 - r0) * self.nb)
        self.lib().orc_sigma(self.p, _ptr(C, _dp), _ptr(out, _dp), r0, r1)
        return out

    def davidson(self, W0: np.ndarray, max_it: int, max_nb: int, eps: float, max_trace: int = 100000):
        W = np.ascontiguousarray(W0, dtype=np.float64).ravel().copy()
        te = np.zeros(max_trace)
        tt = np.zeros(max_trace)
        ns = ctypes.c_int(0)
        e = self.lib().orc_davidson(self.p, _ptr(W, _dp), max_it, max_nb, eps, _ptr(te, _dp), _ptr(tt, _dp),
                                    max_trace, ctypes.byref(ns))
        n = min(ns.value, max_trace)
        return e, W, te[:n], tt[:n]

    def correlation(self, W: np.ndarray):
        L = self.norb
        W = np.ascontiguousarray(W, dtype=np.float64).ravel()
        r1 = np.zeros(2 * L * L)
        r2 = np.zeros(4 * L ** 4)
        self.lib().orc_correlation(self.p, _ptr(W, _dp), _ptr(r1, _dp), _ptr(r2, _dp))
        return r1, r2

    def occupation(self, W: np.ndarray) -> np.ndarray:
        W = np.ascontiguousarray(W, dtype=np.float64).ravel()
        d = np.zeros(2 * self.norb)
        self.lib().orc_occupation(self.p, _ptr(W, _dp), _ptr(d, _dp))
        return d


def phase(astr: np.ndarray, bstr: np.ndarray) -> np.ndarray:
    """Diagonal +-1 that maps the reference's interleaved spin-orbital sign
    convention to the alpha-string-then-beta-string convention:
    phi(a, b) = (-1)^#{(p in a, r in b) : r < p}.  Returned as [na, nb]."""
    L = 64
    a = np.asarray(astr, dtype=np.uint64)
    b = np.asarray(bstr, dtype=np.uint64)
    cnt = np.zeros((len(a), len(b)), dtype=np.int64)
    for p in range(L):
        ap = ((a >> np.uint64(p)) & np.uint64(1)).astype(np.int64)
        if not ap.any():
            continue
        mask = np.uint64((1 << p) - 1)
        bc = np.array([bin(int(x) & int(mask)).count("1") for x in (b & mask)], dtype=np.int64)
        cnt += ap[:, None] * bc[None, :]
    return np.where(cnt % 2 == 1, -1.0, 1.0)


REF_GENERIC_SO = os.path.join(HERE, "_ref", "libsbdref_generic.so")


class RefGeneric:
    """The reference's own generic operator algebra (basic/): GeneralOp built
    with its operators, NormalOrdering, Simplify and GeneralOp_From_FCIDump,
    exported as (diagonal, off-diagonal) lists of (coef, [(dag, site), ...])."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(REF_GENERIC_SO)
            vp = ctypes.c_void_p
            ip = ctypes.POINTER(ctypes.c_int)
            lib.sbdrefg_new.restype = vp
            lib.sbdrefg_free.argtypes = [vp]
            lib.sbdrefg_add_product.argtypes = [vp, ctypes.c_double, ctypes.c_int, ip]
            lib.sbdrefg_normal_order.argtypes = [vp, ctypes.c_int]
            lib.sbdrefg_simplify.argtypes = [vp]
            lib.sbdrefg_from_fcidump.restype = vp
            lib.sbdrefg_from_fcidump.argtypes = [ctypes.c_char_p, ip, ip]
            lib.sbdrefg_count.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                                          ctypes.POINTER(ctypes.c_size_t)]
            lib.sbdrefg_export.argtypes = [vp, ctypes.c_int, _dp, ip, ctypes.POINTER(ctypes.c_int64), ip]
            cls._lib = lib
        return cls._lib

    def __init__(self, handle=None):
        self.h = handle if handle is not None else self.lib().sbdrefg_new()

    @classmethod
    def from_fcidump(cls, path: str):
        L, N = ctypes.c_int(0), ctypes.c_int(0)
        h = cls.lib().sbdrefg_from_fcidump(path.encode(), ctypes.byref(L), ctypes.byref(N))
        return cls(h), L.value, N.value

    def close(self):
        if self.h:
            self.lib().sbdrefg_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, coef: float, ops):
        arr = np.asarray([int(q) | (0x10000 if d else 0) for d, q in ops] or [0], dtype=np.int32)
        self.lib().sbdrefg_add_product(self.h, float(coef), len(ops), arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))

    def normal_order(self, sign: bool = True):
        self.lib().sbdrefg_normal_order(self.h, 1 if sign else 0)

    def simplify(self):
        self.lib().sbdrefg_simplify(self.h)

    def terms(self):
        out = []
        for lst in (0, 1):
            nt, no = ctypes.c_size_t(0), ctypes.c_size_t(0)
            self.lib().sbdrefg_count(self.h, lst, ctypes.byref(nt), ctypes.byref(no))
            coef = np.zeros(max(nt.value, 1))
            ndag = np.zeros(max(nt.value, 1), dtype=np.int32)
            off = np.zeros(nt.value + 1, dtype=np.int64)
            ops = np.zeros(max(no.value, 1), dtype=np.int32)
            ip = ctypes.POINTER(ctypes.c_int)
            self.lib().sbdrefg_export(self.h, lst, coef.ctypes.data_as(_dp), ndag.ctypes.data_as(ip),
                                      off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ops.ctypes.data_as(ip))
            out.append([(float(coef[m]), [(bool(x >> 16 & 1), int(x & 0xFFFF)) for x in ops[off[m]:off[m + 1]]])
                        for m in range(nt.value)])
        return out[0], out[1]
