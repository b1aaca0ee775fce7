"""Seeded synthetic inputs for the tensor-product-basis Davidson workloads.

The reference ships no usable sample input (its only FCIDUMP is missing), so
every workload here is generated from a seed:

* integrals: h symmetric, diagonal uniform[-2,-0.5] sorted ascending,
  off-diagonal N(0, 0.05^2); (pq|rs) = sum_{l < 2*norb} B_l[p,q] B_l[r,s] with
  B_l symmetric N(0,1)*0.3*exp(-l/norb) (positive semi-definite, 8-fold
  symmetric); E_core = 0.  Draw order: off-diagonal h, diagonal h, then B.
* strings: either every C(norb, ne) string, or every string of excitation rank
  <= 2 from the aufbau string (orbitals 0..ne-1) followed by higher-rank strings
  drawn without replacement with weight exp(-sum of occupied h_pp).  Drawing
  successively in proportion to the weight among the strings not yet drawn is
  the same distribution as Gumbel-top-k over all strings, and needs no
  enumeration of C(norb, ne).  When the rank <= 2 set alone exceeds the request,
  the heaviest rank <= 2 strings are kept.

Files are written in the formats the reference reads: FCIDUMP
(framework/fcidump.h:27-139, integral lines "value i j k l", 8-fold unique,
one-body "value i j 0 0", core "value 0 0 0 0") and the alpha-string text file
(one string per line, rightmost character = orbital 0,
framework/bit_manipulation.h:158-172).
"""
from __future__ import annotations

import itertools
import math
import os
from dataclasses import dataclass

import numpy as np

# Named workloads.  (norb, n_alpha = n_beta, strings per spin or None for the
# full string space).
CONFIGS = {
    "c0_L12_4e_full": (12, 4, None),       # 495 x 495 = 245,025 determinants
    "c1_L26_6e_4000": (26, 6, 4000),       # 16.0M determinants
    "c2_L36_8e_12000": (36, 8, 12000),     # 144M determinants
    "c4_L48_10e_20000": (48, 10, 20000),   # 400M determinants
}


@dataclass
class Integrals:
    norb: int
    ecore: float
    h: np.ndarray      # [L, L]
    eri: np.ndarray    # [L, L, L, L], chemists' (pq|rs)


def make_integrals(norb: int, seed: int) -> Integrals:
    rng = np.random.default_rng(seed)
    off = rng.normal(0.0, 0.05, size=(norb, norb))
    off = np.triu(off, 1)
    h = off + off.T
    h[np.diag_indices(norb)] = np.sort(rng.uniform(-2.0, -0.5, size=norb))
    nl = 2 * norb
    B = rng.normal(0.0, 1.0, size=(nl, norb, norb))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    B *= (0.3 * np.exp(-np.arange(nl) / norb))[:, None, None]
    eri = np.einsum("lpq,lrs->pqrs", B, B, optimize=True)
    return Integrals(norb, 0.0, h, eri)


def pair_index(i: int, j: int) -> int:
    a, b = max(i, j), min(i, j)
    return a * (a + 1) // 2 + b


def pack_eri(eri: np.ndarray) -> np.ndarray:
    """8-fold packed store in the reference layout (chemistry/basic/integrals.h:34-43)."""
    L = eri.shape[0]
    P = L * (L + 1) // 2
    ii, jj = np.tril_indices(L)            # ij = i(i+1)/2 + j with i >= j, row-major tril order
    M = eri[ii, jj][:, ii, jj]             # [P, P]
    a, b = np.tril_indices(P)
    out = np.empty(P * (P + 1) // 2)
    out[a * (a + 1) // 2 + b] = M[a, b]
    return out


def unpack_eri(store: np.ndarray, L: int) -> np.ndarray:
    P = L * (L + 1) // 2
    ii, jj = np.tril_indices(L)
    pidx = np.zeros((L, L), dtype=np.int64)
    pidx[ii, jj] = np.arange(P)
    pidx[jj, ii] = np.arange(P)
    A = pidx[:, :, None, None]
    Bm = pidx[None, None, :, :]
    hi = np.maximum(A, Bm)
    lo = np.minimum(A, Bm)
    return store[hi * (hi + 1) // 2 + lo]


def write_fcidump(path: str, ints: Integrals, nelec: int, ms2: int = 0) -> None:
    L = ints.norb
    lines = [f" &FCI NORB={L},NELEC={nelec},MS2={ms2},",
             "  ORBSYM=" + ",".join(["1"] * L) + ",",
             "  ISYM=1,", " &END"]
    eri = ints.eri
    for i in range(L):
        for j in range(i + 1):
            ij = pair_index(i, j)
            for k in range(L):
                for l in range(k + 1):
                    if pair_index(k, l) > ij:
                        continue
                    lines.append(f"{eri[i, j, k, l]: .16e} {i + 1} {j + 1} {k + 1} {l + 1}")
    for i in range(L):
        for j in range(i + 1):
            lines.append(f"{ints.h[i, j]: .16e} {i + 1} {j + 1} 0 0")
    lines.append(f"{ints.ecore: .16e} 0 0 0 0")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def string_to_text(s: int, norb: int) -> str:
    return "".join("1" if (s >> (norb - 1 - i)) & 1 else "0" for i in range(norb))


def write_strings(path: str, strings, norb: int) -> None:
    with open(path, "w") as f:
        for s in strings:
            f.write(string_to_text(int(s), norb) + "\n")


def full_strings(norb: int, ne: int) -> np.ndarray:
    out = [sum(1 << i for i in c) for c in itertools.combinations(range(norb), ne)]
    return np.array(sorted(out), dtype=np.uint64)


def _rank(s: int, aufbau: int) -> int:
    return bin(s & ~aufbau).count("1")


def _low_rank_strings(norb: int, ne: int, max_rank: int = 2):
    occ = list(range(ne))
    vir = list(range(ne, norb))
    aufbau = (1 << ne) - 1
    out = []
    for k in range(max_rank + 1):
        for holes in itertools.combinations(occ, k):
            for parts in itertools.combinations(vir, k):
                s = aufbau
                for hh in holes:
                    s &= ~(1 << hh)
                for pp in parts:
                    s |= 1 << pp
                out.append(s)
    return out


def selected_strings(norb: int, ne: int, count: int, h_diag: np.ndarray, seed: int) -> np.ndarray:
    aufbau = (1 << ne) - 1
    x = np.exp(-np.asarray(h_diag, dtype=np.float64))
    logw = lambda s: -sum(h_diag[p] for p in range(norb) if (s >> p) & 1)
    low = _low_rank_strings(norb, ne, 2)
    if len(low) >= count:
        low.sort(key=lambda s: (-logw(s), s))
        return np.array(sorted(low[:count]), dtype=np.uint64)
    chosen = set(low)
    # e[k][i] = elementary symmetric polynomial of degree k over x[i:]
    e = np.zeros((ne + 1, norb + 1))
    e[0, :] = 1.0
    for i in range(norb - 1, -1, -1):
        for k in range(1, ne + 1):
            e[k, i] = e[k, i + 1] + x[i] * e[k - 1, i + 1]
    rng = np.random.default_rng(seed)
    need = count - len(chosen)
    guard = 0
    while need > 0:
        guard += 1
        if guard > 1000 * count:
            raise RuntimeError("string sampler did not find enough strings")
        k = ne
        s = 0
        u = rng.random(norb)
        for i in range(norb):
            if k == 0:
                break
            p_in = x[i] * e[k - 1, i + 1] / e[k, i]
            if u[i] < p_in:
                s |= 1 << i
                k -= 1
        if _rank(s, aufbau) <= 2 or s in chosen:
            continue
        chosen.add(s)
        need -= 1
    return np.array(sorted(chosen), dtype=np.uint64)


def make_workload(name: str, seed: int = 0):
    """Return (Integrals, n_electrons_per_spin, sorted strings) for a named workload."""
    norb, ne, count = CONFIGS[name]
    ints = make_integrals(norb, seed)
    if count is None:
        strs = full_strings(norb, ne)
    else:
        strs = selected_strings(norb, ne, count, np.diag(ints.h), seed + 1)
    return ints, ne, strs


def make_small(norb: int, ne: int, count: int | None, seed: int):
    ints = make_integrals(norb, seed)
    if count is None or count >= math.comb(norb, ne):
        strs = full_strings(norb, ne)
    else:
        strs = selected_strings(norb, ne, count, np.diag(ints.h), seed + 1)
    return ints, ne, strs


def write_workload(dirpath: str, ints: Integrals, ne: int, strs) -> tuple[str, str]:
    os.makedirs(dirpath, exist_ok=True)
    fp = os.path.join(dirpath, "fcidump.txt")
    dp = os.path.join(dirpath, "alphadets.txt")
    write_fcidump(fp, ints, 2 * ne)
    write_strings(dp, strs, ints.norb)
    return fp, dp
