"""FCIDUMP and alpha-string file readers with the reference's semantics.

* FCIDUMP (framework/fcidump.h:27-139): header between "&FCI" and "&END"
  joined and split on ',' into KEY=VALUE pairs; then one integral per line,
  "value i j k l" (1-based; k=l=0 one-body; all zero core energy).
  Integral placement follows chemistry/basic/makeintegrals.h:10-55: the
  one-body value is stored symmetric, two-body values fill the 8-fold
  symmetric store.
* Alpha strings (chemistry/basic/makedeterminants.h:160-185): one string per
  line, rightmost character = orbital 0; the set is sorted ascending by its
  numeric value and duplicates are dropped (framework/bit_manipulation.h:324-330).
"""
from __future__ import annotations

import numpy as np


class FCIDump:
    def __init__(self, header: dict, norb: int, nelec: int, ecore: float, h: np.ndarray, eri: np.ndarray):
        self.header = header
        self.norb = norb
        self.nelec = nelec
        self.ecore = ecore
        self.h = h
        self.eri = eri


def read_fcidump(path: str) -> FCIDump:
    header_text = ""
    in_header = True
    rows = []
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            if not line or line[0] == "!":
                continue
            if in_header:
                if "&END" in line:
                    in_header = False
                    continue
                pos = line.find("&FCI")
                if pos >= 0:
                    line = line[:pos] + line[pos + 4:]
                header_text += line
            else:
                parts = line.split()
                if len(parts) < 5:
                    continue
                rows.append((float(parts[0]), int(parts[1]), int(parts[2]), int(parts[3]), int(parts[4])))
    header = {}
    for tok in header_text.split(","):
        if "=" in tok:
            k, v = tok.split("=", 1)
            header[k.strip(" \t")] = v.strip(" \t")
    norb = int(header["NORB"])
    nelec = int(header.get("NELEC", "0"))
    L = norb
    h = np.zeros((L, L))
    eri = np.zeros((L, L, L, L))
    ecore = 0.0
    for v, i, j, k, l in rows:
        if i == 0 and j == 0 and k == 0 and l == 0:
            ecore = v
        elif k == 0 and l == 0:
            h[i - 1, j - 1] = v
            h[j - 1, i - 1] = v
        else:
            p, q, r, s = i - 1, j - 1, k - 1, l - 1
            for (a, b, c, d) in ((p, q, r, s), (q, p, r, s), (p, q, s, r), (q, p, s, r),
                                 (r, s, p, q), (s, r, p, q), (r, s, q, p), (s, r, q, p)):
                eri[a, b, c, d] = v
    return FCIDump(header, norb, nelec, ecore, h, eri)


def read_strings(path: str, norb: int) -> np.ndarray:
    out = set()
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            if not line:
                continue
            v = 0
            for i in range(norb):
                if line[norb - 1 - i] == "1":
                    v |= 1 << i
            out.add(v)
    return np.array(sorted(out), dtype=np.uint64)
