"""Generate the golden fixtures in this directory by running the reference itself.

The reference (r-ccs-cms/sbd, unmodified headers) is compiled by oracle/Makefile
into oracle/_ref/libsbdref.so at MPI world size 1.  Each case writes a seeded
synthetic FCIDUMP and alpha-string file, runs the reference's own entry points
on them and stores the outputs:

    strings       alpha/beta strings in the reference's order (packed, orbital i = bit i)
    tables        singles/doubles ket lists per bra string (helper.h:132-182)
    hii           diagonal (qcham.h:314-366)
    sigma         H*C for a seeded normalised N(0,1) vector C (mult.h:387-648)
    energy/trace  sbd::tpb::diag at --block 10 --tolerance 1e-8 (sbdiag.h:102-456)
    W             the ground state the reference saves (restart.h:20-66)
    density/rdm   occupations (rdm 0) and 1/2-RDMs (rdm 1, correlation.h)

Usage:  python tests/golden/make_golden.py            (small cases, ~1 min)
        python tests/golden/make_golden.py --config0  (adds the 245,025-determinant
                                                       Davidson; ~40 min on 8 cores)
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from sbd_b200 import synth  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# name: (norb, electrons per spin, strings per spin or None = full space, seed, shuffle)
CASES = {
    "g_L8_3e_full": (8, 3, None, 0, 0),
    "g_L10_3e_sel80": (10, 3, 80, 3, 0),
    "g_L8_3e_shuffled": (8, 3, None, 7, 1),
    "g_L12_4e_full": (12, 4, None, 0, 0),
}


def read_saved_w(path: str, na: int, nb: int) -> np.ndarray:
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(24), dtype=np.uint64)
        ar, br, dl = (int(x) for x in hdr)
        f.read(8 * dl * (ar + br))
        return np.frombuffer(f.read(8 * ar * br), dtype=np.float64).copy()


def seeded_vector(n: int, seed: int) -> np.ndarray:
    C = np.random.default_rng(seed).normal(size=n)
    return C / np.linalg.norm(C)


def run_case(name: str, full_diag: bool) -> None:
    norb, ne, count, seed, shuffle = CASES[name]
    ints, ne, strs = synth.make_small(norb, ne, count, seed)
    with tempfile.TemporaryDirectory() as td:
        fp, dp = synth.write_workload(td, ints, ne, strs)
        ref = oracle.Reference(fp, dp, 20, shuffle)
        out = {"norb": norb, "ne": ne, "seed": seed, "shuffle": shuffle}
        a, b = ref.strings(0), ref.strings(1)
        out["astr"], out["bstr"] = a, b
        for spin in (0, 1):
            for kind, kname in ((0, "s"), (1, "d")):
                off, idx = ref.table(spin, kind)
                out[f"t_{'ab'[spin]}{kname}_off"] = off
                out[f"t_{'ab'[spin]}{kname}_idx"] = idx.astype(np.uint32)
        out["hii"] = ref.hii()
        n = len(a) * len(b)
        C = seeded_vector(n, 1234)
        out["C_seed"] = 1234
        out["C_checksum"] = np.array([C.sum(), (C * np.arange(n)).sum()])
        big = n > 20000
        rows = (0, 8) if big else (0, len(a))
        out["sigma_rows"] = np.array(rows)
        out["sigma"] = ref.sigma(C, rows)
        if not big or full_diag:
            save = os.path.join(td, "wf")
            e, dens, r1, r2 = ref.diag(1000, 10, 1e-8, 0 if big else 1, save)
            out["energy"] = e
            tr = oracle.parse_trace(ref.last_output())
            out["trace"] = np.array([[t[0], t[1], t[2], t[3]] for t in tr])
            out["density"] = dens
            W = read_saved_w(save + "000000", len(a), len(b))
            out["W"] = W
            if not big:
                out["rdm1"], out["rdm2"] = r1, r2
                co, tw = ref.carryover(W, 0.5, 0.01)
                out["carry_ratio_strings"], out["carry_ratio_weight"] = co, tw
                co2, _ = ref.carryover(W, 0.0, 0.01)
                out["carry_thr_strings"] = co2
        ref.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "written", {k: getattr(v, "shape", v) for k, v in out.items() if k in ("energy", "sigma")})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config0", action="store_true", help="also run the full 245,025-determinant Davidson")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    oracle.build()
    for name in CASES:
        if args.only and name != args.only:
            continue
        run_case(name, args.config0 and name == "g_L12_4e_full")


if __name__ == "__main__":
    main()
