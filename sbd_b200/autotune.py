"""Launch shapes of the FP64 alpha-beta sigma kernel by size class.

The alpha-beta kernel (csrc/sigma.cu) takes G alpha singles per CTA and NT
threads per CTA.  The default picks the largest G whose integral block fits in
shared memory and 512 or 1024 threads, which suits bases of thousands of
strings; on small bases (hundreds of beta strings, a few warps of work per
CTA) smaller CTAs and groups keep more SMs busy.  `tune` times every shape
that fits (sbdgpu_autotune) on a set of contexts and keeps, per size class,
the shape with the least total sigma time; the table is a JSON file
(sbd_b200/tuning.json is the one committed, made on a B200 by

    python -m sbd_b200.autotune --out sbd_b200/tuning.json

over the many-small-problems workload) and `apply` sets a context's shape
from it.
"""
from __future__ import annotations

import argparse
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.json")

_NB_EDGES = [256, 512, 1024, 2048, 4096, 8192, 16384, 65536]
_P_EDGES = [64, 128, 256, 512, 1024, 4096]


def size_class(na: int, nb: int, norb: int) -> str:
    """Bucket of (beta strings, folded orbital pairs P = L(L+1)/2)."""
    P = norb * (norb + 1) // 2
    bn = next(e for e in _NB_EDGES + [1 << 62] if nb <= e)
    bp = next(e for e in _P_EDGES + [1 << 62] if P <= e)
    return f"nb<={bn},P<={bp}"


def tune(ctxs, reps: int = 3):
    """{class: {"ab_group", "ab_threads", "ms", "default_ms", "contexts"}}."""
    per = {}
    for c in ctxs:
        key = size_class(c.na, c.nb, c.norb)
        c.set_tuning(0, 0)
        c.hii()
        default_ms = _time_default(c, reps)
        g, t, ms = c.autotune(reps)
        e = per.setdefault(key, {"shapes": {}, "default_ms": 0.0, "contexts": 0})
        e["default_ms"] += default_ms
        e["contexts"] += 1
        e["shapes"][(g, t)] = e["shapes"].get((g, t), 0.0) + ms
    table = {}
    for key, e in per.items():
        (g, t), ms = min(e["shapes"].items(), key=lambda kv: kv[1])
        table[key] = {"ab_group": g, "ab_threads": t, "ms": ms, "default_ms": e["default_ms"],
                      "contexts": e["contexts"]}
    return table


def _time_default(c, reps):
    """Device time of the default shape's FP64 sigma (the context's event split)."""
    C = np.ones(c.n) / math.sqrt(c.n)
    c.sigma(C)
    tot = 0.0
    for _ in range(reps):
        c.sigma(C)
        tot += c.last_sigma_ms()[3]
    return tot / reps


def load(path: str = TABLE):
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f).get("classes", {})


def apply(ctx, table) -> bool:
    """Set the context's shape from the table; False when its class is absent
    or the shape does not fit (the default stays)."""
    e = table.get(size_class(ctx.na, ctx.nb, ctx.norb))
    if not e:
        return False
    try:
        ctx.set_tuning(e["ab_group"], e["ab_threads"])
        return True
    except Exception:
        return False


def _workload(n, seed=2024):
    """The many-small-problems workload: norb 10-20, 3-6 electrons per spin,
    200-2000 selected strings per spin (capped at C(norb, ne))."""
    from . import synth
    rng = np.random.default_rng(seed)
    for i in range(n):
        L = int(rng.integers(10, 21))
        ne = int(rng.integers(3, 7))
        cnt = min(int(rng.integers(200, 2001)), math.comb(L, ne))
        yield synth.make_small(L, ne, cnt, 1000 + i)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TABLE)
    ap.add_argument("--problems", type=int, default=64)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    from . import context_from_integrals
    ctxs = [context_from_integrals(ints, strs, strs) for ints, ne, strs in _workload(args.problems)]
    table = tune(ctxs, args.reps)
    for c in ctxs:
        c.close()
    with open(args.out, "w") as f:
        json.dump({"device": "B200", "made_by": "python -m sbd_b200.autotune", "problems": args.problems,
                   "classes": table}, f, indent=1, sort_keys=True)
    print(json.dumps(table, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()
