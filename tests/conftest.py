import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the in-tree libsbdgpu.so")


def _ensure_built():
    import oracle
    from sbd_b200 import build
    # make builds the reference checker only where the reference checkout is present
    if (not os.path.exists(oracle.ORACLE_SO) or not oracle.reference_available()
            or not os.path.exists(oracle.REF_GENERIC_SO)):
        oracle.build()
    if not os.path.exists(build.LIB):
        build.build_lib()


_ensure_built()


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


GOLDEN_CASES = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


@pytest.fixture(params=GOLDEN_CASES)
def golden(request):
    g = load_golden(request.param)
    g["name"] = request.param
    return g


def golden_integrals(g):
    """Rebuild the integrals of a golden case exactly as the reference read them."""
    import tempfile
    from sbd_b200 import fcidump, synth
    ints = synth.make_integrals(int(g["norb"]), int(g["seed"]))
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "fcidump.txt")
        synth.write_fcidump(p, ints, 2 * int(g["ne"]))
        fd = fcidump.read_fcidump(p)
    return fd


def seeded_vector(n, seed):
    C = np.random.default_rng(seed).normal(size=n)
    return C / np.linalg.norm(C)
