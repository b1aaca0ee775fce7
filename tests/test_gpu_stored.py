"""Method 1 (stored Hamiltonian) on the GPU against the reference's outputs.

The reference's makeQCham (chemistry/tpb/qcham.h:204-300) stores, for every
bra determinant (ia, ib), one element per alpha single and double of ia, per
beta single and double of ib, and per pair of an alpha single of ia with a
beta single of ib; the count follows from the reference's own tables.  Its
stored mult (chemistry/tpb/mult.h:13-123) gives the same sigma as the direct
one, so the golden sigma, energies and traces apply unchanged."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
import sbd_b200
from conftest import golden_integrals, load_golden, seeded_vector
from sbd_b200 import build, synth
from test_gpu_parity import _seeded_system, gpu_ctx

pytestmark = pytest.mark.gpu


def _stored_count(g):
    sa = np.diff(g["t_as_off"].astype(np.int64))
    da = np.diff(g["t_ad_off"].astype(np.int64))
    sb = np.diff(g["t_bs_off"].astype(np.int64))
    db = np.diff(g["t_bd_off"].astype(np.int64))
    na, nb = len(sa), len(sb)
    return int(nb * (sa + da).sum() + na * (sb + db).sum() + sa.sum() * sb.sum())


def test_stored_count_and_sigma(golden):
    ctx = gpu_ctx(golden)
    nnz = ctx.store_hamiltonian()
    assert nnz == _stored_count(golden)
    C = seeded_vector(ctx.n, int(golden["C_seed"]))
    r0, r1 = (int(x) for x in golden["sigma_rows"])
    s = ctx.sigma(C)[r0 * ctx.nb:r1 * ctx.nb]
    ref = golden["sigma"]
    assert np.abs(s - ref).max() <= 1e-12 * np.abs(ref).max()
    # releasing returns to the on-the-fly build with the same result
    ctx.release_hamiltonian()
    s2 = ctx.sigma(C)[r0 * ctx.nb:r1 * ctx.nb]
    assert np.abs(s2 - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("norb,ne,count,seed", [(9, 3, 40, 5), (10, 4, 60, 6)])
def test_stored_sigma_ragged_vs_oracle(norb, ne, count, seed):
    ints, a, b = _seeded_system(norb, ne, count, seed, ragged=True)
    assert len(a) != len(b)
    ctx = sbd_b200.context_from_integrals(ints, a, b)
    ctx.store_hamiltonian()
    orc = oracle.Oracle(norb, a, b, ints.ecore, ints.h, ints.eri)
    C = seeded_vector(ctx.n, seed)
    ref = orc.sigma(C)
    assert np.abs(ctx.sigma(C) - ref).max() <= 1e-12 * np.abs(ref).max()


def test_stored_davidson(golden):
    if "energy" not in golden:
        pytest.skip("fixture has no Davidson result")
    ctx = gpu_ctx(golden)
    ctx.store_hamiltonian()
    W0 = np.zeros(ctx.n)
    W0[0] = 1.0
    e, W, te, tt = ctx.davidson(W0, 1000, 10, 1e-8)
    assert abs(e - float(golden["energy"])) < 1e-10
    tr = golden["trace"]
    k = len(tr) if ctx.n <= 20000 else 4
    if ctx.n <= 20000:
        assert len(te) == len(tr)
    np.testing.assert_allclose(tt[:k], tr[:k, 2], rtol=2e-5)
    assert tt[-1] < 1e-8
    assert abs(abs(np.dot(W, golden["W"])) - 1.0) < 1e-10


def test_stored_full_config0_vs_oracle():
    """Every row at 245,025 determinants (349M stored elements, 4.2 GB)."""
    g = load_golden("g_L12_4e_full")
    ctx = gpu_ctx(g)
    assert ctx.store_hamiltonian() == _stored_count(g)
    fd = golden_integrals(g)
    orc = oracle.Oracle(12, g["astr"], g["bstr"], fd.ecore, fd.h, fd.eri)
    C = seeded_vector(ctx.n, 78)
    ref = orc.sigma(C)
    assert np.abs(ctx.sigma(C) - ref).max() <= 1e-12 * np.abs(ref).max()


def test_stored_too_large_is_refused():
    """16M determinants would need ~480 GB of stored elements: refused before
    any allocation, and the context keeps working on the fly."""
    ints, ne, strs = synth.make_workload("c1_L26_6e_4000", seed=0)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs)
    with pytest.raises(sbd_b200.SbdGpuError, match="stored Hamiltonian: needs"):
        ctx.store_hamiltonian()
    x = seeded_vector(ctx.n, 3)
    hx = ctx.sigma(x)
    assert np.isfinite(hx).all()


def test_sample_driver_method1():
    g = load_golden("g_L8_3e_full")
    exe = build.build_driver()
    ints, ne, strs = synth.make_small(8, 3, None, int(g["seed"]))
    with tempfile.TemporaryDirectory() as td:
        fp, dp = synth.write_workload(td, ints, ne, strs)
        r = subprocess.run([exe, "--fcidump", fp, "--adetfile", dp, "--method", "1", "--block", "10",
                            "--iteration", "1000", "--tolerance", "1e-8", "--rdm", "0"],
                           cwd=td, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert "Elapsed time for make Hamiltonian" in r.stdout
        e = float(re.search(r"Sample-based diagonalization: Energy = (\S+)", r.stdout).group(1))
        assert abs(e - float(g["energy"])) < 1e-10
