"""Mixed-precision path (FP32 vectors and sigma; FP64 dot products, Ritz step,
residual norms and a final FP64 refinement sigma) against the reference's
FP64 results: sigma to FP32 accuracy, ground-state energy within 1e-6 Eh."""
import numpy as np
import pytest

import sbd_b200
from conftest import seeded_vector
from test_gpu_parity import gpu_ctx

pytestmark = pytest.mark.gpu


def test_mixed_sigma_accuracy(golden):
    ctx = gpu_ctx(golden)
    C = seeded_vector(ctx.n, int(golden["C_seed"]))
    r0, r1 = (int(x) for x in golden["sigma_rows"])
    s = ctx.sigma(C, precision=sbd_b200.MIXED)[r0 * ctx.nb:r1 * ctx.nb]
    ref = golden["sigma"]
    # FP32 data and accumulation over a few hundred terms per element
    assert np.abs(s - ref).max() <= 2e-5 * np.abs(ref).max()


def test_mixed_davidson_energy(golden):
    if "energy" not in golden:
        pytest.skip("fixture has no Davidson result")
    ctx = gpu_ctx(golden)
    W0 = np.zeros(ctx.n)
    W0[0] = 1.0
    e, W, te, tt = ctx.davidson(W0, 1000, 10, 1e-4, precision=sbd_b200.MIXED)
    assert abs(e - float(golden["energy"])) < 1e-6
    assert tt[-1] < 1e-4
    assert abs(abs(np.dot(W, golden["W"])) - 1.0) < 1e-6


def test_mixed_davidson_olsen_correction(golden):
    """Olsen's correction (the diagonal correction made P-orthogonal to the
    Ritz vector) reaches the reference's energy with the thick restart; an
    unknown correction is refused."""
    if "energy" not in golden:
        pytest.skip("fixture has no Davidson result")
    ctx = gpu_ctx(golden)
    W0 = np.zeros(ctx.n)
    W0[0] = 1.0
    e, W, te, tt = ctx.davidson(W0, 1000, 10, 1e-5, precision=sbd_b200.MIXED, restart_keep=3, restart_prev=1,
                                precond=sbd_b200.PRECOND_OLSEN)
    assert abs(e - float(golden["energy"])) < 1e-6
    assert tt[-1] < 1e-5
    assert abs(abs(np.dot(W, golden["W"])) - 1.0) < 1e-6
    with pytest.raises(sbd_b200.SbdGpuError):
        ctx.davidson(W0, 10, 10, 1e-5, precision=sbd_b200.MIXED, precond=3)


def test_mixed_thick_restart(golden):
    """Thick restart (the 3 lowest Ritz vectors and their sigma kept) reaches the
    same energy in no more sigma builds than the reference's collapse restart."""
    if "energy" not in golden:
        pytest.skip("fixture has no Davidson result")
    ctx = gpu_ctx(golden)
    W0 = np.zeros(ctx.n)
    W0[0] = 1.0
    e1, _, t1, tt1 = ctx.davidson(W0, 1000, 10, 1e-5, precision=sbd_b200.MIXED)
    e3, W3, t3, tt3 = ctx.davidson(W0, 1000, 10, 1e-5, precision=sbd_b200.MIXED, restart_keep=3)
    assert abs(e3 - float(golden["energy"])) < 1e-6
    assert tt3[-1] < 1e-5
    assert len(t3) <= len(t1)
    # and with the previous step's Ritz vector kept as well (GD+k style)
    e4, W4, t4, tt4 = ctx.davidson(W0, 1000, 10, 1e-5, precision=sbd_b200.MIXED, restart_keep=3, restart_prev=1)
    assert abs(e4 - float(golden["energy"])) < 1e-6
    assert tt4[-1] < 1e-5
    assert len(t4) <= len(t1)
    # the previous vector alone with the collapse restart
    e5, _, t5, tt5 = ctx.davidson(W0, 1000, 10, 1e-5, precision=sbd_b200.MIXED, restart_prev=1)
    assert abs(e5 - float(golden["energy"])) < 1e-6 and tt5[-1] < 1e-5


@pytest.mark.parametrize("norb,ne,count,seed", [(16, 5, 1100, 31), (18, 4, 1500, 32)])
def test_mixed_sigma_dense_same_spin(norb, ne, count, seed):
    """From 1,024 strings per spin the FP32 sigma takes its same-spin terms from
    dense split-FP16 tensor-core products (the string-only operator) plus the
    singles' Coulomb part and the diagonal from a rows kernel: FP32-class
    against the FP64 sigma, and its Davidson lands on the FP64 energy."""
    import sbd_b200
    from sbd_b200 import synth
    from conftest import seeded_vector
    ints, ne, strs = synth.make_small(norb, ne, count, seed)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs)
    C = seeded_vector(ctx.n, seed)
    s64 = ctx.sigma(C)
    s32 = ctx.sigma(C, precision=sbd_b200.MIXED)
    assert np.abs(s32 - s64).max() <= 2e-5 * np.abs(s64).max()
    # an unnormalised vector (the FP16 split rescales by a power of two)
    s32b = ctx.sigma(1e3 * C, precision=sbd_b200.MIXED)
    assert np.abs(s32b - 1e3 * s64).max() <= 2e-5 * 1e3 * np.abs(s64).max()
    W0 = np.random.default_rng(seed).normal(size=ctx.n)
    W0 *= 0.01 / np.linalg.norm(W0)
    W0[0] += 1.0
    e64, _, _, _ = ctx.davidson(W0, 200, 10, 1e-7)
    e32, _, _, tt = ctx.davidson(W0, 200, 10, 1e-4, precision=sbd_b200.MIXED, restart_keep=3, restart_prev=1)
    assert tt[-1] < 1e-4 and abs(e32 - e64) < 1e-6


def test_fp64_same_spin_integer_products_non_finite_input():
    """A NaN or an infinity in C makes sigma non-finite wherever the rows
    kernels make it non-finite (the integer products mark the whole row or
    column they feed), and leaves the finite entries as they were."""
    import sbd_b200
    from sbd_b200 import synth
    from conftest import seeded_vector
    ints, ne, strs = synth.make_small(16, 5, 1100, 33)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs)
    C = seeded_vector(ctx.n, 33)
    C[5 * ctx.nb + 17] = np.nan
    C[700 * ctx.nb + 3] = np.inf
    ctx.set_fp64_same_spin(1)
    ref = ctx.sigma(C)
    ctx.set_fp64_same_spin(0)
    got = ctx.sigma(C)
    bad_ref, bad_got = ~np.isfinite(ref), ~np.isfinite(got)
    assert bad_ref.any() and np.all(bad_got[bad_ref])
    both = ~bad_ref & ~bad_got
    assert both.sum() > ctx.n // 2
    assert np.abs(got[both] - ref[both]).max() <= 1e-12 * np.abs(ref[both]).max()
    # the mixed sigma (split-FP16 same-spin products) carries them as well
    mixed = ctx.sigma(C, precision=sbd_b200.MIXED)
    assert np.all(~np.isfinite(mixed)[bad_ref])
    ctx.close()


@pytest.mark.parametrize("norb,ne,count,seed", [(16, 5, 1100, 31), (18, 4, 1500, 32), (16, 5, 1102, 33)])
def test_fp64_same_spin_integer_products(norb, ne, count, seed):
    """From 1,024 strings per spin (multiples of 4) the FP64 sigma forms its
    same-spin terms as exact INT8 tensor-core products (residues modulo 15
    primes, CRT): equal to the rows kernels to FP64 rounding, for normalised
    and unnormalised vectors; 1,102 strings keep the rows kernels."""
    import sbd_b200
    from sbd_b200 import synth
    from conftest import seeded_vector
    ints, ne, strs = synth.make_small(norb, ne, count, seed)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs)
    C = seeded_vector(ctx.n, seed)
    ctx.set_fp64_same_spin(1)
    ref = ctx.sigma(C)
    ctx.set_fp64_same_spin(0)
    got = ctx.sigma(C)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    C2 = C * np.exp(np.random.default_rng(seed).normal(size=ctx.n) * 4)  # wide dynamic range
    import torch
    free0 = torch.cuda.mem_get_info(0)[0]
    ctx.set_fp64_same_spin(1)  # releases the integer products' buffers (re-made below)
    if count % 4 == 0:
        assert torch.cuda.mem_get_info(0)[0] - free0 >= 15 * (ctx.na ** 2 + ctx.nb ** 2)
    ref2 = ctx.sigma(C2)
    ctx.set_fp64_same_spin(0)
    got2 = ctx.sigma(C2)
    assert np.abs(got2 - ref2).max() <= 1e-12 * np.abs(ref2).max()
    with pytest.raises(sbd_b200.SbdGpuError):
        ctx.set_fp64_same_spin(2)
    ctx.close()
