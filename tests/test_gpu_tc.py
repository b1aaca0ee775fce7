"""Alpha-beta sigma term on the tensor cores (tcgen05, BF16 operands, FP32
accumulation) against the FP64 path, and the Davidson that uses it while the
residual is large (then FP32, then an FP64 refinement sigma) against the
reference energy."""
import numpy as np
import pytest

import oracle
import sbd_b200
from sbd_b200 import synth
from conftest import seeded_vector
from test_gpu_parity import gpu_ctx

pytestmark = pytest.mark.gpu

# BF16 operands (8-bit significand): the alpha-beta sums carry ~0.1 % errors
TC_TOL = 5e-3


def test_tc_sigma_close_to_fp64(golden):
    ctx = gpu_ctx(golden)
    C = seeded_vector(ctx.n, int(golden["C_seed"]))
    s64 = ctx.sigma(C)
    s32 = ctx.sigma(C, precision=sbd_b200.MIXED)
    stc = ctx.sigma(C, precision=sbd_b200.MIXED_TC)
    scale = np.abs(s64).max()
    assert np.abs(s32 - s64).max() <= 2e-5 * scale
    assert np.abs(stc - s64).max() <= TC_TOL * scale


@pytest.mark.parametrize("norb,ne,count,seed", [(16, 5, 400, 12), (20, 3, 600, 13), (24, 4, 900, 14)])
def test_tc_sigma_several_m_tiles(norb, ne, count, seed):
    """norb 16-24: 136-300 folded pair rows, i.e. 2-3 tensor-core M tiles."""
    ints, ne, strs = synth.make_small(norb, ne, count, seed)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs)
    C = seeded_vector(ctx.n, seed)
    s64 = ctx.sigma(C)
    stc = ctx.sigma(C, precision=sbd_b200.MIXED_TC)
    assert np.abs(stc - s64).max() <= TC_TOL * np.abs(s64).max()
    # and row-wise against the C restatement of the reference
    orc = oracle.Oracle(norb, strs, strs, ints.ecore, ints.h, ints.eri)
    ref = orc.sigma(C, (0, 16))
    assert np.abs(s64[:16 * ctx.nb] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_tc_davidson_energy(golden):
    if "energy" not in golden:
        pytest.skip("fixture has no Davidson result")
    ctx = gpu_ctx(golden)
    W0 = np.zeros(ctx.n)
    W0[0] = 1.0
    e, W, te, tt = ctx.davidson(W0, 1000, 10, 1e-4, precision=sbd_b200.MIXED_TC)
    assert abs(e - float(golden["energy"])) < 1e-6
    assert tt[-1] < 1e-4
