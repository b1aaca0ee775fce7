"""Failure detection on the GPU without a GPU fault: the bounded mbarrier wait
that the tensor-core kernel uses gives up on a barrier nobody arrives on,
reports it through a status the host reads, and the context keeps working."""
import numpy as np
import pytest

from conftest import load_golden, seeded_vector
from test_gpu_parity import gpu_ctx

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives():
    g = load_golden("g_L8_3e_full")
    ctx = gpu_ctx(g)
    assert ctx.wait_selftest(4096) == (1, 0)
    assert ctx.wait_selftest(1) == (1, 0)
    C = seeded_vector(ctx.n, int(g["C_seed"]))
    r0, r1 = (int(x) for x in g["sigma_rows"])
    s = ctx.sigma(C)[r0 * ctx.nb:r1 * ctx.nb]
    assert np.abs(s - g["sigma"]).max() <= 1e-12 * np.abs(g["sigma"]).max()
    # the tensor-core sigma, whose kernel uses the same wait, also still runs
    # on this context (its timeout flag starts clear)
    import sbd_b200
    stc = ctx.sigma(C, precision=sbd_b200.MIXED_TC)[r0 * ctx.nb:r1 * ctx.nb]
    assert np.abs(stc - g["sigma"]).max() <= 5e-3 * np.abs(g["sigma"]).max()


def test_wait_selftest_rejects_bad_limit():
    import sbd_b200
    ctx = gpu_ctx(load_golden("g_L8_3e_full"))
    with pytest.raises(sbd_b200.SbdGpuError, match="spin_limit"):
        ctx.wait_selftest(0)
    # above the kernel's own poll limit (a caller's huge limit would otherwise
    # make the probe wait for as long as it says)
    with pytest.raises(sbd_b200.SbdGpuError, match="spin_limit"):
        ctx.wait_selftest((1 << 26) + 1)
