"""The no-allocation sigma entry point, sbdgpu_sigma_device_noalloc.

It serves callers that cannot allocate device memory in the middle of a run:
their device memory is owned by a pre-reserved pool or arena, or the call sits
on a path that must not synchronise the device as cudaMalloc/cudaFree can.
Its scratch is a fixed 12 MiB device array inside the library, so it handles
at most 524,288 determinants and needs the context's set-up (tables and H_ii)
done first.

Checked through the C ABI: two calls in a row give the same sigma as the
regular device-vector entry point (within 1e-12 of max|sigma|, the bar of the
other sigma tests); a call that is the context's very first sigma, right after
the set-up, leaves the device's free memory unchanged (the array and the
kernels were loaded when the context was created, not inside the call); a
call before the set-up is refused, and a basis above the limit is refused
before anything runs.  This file is collected last so a failure here leaves
every other test already run.
"""
import ctypes

import numpy as np
import pytest

import sbd_b200
from sbd_b200 import synth

pytestmark = pytest.mark.gpu

SBDGPU_ERR_LIMIT = 4
SBDGPU_ERR_STATE = 5


def _noalloc(ctx, dC, dS) -> int:
    lib = sbd_b200.lib()
    return lib.sbdgpu_sigma_device_noalloc(ctx._h, ctypes.c_void_p(dC), ctypes.c_void_p(dS))


def _unit_vector(n, seed, dev):
    import torch
    g = torch.Generator(device=dev).manual_seed(seed)
    C = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
    return C / torch.linalg.norm(C)


def test_noalloc_first_sigma_after_setup_allocates_nothing():
    import torch

    ints, ne, strs = synth.make_small(10, 3, 100, 21)  # 100 x 100 selected strings
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=0)
    ctx.tables(0)
    ctx.hii()
    dev = torch.device("cuda:0")
    C = _unit_vector(ctx.n, 5, dev)
    out = torch.full_like(C, float("nan"))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    assert _noalloc(ctx, C.data_ptr(), out.data_ptr()) == 0  # the context's first sigma
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    # a module load or a scratch allocation inside the call would take at
    # least one 2 MiB page (the scratch array alone is 12 MiB)
    assert free0 - free1 < (2 << 20), (free0, free1)
    ref = torch.empty_like(C)
    ctx.sigma_device(C.data_ptr(), ref.data_ptr())
    out2 = torch.full_like(C, float("nan"))
    assert _noalloc(ctx, C.data_ptr(), out2.data_ptr()) == 0
    torch.cuda.synchronize()
    r = ref.cpu().numpy()
    for o in (out.cpu().numpy(), out2.cpu().numpy()):
        assert np.all(np.isfinite(o))
        assert np.abs(o - r).max() <= 1e-12 * np.abs(r).max()


def test_noalloc_sigma_matches_regular_entry_point_twice():
    import torch

    ints, ne, strs = synth.make_small(12, 4, None, 0)  # 495 x 495 = 245,025 determinants
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=0)
    dev = torch.device("cuda:0")
    C = torch.zeros(ctx.n, dtype=torch.float64, device=dev)
    S = torch.zeros_like(C)
    # before the set-up the entry point refuses instead of allocating
    assert _noalloc(ctx, C.data_ptr(), S.data_ptr()) == SBDGPU_ERR_STATE
    assert b"set-up" in sbd_b200.lib().sbdgpu_last_error(ctx._h)
    ctx.tables(0)
    ctx.hii()
    for seed in (11, 12):
        C = _unit_vector(ctx.n, seed, dev)
        ref = torch.empty_like(C)
        ctx.sigma_device(C.data_ptr(), ref.data_ptr())
        out = torch.full_like(C, float("nan"))
        assert _noalloc(ctx, C.data_ptr(), out.data_ptr()) == 0
        torch.cuda.synchronize()
        r, o = ref.cpu().numpy(), out.cpu().numpy()
        assert np.all(np.isfinite(o))
        assert np.abs(o - r).max() <= 1e-12 * np.abs(r).max()


def test_noalloc_sigma_rejects_bases_above_its_limit():
    import torch

    ints, ne, strs = synth.make_small(14, 5, 800, 3)  # 800 x 800 = 640,000 determinants
    ctx = sbd_b200.context_from_integrals(ints, strs, strs, device=0)
    ctx.tables(0)
    ctx.hii()
    C = torch.zeros(ctx.n, dtype=torch.float64, device="cuda:0")
    S = torch.zeros_like(C)
    assert _noalloc(ctx, C.data_ptr(), S.data_ptr()) == SBDGPU_ERR_LIMIT
    assert b"524288" in sbd_b200.lib().sbdgpu_last_error(ctx._h)
