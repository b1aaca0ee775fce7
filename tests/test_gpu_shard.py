"""The per-rank block sigma of the alpha-row sharding on the GPU
(sbdgpu_sigma_rows_device): rows of the full sigma for uneven blocks (odd
first rows included), and the sharded Davidson driver on a one-rank NCCL
group against the single-GPU Davidson."""
import datetime
import socket

import numpy as np
import pytest

import sbd_b200
from sbd_b200 import synth
from sbd_b200.shard import mpi_range

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("norb,ne,count,seed,nblocks", [(12, 4, None, 0, 3), (16, 5, 401, 12, 4), (20, 3, 600, 13, 7)])
def test_row_blocks_equal_full_sigma(norb, ne, count, seed, nblocks):
    import torch
    ints, ne, strs = synth.make_small(norb, ne, count, seed)
    ctx = sbd_b200.context_from_integrals(ints, strs, strs)
    dev = torch.device("cuda:0")
    g = torch.Generator(device=dev).manual_seed(seed)
    C = torch.randn(ctx.n, dtype=torch.float64, device=dev, generator=g)
    C /= torch.linalg.norm(C)
    full = torch.empty_like(C)
    ctx.sigma_device(C.data_ptr(), full.data_ptr())
    blocks = [mpi_range(nblocks, k, 0, ctx.na) for k in range(nblocks)] + [(1, 4), (ctx.na - 1, ctx.na), (5, 5)]
    ref = full.cpu().numpy()
    scale = np.abs(ref).max()
    for r0, r1 in blocks:
        out = torch.full((max(r1 - r0, 1) * ctx.nb,), float("nan"), dtype=torch.float64, device=dev)
        ctx.sigma_rows_device(C.data_ptr(), out.data_ptr(), r0, r1)
        got = out.cpu().numpy()[:(r1 - r0) * ctx.nb]
        assert np.abs(got - ref[r0 * ctx.nb:r1 * ctx.nb]).max(initial=0.0) <= 1e-12 * scale, (r0, r1)
    with pytest.raises(sbd_b200.SbdGpuError):
        ctx.sigma_rows_device(C.data_ptr(), full.data_ptr(), 3, ctx.na + 1)


def test_sharded_davidson_one_rank_nccl():
    import torch
    import torch.distributed as dist
    from sbd_b200.shard import AlphaRowShards, davidson, gpu_block_sigma
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ints, ne, strs = synth.make_small(12, 4, None, 0)
        ctx = sbd_b200.context_from_integrals(ints, strs, strs)
        sh = AlphaRowShards(ctx.na, ctx.nb)
        W0 = np.zeros(ctx.n)
        W0[0] = 1.0
        e_ref, _, te, _ = ctx.davidson(W0, 200, 10, 1e-8)
        dev = torch.device("cuda:0")
        hii = torch.from_numpy(sh.local(ctx.hii()).copy()).to(dev)
        w = torch.from_numpy(sh.local(W0).copy()).to(dev)
        e, W, trace = davidson(sh, gpu_block_sigma(ctx), hii, w, 200, 10, 1e-8)
        assert abs(e - e_ref) < 1e-10
        assert trace[-1][1] < 1e-8
    finally:
        dist.destroy_process_group()
