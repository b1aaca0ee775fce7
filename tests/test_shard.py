"""Alpha-row sharding on CPU with gloo ranks (sbd_b200/shard.py): the block
ranges follow the reference's get_mpi_range; with two and three ranks the
gathered rows' sigma equals the single-process sigma exactly; and the
sharded Davidson reaches the single-process energy.  Each rank's block sigma
here is the C restatement of the reference's mult restricted to its rows (on
GPUs it is sbdgpu_sigma_rows_device); the ranges, the all-gather, the
distributed inner products and the Davidson driver are the product code."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_ranges_follow_get_mpi_range():
    sys.path.insert(0, ROOT)
    from sbd_b200.shard import mpi_range
    # framework/mpi_utility.h:14-36: the first n % size ranks take one more
    assert [mpi_range(3, r, 0, 10) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert [mpi_range(4, r, 5, 13) for r in range(4)] == [(5, 7), (7, 9), (9, 11), (11, 13)]
    for n in (1, 7, 495, 4000):
        for size in (1, 2, 3, 8):
            if size > n:
                continue
            rs = [mpi_range(size, r, 0, n) for r in range(size)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(e - b for b, e in rs) - min(e - b for b, e in rs) <= 1


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import oracle
    from sbd_b200 import synth
    from sbd_b200.shard import AlphaRowShards, davidson
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ints, ne, strs = synth.make_small(8, 3, None, 4)  # 56 x 56 = 3,136 determinants
        orc = oracle.Oracle(8, strs, strs, ints.ecore, ints.h, ints.eri)
        na = nb = len(strs)
        sh = AlphaRowShards(na, nb, adet_comm_size=world)

        def block_sigma(full, r0, r1):
            return torch.from_numpy(orc.sigma(full.numpy(), (r0, r1)))

        C = np.random.default_rng(9).normal(size=na * nb)
        C /= np.linalg.norm(C)
        full_ref = orc.sigma(C)
        local = sh.sigma(torch.from_numpy(sh.local(C).copy()), block_sigma).numpy()
        exact = bool(np.array_equal(local, sh.local(full_ref)))
        gathered = sh.gather(torch.from_numpy(local)).numpy()
        W0 = np.zeros(na * nb)
        W0[0] = 1.0
        hii = torch.from_numpy(sh.local(orc.hii()).copy())
        e, W, trace = davidson(sh, block_sigma, hii, torch.from_numpy(sh.local(W0).copy()), 100, 10, 1e-8)
        out.put((rank, exact, bool(np.array_equal(gathered, full_ref)), e, len(trace), sh.r0, sh.r1))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_sigma_and_davidson_gloo(world):
    sys.path.insert(0, ROOT)
    import oracle
    from sbd_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = {}
    for _ in ps:
        r = q.get(timeout=300)
        res[r[0]] = r[1:]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    ints, ne, strs = synth.make_small(8, 3, None, 4)
    orc = oracle.Oracle(8, strs, strs, ints.ecore, ints.h, ints.eri)
    W0 = np.zeros(len(strs) ** 2)
    W0[0] = 1.0
    e_ref, _, te, _ = orc.davidson(W0, 100, 10, 1e-8)
    rows = sorted((v[4], v[5]) for v in res.values())
    assert rows[0][0] == 0 and rows[-1][1] == len(strs)
    for rank, (exact, gathered_ok, e, nsteps, r0, r1) in res.items():
        assert exact and gathered_ok
        assert abs(e - e_ref) < 1e-10, (e, e_ref)
        assert abs(nsteps - len(te)) <= 2
