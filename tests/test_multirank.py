"""The N > 1 bookkeeping of bench.py on CPU: two gloo ranks (the GPU path runs
independent replicas, so its only cross-rank steps are the barrier and the
max-over-ranks timing), and the reference arm's rule that ranks other than 0
exit without work."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    assert bench.dist_env() == (rank, world, rank)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    dist.barrier()
    # rank r measured (10 + r, 100 - r) ms: the job takes the slowest of each
    got = bench.max_over_ranks([10.0 + rank, 100.0 - rank], dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, got))


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == [11.0, 100.0] and res[1] == [11.0, 100.0]


def test_reference_arm_nonzero_rank_exits_without_work(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class Args:
        workload = "c2_L36_8e_12000"
        steps = 1
        warmup = 0
        ref_budget = 1.0
    assert bench.run_reference(Args()) == 0


def test_reference_arm_json_contract():
    """bench.py --impl reference on rank 0 (CPU only): one JSON line with the
    contract's keys, timing the compiled reference's own mult."""
    import json
    import subprocess
    import oracle
    if not oracle.reference_available():
        pytest.skip("compiled reference not available")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--workload", "c1_L26_6e_4000", "--ref-budget", "5"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600,
                       env={**os.environ, "RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    for k in ("metric", "unit", "config", "cpu_baseline", "e2e", "steps", "warmup"):
        assert k in line
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0
