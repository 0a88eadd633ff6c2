"""The multi-GPU path of bench.py on CPU: world size 2 over gloo.  Every rank
advances its own cavity (no data-path collective); the step time is the max
over ranks and the value counts every rank's updates."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(times[rank], dist, "cpu")
        out[rank] = (t, bench.weak_value(world, 1000, 10, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_weak_value_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    port = _free_port()
    times = [0.25, 0.5]
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, times, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(2):
        t, v = res[r]
        assert t == 0.5                       # the slowest rank sets the time
        assert v == pytest.approx(2 * 1000 * 10 / 0.5)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(0.3, None, "cpu") == 0.3
    assert bench.weak_value(1, 64000 * 1000, 20, 0.02) == pytest.approx(6.4e10)


def test_reference_arm_on_a_non_zero_rank_does_no_work():
    """Under torchrun only rank 0 times the reference; the other ranks exit 0
    at once without printing."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
