"""Multi-process slab runs on the device: a cavity split over the ranks of a
torch.distributed group (RankSlab, one slab per process) gives bitwise the
state of the single-process slab group.  The two ranks run as two processes
on one GPU over gloo: their kernels never wait on each other (the host
exchanges the combine words and the ghost rows between launches), so sharing
the device changes nothing but the timing."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, name, kw, precision, steps, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        from alebgk4paper_b200 import Case
        from alebgk4paper_b200.slab import RankSlab
        rs = RankSlab(Case(name, **kw), precision=precision, device=0)
        rs.step(steps)
        g, m, rows = rs.owned()
        out[rank] = (g, m, rows)
        rs.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,kw,precision", [
    ("cavity2d", dict(Nx=32, Nv=16, lid_speed=5.0), 64),
    ("cavity3d", dict(Nx=24, Nv=8, lid_speed=10.0), 32),
])
def test_rank_slabs_equal_the_slab_group(gpu, name, kw, precision):
    from alebgk4paper_b200 import Case
    from alebgk4paper_b200.slab import SlabGroup
    steps, world = 6, 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as man:
        out = man.dict()
        procs = [ctx.Process(target=_worker,
                             args=(r, world, port, name, kw, precision, steps, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
        # a worker stuck in a collective would otherwise outlive the test
        for p in procs:
            if p.is_alive():
                p.terminate()
                p.join(30)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    group = SlabGroup(Case(name, **kw), world, precision=precision)
    group.step(steps)
    g, m = group.download_full()
    group.close()
    for rank in range(world):
        gr, mr, (a, b) = res[rank]
        np.testing.assert_array_equal(gr, g[a:b])
        np.testing.assert_array_equal(mr[:, :6], m[a:b, :6])
