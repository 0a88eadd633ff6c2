"""Host side of multi-process slab runs (RankSlab) on CPU: two ranks over
gloo, with a stand-in for the device library that records what the driver
hands it.  Checked: the combine words reach every rank all-gathered in rank
order for phases 4 (set-up), 0, 1, 2, 3 of every step; the ghost rows of the
state being written are the neighbour's owned rows (by global row); the step
ends with finish.  The device side of the same calls is the slab group's
(tests/test_gpu_slab.py)."""
import ctypes
import datetime
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT

ROW_BYTES = 16      # stand-in row: 4 float32 values


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _FakeSolver:
    def __init__(self, sub):
        self.ctx = ctypes.c_void_p(1)
        self.sub = sub

    def close(self):
        pass


class _FakeLib:
    """Slab state: rows of the state being written, as global-row tags."""

    def __init__(self, rank, base, n):
        self.rank, self.base, self.n = rank, base, n
        self.next_f = np.full((n, ROW_BYTES), 255, np.uint8)   # ghost rows start as junk
        self.next_m = np.full((n, 6), -1.0)
        self.own = None
        self.step = 0
        self.log = []

    def alebgk_device_state(self, ctx, f, ldf, es):
        ldf._obj.value = ROW_BYTES // 4
        es._obj.value = 4
        return 0

    def _words(self, q):
        return [100.0 * (self.rank + 1) + q, 10.0 * self.step + q, float(self.rank), 0.0]

    def _put_words(self, ptr, w):
        a = np.ctypeslib.as_array(ptr, shape=(4,))
        a[:] = w

    def alebgk_rank_slab_init(self, ctx, nranks, lo, hi, words):
        self.own = (lo, hi)
        self._put_words(words, self._words(9))
        self.log.append(("init", nranks))
        return 0

    def alebgk_rank_slab_segment(self, ctx, seg, words):
        if seg == 0:
            # the step writes the owned rows: tag = global row, step
            lo, hi = self.own
            for i in range(lo, hi):
                self.next_f[i] = (self.base + i + 7 * self.step) % 251
                self.next_m[i] = self.base + i + 1000.0 * self.step
        self._put_words(words, self._words(seg))
        self.log.append(("segment", seg))
        return 0

    def alebgk_rank_slab_combine(self, ctx, phase, nranks, allw):
        self.log.append(("combine", phase, np.ctypeslib.as_array(allw, shape=(4 * nranks,)).copy()))
        return 0

    def alebgk_rank_slab_rows(self, ctx, start, count, f, m, put):
        fb = np.ctypeslib.as_array(ctypes.cast(f, ctypes.POINTER(ctypes.c_uint8)),
                                   shape=(count * ROW_BYTES,))
        mb = np.ctypeslib.as_array(m, shape=(count * 6,))
        if put:
            self.next_f[start:start + count] = fb.reshape(count, ROW_BYTES)
            self.next_m[start:start + count] = mb.reshape(count, 6)
        else:
            fb[:] = self.next_f[start:start + count].ravel()
            mb[:] = self.next_m[start:start + count].ravel()
        self.log.append(("rows", start, count, put))
        return 0

    def alebgk_rank_slab_finish(self, ctx):
        self.log.append(("finish",))
        self.checked = (self.next_f.copy(), self.next_m.copy())
        self.step += 1
        return 0


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import alebgk4paper_b200 as ab
        from alebgk4paper_b200.slab import RankSlab, plan_slabs
        case = ab.Case("cavity2d", 24, 4)
        plan = plan_slabs(case, world)
        sl = plan["slabs"][rank]
        base = sl["k0"] * plan["stride"]
        n = (sl["k1"] - sl["k0"]) * plan["stride"]
        lib = _FakeLib(rank, base, n)
        rs = RankSlab(case, lib=lib, solver_factory=_FakeSolver)
        rs.step(2)
        out[rank] = dict(log=lib.log, f=lib.checked[0], m=lib.checked[1], base=base, n=n,
                         own=lib.own, plan=plan)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_rank_slab_exchanges_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as man:
        out = man.dict()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        # a worker stuck in a collective would otherwise outlive the test
        for p in procs:
            if p.is_alive():
                p.terminate()
                p.join(30)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    for rank in (0, 1):
        r = res[rank]
        log = r["log"]
        assert log[0] == ("init", 2)
        combines = [e for e in log if e[0] == "combine"]
        # set-up, then phases 0..3 per step
        assert [c[1] for c in combines] == [4, 0, 1, 2, 3, 0, 1, 2, 3]
        # words all-gathered in rank order: rank i's first word is 100 (i + 1) + q
        q_of = {4: 9, 0: 0, 1: 1, 2: 2, 3: 3}
        for _, phase, allw in combines:
            for i in (0, 1):
                assert allw[4 * i] == 100.0 * (i + 1) + q_of[phase]
                assert allw[4 * i + 2] == float(i)
        # every step: 4 segments, then the rows, then finish
        kinds = [e[0] for e in log[1:]]
        assert kinds.count("finish") == 2 and kinds[-1] == "finish"
        # after the last step every row (owned and ghost) holds its global tag
        base, n = r["base"], r["n"]
        step = 1
        for i in range(n):
            assert (r["f"][i] == (base + i + 7 * step) % 251).all(), (rank, i)
            assert (r["m"][i] == base + i + 1000.0 * step).all(), (rank, i)


class _RecordingDist:
    """Stands in for torch.distributed under an NCCL group: records how the
    ghost-row exchange posts its point-to-point operations."""

    class P2POp:
        def __init__(self, op, tensor, peer, group=None):
            self.op, self.tensor, self.peer, self.group = op, tensor, peer, group

    class _Work:
        def wait(self):
            return True

    def __init__(self):
        self.batches, self.direct = [], 0

    def get_backend(self, group=None):
        return "nccl"

    def irecv(self, *a, **k):
        self.direct += 1
        return self._Work()

    def isend(self, *a, **k):
        self.direct += 1
        return self._Work()

    def batch_isend_irecv(self, ops):
        self.batches.append([(o.op.__name__, o.peer) for o in ops])
        return [self._Work() for _ in ops]


def test_nccl_ghost_exchange_is_one_batched_call():
    """Under NCCL every receive and send of a step's ghost-row exchange goes
    through a single batch_isend_irecv call (grouped point-to-point), never
    as separately queued isend/irecv, which can deadlock two ranks that
    exchange with each other."""
    import torch
    from alebgk4paper_b200.slab import RankSlab
    rs = RankSlab.__new__(RankSlab)
    rs.dist = _RecordingDist()
    rs.group = None
    rs.ctx = ctypes.c_void_p(1)
    rs.row_bytes = ROW_BYTES
    rs.device = 0
    rs.recvs = [(0, 10, 3), (2, 40, 3)]
    rs.sends = [(0, 13, 3), (2, 37, 3)]
    lib = _FakeLib(1, 0, 50)
    lib.own = (13, 40)
    rs.lib = lib
    rs._tensor = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    rs._halo()
    assert rs.dist.direct == 0
    assert len(rs.dist.batches) == 1
    ops = rs.dist.batches[0]
    assert sorted(ops) == sorted([("irecv", 0)] * 2 + [("irecv", 2)] * 2 +
                                 [("isend", 0)] * 2 + [("isend", 2)] * 2)
