"""Slab mode, host side: the slab plan (owned rows, halo, ghost copies) and
the renumbered neighbour lists of each slab."""
import numpy as np
import pytest

from alebgk4paper_b200 import Case
from alebgk4paper_b200.slab import _SlabCase, plan_slabs


@pytest.mark.parametrize("n", [2, 3, 5])
def test_plan_covers_every_row_once(n):
    c = Case("cavity3d", Nx=40, Nv=4)
    plan = plan_slabs(c, n)
    assert plan["rows"] == 40 and plan["stride"] == 1600 and plan["halo"] == 4
    owned = np.concatenate([np.arange(s["r0"], s["r1"]) for s in plan["slabs"]])
    assert np.array_equal(owned, np.arange(40))
    st = plan["stride"]
    for s in plan["slabs"]:
        assert s["r1"] - s["r0"] >= 8
        lo, hi = s["own"]
        assert (hi - lo) == (s["r1"] - s["r0"]) * st
    # every ghost block is a copy of owned rows of the same global rows
    for dst, dstart, src, sstart, cnt in plan["copies"]:
        d, s = plan["slabs"][dst], plan["slabs"][src]
        g_dst = d["k0"] * st + dstart
        g_src = s["k0"] * st + sstart
        assert g_dst == g_src and cnt == 4 * st
        assert s["own"][0] <= sstart and sstart + cnt <= s["own"][1]
    assert len(plan["copies"]) == 2 * (n - 1)


def test_plan_rejects_thin_slabs_and_bodies():
    with pytest.raises(ValueError, match="two halos"):
        plan_slabs(Case("cavity3d", Nx=12, Nv=4), 2)
    with pytest.raises(ValueError, match="without bodies"):
        plan_slabs(Case("cavity2d-square", Nx=24, Nv=4), 2)


@pytest.mark.parametrize("name,Nx,n", [("cavity2d", 24, 2), ("cavity3d", 20, 2),
                                       ("cavity2d", 33, 3)])
def test_owned_particles_keep_their_whole_stencil(name, Nx, n):
    c = Case(name, Nx=Nx, Nv=4)
    plan = plan_slabs(c, n)
    st = plan["stride"]
    for sl in plan["slabs"]:
        sc = _SlabCase(c, sl["k0"], sl["k1"], st)
        base = sl["k0"] * st
        lo, hi = sl["own"]
        for i in range(lo, hi):
            gi = base + i
            assert sc.nnb[i] == c.nnb[gi]
            assert np.array_equal(sc.nbr[i, :sc.nnb[i]] + base, c.nbr[gi, :c.nnb[gi]])
        assert np.array_equal(sc.xyz, c.xyz[base:base + sc.N])


@pytest.mark.parametrize("name,kw,n", [("cavity2d", dict(Nx=33, Nv=4), 3),
                                       ("cavity3d", dict(Nx=24, Nv=4), 2),
                                       ("cavity2d", dict(Nx=48, Nv=4), 4)])
def test_rank_halo_plan_pairs_every_send_with_a_receive(name, kw, n):
    """Per rank, the ghost copies split into sends (own rows to a neighbour)
    and receives (ghost rows from a neighbour); over all ranks every copy is
    one send and one receive of the same size, sends read owned rows and
    receives write ghost rows only."""
    from alebgk4paper_b200.slab import rank_halo_plan
    case = Case(name, **kw)
    plan = plan_slabs(case, n)
    sends, recvs = {}, {}
    for r in range(n):
        s, v = rank_halo_plan(plan, r)
        lo, hi = plan["slabs"][r]["own"]
        for peer, start, count in s:
            assert lo <= start and start + count <= hi
            sends.setdefault((r, peer), []).append(count)
        for peer, start, count in v:
            assert start + count <= lo or start >= hi
            recvs.setdefault((peer, r), []).append(count)
        # neighbours only
        assert all(abs(peer - r) == 1 for peer, _, _ in s + v)
    assert sends == recvs
    assert sum(len(x) for x in sends.values()) == len(plan["copies"]) == 2 * (n - 1)
