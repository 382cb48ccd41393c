"""The z-slab exchange plan (lbman_halo_plan, host only) and its delivery by
torch.distributed point-to-point operations on gloo CPU ranks.

The slabs are emulated with host arrays shaped like a slab's device arrays
(owned planes plus two ghost planes per side), filled with codes of the
global plane, field and component, in the manner of the reference's pack /
unpack checks (tests/mpi/test_halo_exchange_qtensor.cc,
tests/mpi/test_halo_exchange_lbm.cc): after an exchange every ghost plane
must hold exactly the neighbour's owned plane it stands for, for the fields
and population slots the plan names, and nothing else may change.  The
device side (spans resolved to buffers, the merge of the F_OUT arrivals and
the bitwise equality of a split box with the whole box) is covered by
tests/test_gpu_slab.py.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from lbman3d_b200 import _native as N  # noqa: E402
from lbman3d_b200 import slab as SL  # noqa: E402

EZ = [0, 0, 0, 0, 0, 1, -1, 1, 1, 1, 1, -1, -1, -1, -1]
UP = [k for k in range(15) if EZ[k] == 1]
DOWN = [k for k in range(15) if EZ[k] == -1]


def test_split_planes():
    assert SL.split_planes(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert SL.split_planes(4, 2) == [(0, 2), (2, 2)]
    with pytest.raises(ValueError):
        SL.split_planes(5, 3)


@pytest.mark.parametrize("nzl", [2, 3, 7])
def test_plan_shapes(nzl):
    send, recv = SL.halo_plan(nzl, N.HALO_QU)
    assert [len(a) for a in send + recv] == [8] * 4
    for f, (ps, pr) in enumerate(zip(send, recv)):
        assert [(s["field"], s["comp"]) for s in ps] == [(N.FIELD_Q, k) for k in range(5)] + [(N.FIELD_U, k) for k in range(3)]
        assert [(s["field"], s["comp"]) for s in pr] == [(s["field"], s["comp"]) for s in ps]
        assert all(s["planes"] == 2 for s in ps + pr)
        assert {s["plane"] for s in ps} == {0 if f == 0 else nzl - 2}
        assert {s["plane"] for s in pr} == {-2 if f == 0 else nzl}
    # before an odd in-place step: the slots pointing at the neighbour
    send, recv = SL.halo_plan(nzl, N.HALO_F_IN)
    assert [s["comp"] for s in send[0]] == UP and [s["comp"] for s in recv[1]] == UP
    assert [s["comp"] for s in send[1]] == DOWN and [s["comp"] for s in recv[0]] == DOWN
    assert {(s["plane"], s["planes"]) for s in send[0]} == {(0, 1)}
    assert {(s["plane"], s["planes"]) for s in send[1]} == {(nzl - 1, 1)}
    assert {s["plane"] for s in recv[0]} == {-1} and {s["plane"] for s in recv[1]} == {nzl}
    # after it: the ghost slots go back, into the neighbour's staging area
    send, recv = SL.halo_plan(nzl, N.HALO_F_OUT)
    assert [s["comp"] for s in send[0]] == DOWN and [s["comp"] for s in send[1]] == UP
    assert {s["plane"] for s in send[0]} == {-1} and {s["plane"] for s in send[1]} == {nzl}
    for f in range(2):
        assert [(s["field"], s["comp"], s["plane"]) for s in recv[f]] == [(N.FIELD_FSTAGE, k, f) for k in range(5)]


def test_plan_rejects_bad_arguments():
    M = N.HALO_MAX_SPANS
    import ctypes as C
    s, r, n = (N.lbman_halo_span * (2 * M))(), (N.lbman_halo_span * (2 * M))(), C.c_int()
    assert N.lib().lbman_halo_plan(1, N.HALO_QU, s, r, C.byref(n)) == N.ERR_ARG
    assert N.lib().lbman_halo_plan(4, 7, s, r, C.byref(n)) == N.ERR_ARG


# ---- delivery between ranks --------------------------------------------------

NX, NY = 4, 3


def code(field, comp, gz, nzg):
    """Value of every cell of plane gz (mod nzg) of a field component, plus the
    cell index so misplaced rows show up too."""
    return ((field * 16 + comp) * 1000 + gz % nzg) * 100 + np.arange(NX * NY, dtype=np.float64)


class HostSlab:
    """A slab's fields as host arrays with the device layout: [comp][plane][y][x]
    with planes -2 .. nzl+1 stored at 0 .. nzl+3; the F_OUT staging area
    [face][slot][y][x]."""

    def __init__(self, z0, nzl, nzg):
        self.z0, self.nzl, self.nzg = z0, nzl, nzg
        shape = lambda nc: (nc, nzl + 4, NX * NY)
        self.a = {N.FIELD_Q: np.full(shape(5), np.nan), N.FIELD_U: np.full(shape(3), np.nan),
                  N.FIELD_F: np.full(shape(15), np.nan), N.FIELD_FSTAGE: np.full((2, 5, NX * NY), np.nan)}
        for fld, nc in ((N.FIELD_Q, 5), (N.FIELD_U, 3), (N.FIELD_F, 15)):
            for c in range(nc):
                for p in range(nzl):
                    self.a[fld][c, p + 2] = code(fld, c, z0 + p, nzg)

    def view(self, s):
        if s["field"] == N.FIELD_FSTAGE:
            return self.a[N.FIELD_FSTAGE][s["plane"], s["comp"]]
        return self.a[s["field"]][s["comp"], s["plane"] + 2:s["plane"] + 2 + s["planes"]]


def _rank(rank, world, port, nzg, out):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        z0, nzl = SL.split_planes(nzg, world)[rank]
        hs = HostSlab(z0, nzl, nzg)
        tt = lambda s: torch.from_numpy(hs.view(s)).view(-1)
        for phase in (N.HALO_QU, N.HALO_F_IN):
            send, recv = SL.halo_plan(nzl, phase)
            SL.p2p_exchange(send, recv, tt, rank, world, dist)
        f_in = hs.a[N.FIELD_F].copy()
        # what an odd step would have scattered into the ghost planes
        for k in DOWN:
            hs.a[N.FIELD_F][k, 1] = code(7, k, z0 - 1, nzg) + 0.5
        for k in UP:
            hs.a[N.FIELD_F][k, nzl + 2] = code(7, k, z0 + nzl, nzg) + 0.5
        send, recv = SL.halo_plan(nzl, N.HALO_F_OUT)
        SL.p2p_exchange(send, recv, tt, rank, world, dist)
        res = {k: v.copy() for k, v in hs.a.items()}
        out.put((rank, z0, nzl, f_in, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
@pytest.mark.parametrize("world,nzg", [(2, 9), (3, 10)])
def test_exchange_between_ranks_fills_exactly_the_planned_ghosts(world, nzg):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, nzg, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = [out.get(timeout=200) for _ in range(world)]
    for p in procs:
        p.join(60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    for rank, z0, nzl, f_in, a in got:
        # owned planes untouched
        for fld, nc in ((N.FIELD_Q, 5), (N.FIELD_U, 3)):
            for c in range(nc):
                for p in range(nzl):
                    np.testing.assert_array_equal(a[fld][c, p + 2], code(fld, c, z0 + p, nzg))
                # Q and u: two ghost planes per side, the neighbours' owned planes
                for g in (-2, -1, nzl, nzl + 1):
                    np.testing.assert_array_equal(a[fld][c, g + 2], code(fld, c, z0 + g, nzg))
        F = a[N.FIELD_F]
        for k in range(15):
            for p in range(nzl):
                np.testing.assert_array_equal(F[k, p + 2], code(N.FIELD_F, k, z0 + p, nzg))
            # F_IN: the slots a boundary cell gathers from, in one ghost plane
            # per side, hold the neighbour's boundary plane; the other slots
            # and the second ghost planes are untouched
            if k in DOWN:
                np.testing.assert_array_equal(f_in[k, 1], code(N.FIELD_F, k, z0 - 1, nzg))
            else:
                assert np.isnan(f_in[k, 1]).all()
            if k in UP:
                np.testing.assert_array_equal(f_in[k, nzl + 2], code(N.FIELD_F, k, z0 + nzl, nzg))
            else:
                assert np.isnan(f_in[k, nzl + 2]).all()
            assert np.isnan(f_in[k, 0]).all() and np.isnan(f_in[k, nzl + 3]).all()
        # F_OUT: the neighbours' ghost slots land in the staging area: face 0
        # holds what the lower slab scattered upward into its plane above it
        # (this slab's plane 0), face 1 what the upper slab scattered downward
        S = a[N.FIELD_FSTAGE]
        for i, k in enumerate(UP):
            np.testing.assert_array_equal(S[0, i], code(7, k, z0, nzg) + 0.5)
        for i, k in enumerate(DOWN):
            np.testing.assert_array_equal(S[1, i], code(7, k, z0 + nzl - 1, nzg) + 0.5)


# ---- the ensemble across ranks (no exchange) --------------------------------


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_boxes_is_a_cell_balanced_partition(world):
    import lbman3d_b200 as L
    boxes = L.draw_boxes(96, seed=2024)
    shares = L.shard_boxes(boxes, world)
    ids = sorted(i for s in shares for i in s)
    assert ids == list(range(96))
    assert all(s == sorted(s) for s in shares)
    loads = [sum(boxes[i][0].V for i in s) for s in shares]
    assert max(loads) - min(loads) <= max(p.V for p, _ in boxes)
    assert shares == L.shard_boxes(boxes, world)  # deterministic
