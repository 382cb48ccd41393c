"""A box split into z-slabs (lbman_create_slab + the lbman_halo_* exchange)
against the same box in one handle, on one GPU.

The slabs run the same kernels over their owned planes, with every value
beyond them delivered by the exchange, so a split box must reproduce the
whole box bit for bit: in FP64 (the reference's arithmetic) and in FP32 with
both Q+force kernels, after odd and even step counts (the in-place LBM
exchanges populations around odd steps only), on every z-periodic boundary
configuration -- x / y walls of every velocity type, anchoring, a moving
wall -- with even and uneven splits, and one slab whose periodic z faces
meet in itself.  This is the single-GPU form of the multi-GPU check: the
slabs are separate handles that share nothing but the exchanged spans.
"""
import ctypes as C

import numpy as np
import pytest

import lbman3d_b200 as L
from lbman3d_b200 import _native as N
from lbman3d_b200 import slab as SL

pytestmark = pytest.mark.gpu


def _state(grid, seed=5):
    nx, ny, nz = grid
    V = nx * ny * nz
    rng = np.random.default_rng(seed)
    rho = 1.0 + 0.01 * rng.standard_normal(V)
    u = 0.01 * rng.standard_normal(3 * V)
    q = 0.05 * rng.standard_normal(5 * V)
    return rho, u, q


def _params(grid, upwind, **phys):
    nx, ny, nz = grid
    adv = L.Advection.Upwind if upwind else L.Advection.Centred
    return L.Params(nx=nx, ny=ny, nz=nz, kQAdvection=adv, **phys)


# (name, grid, bc, upwind, slab planes)
CASES = [
    ("periodic_2", (24, 20, 16), "periodic", False, [(0, 8), (8, 8)]),
    ("slit_3_uneven", (20, 18, 15), "slit", True, [(0, 4), (4, 6), (10, 5)]),
    ("channel_2", (16, 14, 12), "channel", False, [(0, 5), (5, 7)]),
    ("lid_4", (12, 16, 10), "lid", True, [(0, 2), (2, 3), (5, 2), (7, 3)]),
    ("poiseuille_1", (8, 12, 9), "poiseuille", False, [(0, 9)]),
]


def _compare(a, b, exact, tol=0.0):
    for k in ("rho", "u", "q", "f"):
        if exact:
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        else:
            d = np.max(np.abs(a[k] - b[k])) / np.max(np.abs(b[k]))
            assert d <= tol, (k, d)


@pytest.mark.parametrize("name,grid,bc,upwind,planes", CASES, ids=[c[0] for c in CASES])
def test_fp64_slabs_equal_the_whole_box_bitwise(name, grid, bc, upwind, planes):
    from cases import BC
    p = _params(grid, upwind, ALPHA=0.02, MU=0.005)
    faces = L.from_face_tuples(BC[bc])
    rho, u, q = _state(grid)
    box = L.Simulation(p, faces, L.Precision.FP64, N.KERNELS_SPLIT)
    box.upload(rho, u, q)
    with SL.SlabBox(p, faces, L.Precision.FP64, kernels=N.KERNELS_SPLIT, planes=planes) as sb:
        sb.upload(rho, u, q)
        for n in (1, 2, 4):  # 1, 3, 7 steps: after odd and even in-place steps
            box.step(n)
            sb.step(n)
            _compare(sb.download(f=True), box.download(f=True), exact=True)
        # diagnostics: per-slab sums combined
        d0 = box.reduce(N.DIAG_FLOW | N.DIAG_ENERGY)
        d1 = sb.reduce(N.DIAG_FLOW | N.DIAG_ENERGY)
        for k in ("mass", "px", "py", "pz", "kinetic_energy", "free_energy"):
            assert d1[k] == pytest.approx(d0[k], rel=1e-12, abs=1e-14), k
        assert d1["umax2"] == d0["umax2"]
    box.close()


@pytest.mark.parametrize("kernels,tile", [(N.KERNELS_SPLIT, (32, 8, 0)), (N.KERNELS_SPLIT_PAIR, (30, 10, 3))],
                         ids=["one_point", "pair"])
@pytest.mark.parametrize("bc", ["periodic", "slit"])
def test_fp32_slabs_equal_the_whole_box(kernels, tile, bc):
    from cases import BC
    grid = (32, 20, 14)
    p = _params(grid, bc == "slit", ALPHA=0.02)
    faces = L.from_face_tuples(BC[bc])
    rho, u, q = _state(grid, 9)
    box = L.Simulation(p, faces, L.Precision.FP32, kernels, tile=tile)
    box.upload(rho, u, q)
    with SL.SlabBox(p, faces, L.Precision.FP32, kernels=kernels, tile=tile, planes=[(0, 6), (6, 8)]) as sb:
        sb.upload(rho, u, q)
        for n in (3, 4):
            box.step(n)
            sb.step(n)
            _compare(sb.download(f=True), box.download(f=True), exact=True)
    box.close()


@pytest.mark.parametrize("grid", [(32, 20, 14), (21, 12, 14)], ids=["two_cells", "one_cell"])
def test_fp16_slabs_equal_the_whole_box(grid):
    """FP16 population storage on a periodic box: slabs (in-place kernels
    restricted to the owned planes, population halos in FP16) equal the
    whole box bit for bit, with the two-cells-per-thread kernels (nx even)
    and the one-cell kernels."""
    from cases import BC
    p = _params(grid, False, ALPHA=0.02)
    faces = L.from_face_tuples(BC["periodic"])
    rho, u, q = _state(grid, 11)
    box = L.Simulation(p, faces, L.Precision.FP16, N.KERNELS_SPLIT)
    box.upload(rho, u, q)
    with SL.SlabBox(p, faces, L.Precision.FP16, kernels=N.KERNELS_SPLIT, planes=[(0, 6), (6, 8)]) as sb:
        sb.upload(rho, u, q)
        for n in (3, 4):
            box.step(n)
            sb.step(n)
            _compare(sb.download(f=True), box.download(f=True), exact=True)
    box.close()


def test_seeded_slabs_hold_the_whole_box_field():
    grid = (16, 12, 11)
    p = _params(grid, False)
    faces = L.FullyPeriodicConfig()
    box = L.Simulation(p, faces, L.Precision.FP64, N.KERNELS_SPLIT)
    box.init_seeded(21, 0.5, 1e-3)
    with SL.SlabBox(p, faces, L.Precision.FP64, nslabs=3, kernels=N.KERNELS_SPLIT) as sb:
        sb.init_seeded(21, 0.5, 1e-3)
        _compare(sb.download(f=True), box.download(f=True), exact=True)
        box.step(5)
        sb.step(5)
        _compare(sb.download(f=True), box.download(f=True), exact=True)
    box.close()


def test_out_of_order_calls_are_refused():
    grid = (8, 8, 8)
    p = _params(grid, False)
    faces = L.FullyPeriodicConfig()
    rho, u, q = _state(grid)
    s = SL.Slab(p, faces, L.Precision.FP64, N.KERNELS_SPLIT, z_offset=0, nz_local=8)
    s.upload(rho, u, q)
    h = (C.c_void_p * 1)(s.handle.value)
    with pytest.raises(N.LbmanError) as e:
        s.qtensor_step()  # no Q/u halo yet
    assert e.value.status == N.ERR_STATE
    with pytest.raises(N.LbmanError) as e:
        s.step(1)
    assert e.value.status == N.ERR_STATE
    ex = lambda ph: N.check(N.lib().lbman_slab_exchange(h, 1, ph))
    ex(N.HALO_QU)
    s.qtensor_step()
    ex(N.HALO_F_IN)  # nothing to move before an even step
    s.lbm_step()
    ex(N.HALO_QU)
    s.qtensor_step()
    with pytest.raises(N.LbmanError) as e:
        s.lbm_step()  # odd step without its population halo
    assert e.value.status == N.ERR_STATE
    ex(N.HALO_F_IN)
    s.lbm_step()
    with pytest.raises(N.LbmanError) as e:
        s.download()  # the odd step's scattered populations not merged yet
    assert e.value.status == N.ERR_STATE
    ex(N.HALO_F_OUT)
    s.download()
    with pytest.raises(N.LbmanError):
        s.qtensor_setup()
    s.close()


def test_slab_configurations_refused():
    from cases import BC
    p = _params((8, 8, 8), False)
    with pytest.raises(N.LbmanError) as e:  # walls on z
        SL.Slab(p, L.from_face_tuples(BC["walls"]), L.Precision.FP64, N.KERNELS_SPLIT, 0, 4)
    assert e.value.status == N.ERR_UNSUPPORTED
    with pytest.raises(N.LbmanError) as e:
        SL.Slab(p, L.FullyPeriodicConfig(), L.Precision.FP64, N.KERNELS_FUSED, 0, 4)
    assert e.value.status == N.ERR_UNSUPPORTED
    with pytest.raises(N.LbmanError) as e:  # one plane is less than the Q halo
        SL.Slab(p, L.FullyPeriodicConfig(), L.Precision.FP64, N.KERNELS_SPLIT, 0, 1)
    assert e.value.status == N.ERR_ARG
    with pytest.raises(N.LbmanError) as e:  # outside the box
        SL.Slab(p, L.FullyPeriodicConfig(), L.Precision.FP64, N.KERNELS_SPLIT, 6, 4)
    assert e.value.status == N.ERR_ARG


class _LoopbackDist:
    """torch.distributed stand-in for ranks living in one process: each
    rank's batch of point-to-point operations is recorded, and flush() pairs
    the i-th send from rank a to rank b with the i-th receive that b posted
    from a (NCCL's matching rule) and copies on the device."""

    class P2POp:
        def __init__(self, op, tensor, peer, group=None):
            self.op, self.tensor, self.peer = op, tensor, peer

    def __init__(self):
        self.rank, self.posted = None, {}

    def isend(self, *a):  # identity markers, as in torch.distributed
        raise AssertionError("called through batch_isend_irecv only")

    def irecv(self, *a):
        raise AssertionError("called through batch_isend_irecv only")

    def batch_isend_irecv(self, ops):
        self.posted[self.rank] = list(ops)
        return []

    def flush(self):
        sends, recvs = {}, {}
        for r, ops in self.posted.items():
            for op in ops:
                if op.op == self.isend:
                    sends.setdefault((r, op.peer), []).append(op.tensor)
                else:
                    recvs.setdefault((op.peer, r), []).append(op.tensor)
        assert sends.keys() == recvs.keys()
        for key, ts in sends.items():
            assert len(ts) == len(recvs[key])
            for s, d in zip(ts, recvs[key]):
                assert s.numel() == d.numel()
                d.copy_(s)
        self.posted = {}


@pytest.mark.parametrize("planes", [[(0, 5), (5, 7)], [(0, 4), (4, 4), (8, 4)]], ids=["2_ranks", "3_ranks"])
def test_rank_transport_on_device_memory_equals_the_whole_box(planes):
    """p2p_exchange with device tensors over the spans' addresses (the
    DistributedSlab path, ranks emulated in one process): bitwise the box."""
    import torch
    from cases import BC
    grid = (16, 12, 12)
    p = _params(grid, False, ALPHA=0.02)
    faces = L.from_face_tuples(BC["channel"])
    rho, u, q = _state(grid, 3)
    box = L.Simulation(p, faces, L.Precision.FP64, N.KERNELS_SPLIT)
    box.upload(rho, u, q)
    dev = torch.cuda.current_device()
    cur = torch.cuda.current_stream().cuda_stream
    slabs = [SL.Slab(p, faces, L.Precision.FP64, N.KERNELS_SPLIT, z0, n, dev) for z0, n in planes]
    world = len(slabs)
    nxy = grid[0] * grid[1]
    parts = [SL._split_field(a, nc, nxy, planes) for a, nc in ((rho, 1), (u, 3), (q, 5))]
    for s, r, uu, qq in zip(slabs, *parts):
        s.set_stream(cur)  # the exchange's copies run on torch's current stream
        s.upload(r, uu, qq)

    def exchange(phase):
        fake = _LoopbackDist()
        for r, s in enumerate(slabs):
            send, recv, nb = s.halo_spans(phase)
            fake.rank = r
            SL.p2p_exchange(send, recv, lambda a, nb=nb: SL.device_span(a, nb, dev), r, world, fake)
        fake.flush()
        for s in slabs:
            s.halo_done(phase)

    for _ in range(5):
        exchange(N.HALO_QU)
        for s in slabs:
            s.qtensor_step()
        exchange(N.HALO_F_IN)
        for s in slabs:
            s.lbm_step()
        exchange(N.HALO_F_OUT)
    box.step(5)
    exchange(N.HALO_F_IN)
    outs = [s.download(f=True) for s in slabs]
    ref = box.download(f=True)
    for key, nc in (("rho", 1), ("u", 3), ("q", 5), ("f", 15)):
        got = np.concatenate([o[key].reshape(nc, -1, nxy) for o in outs], axis=1).reshape(-1)
        np.testing.assert_array_equal(got, ref[key], err_msg=key)
    for s in slabs:
        s.close()
    box.close()
