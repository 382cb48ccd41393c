"""One box split into z-slabs across GPUs, or across handles on one GPU.

Replaces the reference's MPI domain decomposition (src/mpi/mpi_context.h,
src/mpi/halo_exchange_qtensor.h:131-209, src/mpi/halo_exchange_lbm.h:304-386)
for the single split axis z; the library side is ``lbman_create_slab`` and the
``lbman_halo_*`` entry points of include/lbman3d.h.

A step of every slab is::

    exchange(QU)     Q (5) and u (3), 2 owned planes -> the neighbours' ghosts
    qtensor_step     Q+force kernel over the owned planes (it computes the
                     passive stresses of the ghost planes itself, so the
                     reference's second, Sigma/tau exchange is not needed)
    exchange(F_IN)   before an odd in-place LBM step: 5 crossing populations
    lbm_step         in-place collide-and-stream over the owned planes
    exchange(F_OUT)  after an odd step: the populations scattered into the
                     ghost planes go back to the neighbours' boundary planes

Even in-place steps touch only their own cells, so the population exchanges
run every other step and move 5 of the 15 slots of one plane.

Two transports deliver the spans the library names:

* :class:`SlabBox` -- one process, all slabs (``lbman_slab_exchange``: peer
  ``cudaMemcpyAsync`` on the receivers' streams, ordered by events);
* :class:`DistributedSlab` -- one rank per GPU, ``torch.distributed``
  point-to-point over NCCL (:func:`p2p_exchange`), the slab's kernels on
  torch's current stream so the exchange needs no host synchronisation.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .boundary import BCConfig, SimBC
from .device import Simulation, make_config
from .params import Params, Precision

PHASES = (N.HALO_QU, N.HALO_F_IN, N.HALO_F_OUT)


def split_planes(nz: int, nslabs: int):
    """(z_offset, nz_local) of each slab: planes split as evenly as possible,
    the larger slabs first.  Every slab owns at least 2 planes."""
    if nslabs < 1 or nz < 2 * nslabs:
        raise ValueError(f"{nz} planes cannot give {nslabs} slabs of at least 2 planes")
    base, extra = divmod(nz, nslabs)
    out, z = [], 0
    for i in range(nslabs):
        n = base + (1 if i < extra else 0)
        out.append((z, n))
        z += n
    return out


def halo_plan(nz_local: int, phase: int):
    """The library's exchange plan for a slab of nz_local planes (host only):
    ``send[f][k]`` goes to the neighbour across face f (0 low z, 1 high z),
    which receives it into its ``recv[1-f][k]``.  Spans are dicts with
    field, comp, plane (owned coordinates; ghosts -2, -1, nz_local,
    nz_local+1) and planes."""
    M = N.HALO_MAX_SPANS
    send, recv, n = (N.lbman_halo_span * (2 * M))(), (N.lbman_halo_span * (2 * M))(), C.c_int()
    N.check(N.lib().lbman_halo_plan(int(nz_local), int(phase), send, recv, C.byref(n)))
    conv = lambda s: {k: getattr(s, k) for k, _ in N.lbman_halo_span._fields_}
    return ([[conv(send[f * M + k]) for k in range(n.value)] for f in range(2)],
            [[conv(recv[f * M + k]) for k in range(n.value)] for f in range(2)])


class Slab(Simulation):
    """Planes [z_offset, z_offset + nz_local) of a box described by
    ``params`` (its nz is the whole box's).  Host arrays (upload, download)
    hold the owned planes only."""

    def __init__(self, params: Params, bc: BCConfig = None, precision: int = Precision.FP64,
                 kernels: int = N.KERNELS_AUTO, z_offset: int = 0, nz_local: int = None, device: int = 0,
                 tile=None):
        nz_local = params.nz if nz_local is None else int(nz_local)
        self.box = params
        self.z_offset, self.nz_local = int(z_offset), nz_local
        self.params = params.with_(nz=nz_local)
        self.bc = bc if bc is not None else SimBC()
        self.precision = precision
        self.device = int(device)
        self.cfg = make_config(self.params, self.bc, precision, kernels, device, tile)
        h = C.c_void_p()
        N.check(N.lib().lbman_create_slab(C.byref(self.cfg), int(params.nz), self.z_offset, C.byref(h)))
        self._h = h

    def halo_spans(self, phase: int):
        """(send, recv, span_bytes): device addresses [2][n] of this phase's
        spans in the current buffers; n = 0 when the phase moves nothing."""
        M = N.HALO_MAX_SPANS
        send, recv = (C.c_void_p * (2 * M))(), (C.c_void_p * (2 * M))()
        nbytes, n = C.c_size_t(), C.c_int()
        N.check(N.lib().lbman_halo_spans(self._h, int(phase), send, recv, C.byref(nbytes), C.byref(n)))
        return ([[send[f * M + k] for k in range(n.value)] for f in range(2)],
                [[recv[f * M + k] for k in range(n.value)] for f in range(2)], nbytes.value)

    def halo_done(self, phase: int):
        N.check(N.lib().lbman_halo_done(self._h, int(phase)))


def _split_field(a: np.ndarray, ncomp: int, nxy: int, parts):
    """Owned-plane blocks of a whole-box field of ncomp components."""
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(ncomp, -1, nxy)
    return [np.ascontiguousarray(a[:, z0:z0 + n]).reshape(-1) for z0, n in parts]


def combine_diag(diags):
    """Whole-box diagnostics from per-slab ones: sums, and the maximum of
    |u|^2."""
    out = {}
    for k in diags[0]:
        if k == "umax2":
            out[k] = max(d[k] for d in diags)
        elif k == "nan_detected":
            out[k] = int(any(d[k] for d in diags))
        elif k == "defect_faces":
            out[k] = -1
        else:
            out[k] = sum(d[k] for d in diags)
    return out


class SlabBox:
    """A box as ``nslabs`` z-slabs driven by one process (slab i on
    ``devices[i % len(devices)]``), exchanging through
    ``lbman_slab_exchange``."""

    def __init__(self, params: Params, bc: BCConfig = None, precision: int = Precision.FP64, nslabs: int = 2,
                 kernels: int = N.KERNELS_AUTO, devices=(0,), tile=None, planes=None):
        self.params = params
        self.parts = list(planes) if planes is not None else split_planes(params.nz, nslabs)
        self.slabs = []
        try:
            for i, (z0, n) in enumerate(self.parts):
                self.slabs.append(Slab(params, bc, precision, kernels, z0, n, devices[i % len(devices)], tile))
        except Exception:
            self.close()
            raise
        self._handles = (C.c_void_p * len(self.slabs))(*[s.handle.value for s in self.slabs])

    @property
    def nxy(self):
        return self.params.nx * self.params.ny

    def close(self):
        for s in self.slabs:
            s.close()
        self.slabs = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def exchange(self, phase: int):
        N.check(N.lib().lbman_slab_exchange(self._handles, len(self.slabs), int(phase)))

    def upload(self, rho, u, q):
        parts = [_split_field(a, nc, self.nxy, self.parts) for a, nc in ((rho, 1), (u, 3), (q, 5))]
        for s, r, uu, qq in zip(self.slabs, *parts):
            s.upload(r, uu, qq)

    def init_seeded(self, seed: int, S0: float, sigma: float = 1e-3):
        for s in self.slabs:
            s.init_seeded(seed, S0, sigma)

    def step(self, n: int = 1):
        for _ in range(int(n)):
            self.exchange(N.HALO_QU)
            for s in self.slabs:
                s.qtensor_step()
            self.exchange(N.HALO_F_IN)
            for s in self.slabs:
                s.lbm_step()
            self.exchange(N.HALO_F_OUT)

    def synchronize(self):
        for s in self.slabs:
            s.synchronize()

    def download(self, f=False):
        """Whole-box fields assembled from the slabs' owned planes."""
        if f:
            self.exchange(N.HALO_F_IN)  # a slab between steps may need its halo to rebuild f
        outs = [s.download(f=f) for s in self.slabs]
        res = {}
        for key, nc in (("rho", 1), ("u", 3), ("q", 5), ("f", 15)):
            if key in outs[0]:
                blocks = [o[key].reshape(nc, -1, self.nxy) for o in outs]
                res[key] = np.concatenate(blocks, axis=1).reshape(-1)
        return res

    def reduce(self, flags: int = N.DIAG_FLOW | N.DIAG_ENERGY):
        if flags & N.DIAG_ENERGY:
            self.exchange(N.HALO_QU)
        return combine_diag([s.reduce(flags) for s in self.slabs])


# ---- one rank per GPU -------------------------------------------------------


class _CudaBytes:
    """A byte range of device memory, for torch.as_tensor (no copy)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3}


def device_span(ptr: int, nbytes: int, device):
    import torch
    return torch.as_tensor(_CudaBytes(ptr, nbytes), device=device)


def p2p_exchange(send, recv, to_tensor, rank: int, world: int, dist, group=None):
    """Delivers one phase's spans between ranks of a ring of slabs
    (world >= 2): send[f][k] to the neighbour across face f, recv[f][k] from
    it.  Every rank posts, per k, its two sends (low face, high face) and its
    two receives (high face, low face), so with two ranks -- one neighbour
    across both faces -- the i-th message between a pair is matched in the
    same order on both sides."""
    lo, hi = (rank - 1) % world, (rank + 1) % world
    ops = []
    for k in range(len(send[0])):
        ops.append(dist.P2POp(dist.isend, to_tensor(send[0][k]), lo, group))
        ops.append(dist.P2POp(dist.isend, to_tensor(send[1][k]), hi, group))
        ops.append(dist.P2POp(dist.irecv, to_tensor(recv[1][k]), hi, group))
        ops.append(dist.P2POp(dist.irecv, to_tensor(recv[0][k]), lo, group))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()


class DistributedSlab:
    """This rank's slab of a box split over the ranks of ``group`` (rank r
    owns the r-th block of planes), exchanging with NCCL point-to-point
    operations.  The slab runs on torch's current stream, so the exchanges
    are ordered with its kernels on the device."""

    def __init__(self, params: Params, bc: BCConfig = None, precision: int = Precision.FP64,
                 kernels: int = N.KERNELS_AUTO, group=None, tile=None):
        import torch
        import torch.distributed as dist
        self.dist, self.group = dist, group
        if dist.is_available() and dist.is_initialized():
            self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        else:  # one process: the whole box in one slab
            self.rank, self.world = 0, 1
        self.device = torch.cuda.current_device()
        z0, n = split_planes(params.nz, self.world)[self.rank]
        self.slab = Slab(params, bc, precision, kernels, z0, n, self.device, tile)
        self.slab.set_stream(torch.cuda.current_stream().cuda_stream)
        self._handles = (C.c_void_p * 1)(self.slab.handle.value)

    def close(self):
        self.slab.close()

    def exchange(self, phase: int):
        if self.world == 1:  # the box's periodic z faces meet in this slab
            N.check(N.lib().lbman_slab_exchange(self._handles, 1, int(phase)))
            return
        send, recv, nbytes = self.slab.halo_spans(phase)
        to_t = lambda p: device_span(p, nbytes, self.device)
        p2p_exchange(send, recv, to_t, self.rank, self.world, self.dist, self.group)
        self.slab.halo_done(phase)

    def step(self, n: int = 1):
        for _ in range(int(n)):
            self.exchange(N.HALO_QU)
            self.slab.qtensor_step()
            self.exchange(N.HALO_F_IN)
            self.slab.lbm_step()
            self.exchange(N.HALO_F_OUT)

    def reduce(self, flags: int = N.DIAG_FLOW | N.DIAG_ENERGY):
        """Whole-box diagnostics: this slab's sums, all-reduced over the ranks."""
        import torch
        if flags & N.DIAG_ENERGY:
            self.exchange(N.HALO_QU)
        d = self.slab.reduce(flags)
        keys = [k for k in d if k not in ("umax2", "nan_detected", "defect_faces")]
        s = torch.tensor([d[k] for k in keys], dtype=torch.float64, device=self.device)
        m = torch.tensor([d["umax2"], float(d["nan_detected"])], dtype=torch.float64, device=self.device)
        if self.world > 1:
            self.dist.all_reduce(s, group=self.group)
            self.dist.all_reduce(m, op=self.dist.ReduceOp.MAX, group=self.group)
        out = dict(zip(keys, s.tolist()))
        out["umax2"], out["nan_detected"], out["defect_faces"] = m[0].item(), int(m[1].item()), -1
        return out
