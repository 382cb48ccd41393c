"""Ensemble runner: many independent boxes advanced together on one GPU
(one launch per kernel per step over all boxes, replayed from CUDA graphs),
over the lbman_ensemble_* C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .boundary import BCConfig, FullyPeriodicConfig, SlitConfig
from .device import make_config
from .params import Params, Precision


class Ensemble:
    def __init__(self, boxes, precision: int = Precision.FP32, kernels: int = N.KERNELS_AUTO,
                 device: int = 0, tile=None):
        """boxes: list of (Params, BCConfig)."""
        self.boxes = list(boxes)
        if not self.boxes:
            raise ValueError("an ensemble needs at least one box")
        cfgs = (N.lbman_config * len(self.boxes))()
        for i, (p, bc) in enumerate(self.boxes):
            cfgs[i] = make_config(p, bc, precision, kernels, device, tile)
        h = C.c_void_p()
        N.check(N.lib().lbman_ensemble_create(cfgs, len(self.boxes), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            N.lib().lbman_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __len__(self):
        return len(self.boxes)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_ptr: int):
        N.check(N.lib().lbman_ensemble_set_stream(self._h, C.c_void_p(stream_ptr)))

    def init_seeded(self, seed: int, sigma: float = 1e-3):
        N.check(N.lib().lbman_ensemble_init_seeded(self._h, int(seed), float(sigma)))

    def init_seeded_each(self, seeds, sigma: float = 1e-3):
        """One seed per box (lbman_ensemble_init_seeded_each)."""
        s = (C.c_uint64 * len(self.boxes))(*[int(v) for v in seeds])
        if len(seeds) != len(self.boxes):
            raise ValueError("one seed per box")
        N.check(N.lib().lbman_ensemble_init_seeded_each(self._h, s, float(sigma)))

    def upload(self, box: int, rho, u, q):
        c = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        N.check(N.lib().lbman_ensemble_upload(self._h, int(box), N.dptr(c(rho)), N.dptr(c(u)), N.dptr(c(q))))

    def download(self, box: int, f=False):
        V = self.boxes[box][0].V
        out = dict(rho=np.empty(V), u=np.empty(3 * V), q=np.empty(5 * V))
        if f:
            out["f"] = np.empty(15 * V)
        N.check(N.lib().lbman_ensemble_download(self._h, int(box), N.dptr(out["rho"]), N.dptr(out["u"]),
                                                N.dptr(out["q"]), N.dptr(out.get("f"))))
        return out

    def step(self, n: int = 1):
        N.check(N.lib().lbman_ensemble_step(self._h, int(n)))

    def synchronize(self):
        N.check(N.lib().lbman_ensemble_synchronize(self._h))

    def set_shape(self, kernels: int, tile_x: int, tile_y: int, zchunk: int = 0):
        N.check(N.lib().lbman_ensemble_set_shape(self._h, kernels, tile_x, tile_y, zchunk))

    def shape(self):
        s = N.lbman_shape()
        N.check(N.lib().lbman_ensemble_get_shape(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in N.lbman_shape._fields_}

    def autotune(self, steps_per_trial: int = 5):
        s, n = N.lbman_shape(), C.c_int()
        N.check(N.lib().lbman_ensemble_autotune(self._h, int(steps_per_trial), C.byref(s), C.byref(n)))
        d = {k: getattr(s, k) for k, _ in N.lbman_shape._fields_}
        d["trials"] = n.value
        return d

    def info(self):
        cells, steps, launches = C.c_int64(), C.c_int64(), C.c_int64()
        N.check(N.lib().lbman_ensemble_info(self._h, C.byref(cells), C.byref(steps), C.byref(launches)))
        return {"cells": cells.value, "steps": steps.value, "launches": launches.value}


def shard_boxes(boxes, world: int):
    """Box indices of each of `world` ranks: a cell-balanced greedy
    assignment (largest box first, to the least-loaded rank, ties to the
    lower rank), each rank's list in increasing order.  The loads differ by
    at most the largest box's cell count."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(boxes)), key=lambda i: (-boxes[i][0].V, i))
    load, share = [0] * world, [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += boxes[i][0].V
        share[r].append(i)
    return [sorted(s) for s in share]


class ShardedEnsemble(Ensemble):
    """Rank `rank`'s share of an ensemble spread over `world` GPUs
    (shard_boxes): the boxes are independent, so the ranks exchange nothing
    while stepping.  Box ids are indices in the whole ensemble; seeding uses
    them, so every box's field does not depend on the rank count."""

    def __init__(self, boxes, rank: int, world: int, precision: int = Precision.FP32,
                 kernels: int = N.KERNELS_AUTO, device: int = 0, tile=None):
        self.all_boxes = list(boxes)
        self.ids = shard_boxes(self.all_boxes, world)[rank]
        self.local = {g: i for i, g in enumerate(self.ids)}
        super().__init__([self.all_boxes[g] for g in self.ids], precision, kernels, device, tile)

    def init_seeded(self, seed: int, sigma: float = 1e-3):
        self.init_seeded_each([seed + g for g in self.ids], sigma)

    def download_box(self, box_id: int, f=False):
        """Fields of box `box_id` (an index in the whole ensemble) held here."""
        return self.download(self.local[box_id], f=f)


SIDES = (24, 32, 48, 64, 96)


def draw_boxes(n: int, seed: int, base: Params = None):
    """The batching workload's boxes, drawn from `seed`: cubic or slab shapes
    with every side in {24, 32, 48, 64, 96} (a slab's x side is drawn below
    its equal y = z sides, x being the confined axis of the slit), half fully
    periodic and half slit (free-slip plates confining x), zeta log-uniform in
    [1e-3, 3e-2], LAMBDA uniform in [0.1, 0.7]."""
    base = base or Params()
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        s = int(rng.choice(SIDES))
        if rng.random() < 0.5:
            nx = ny = nz = s
        else:
            smaller = [v for v in SIDES if v < s] or [s]
            nx, ny, nz = int(rng.choice(smaller)), s, s
        zeta = float(np.exp(rng.uniform(np.log(1e-3), np.log(3e-2))))
        lam = float(rng.uniform(0.1, 0.7))
        bc: BCConfig = FullyPeriodicConfig() if i % 2 == 0 else SlitConfig()
        out.append((base.with_(nx=nx, ny=ny, nz=nz, ALPHA=zeta, LAMBDA=lam), bc))
    return out
