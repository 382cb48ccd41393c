"""lbman_flow_reduce_noalloc: the flow diagnostics over caller-owned device
fields, with its scratch in a fixed array inside the library, for callers
that cannot call cudaMalloc (a host framework whose allocator holds the
device memory, or a stepping loop that must not allocate or free).

Checked through the C ABI against lbman_reduce, which computes the same sums
with scratch it allocated itself, on two calls in a row (the second call's
relative-change term depends on the velocity the first call stored).  This
file sorts last so a run that stops at the first failure has already run
every other test; it passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

import lbman3d_b200 as L
from lbman3d_b200 import _native as N

pytestmark = pytest.mark.gpu

KEYS = ("mass", "px", "py", "pz", "kinetic_energy", "rel_change_num", "rel_change_den", "umax2")


def _noalloc(ncells, precision, rho, u, upast, stream):
    d = N.lbman_diag()
    st = N.lib().lbman_flow_reduce_noalloc(ncells, precision, C.c_void_p(rho.data_ptr()),
                                           C.c_void_p(u.data_ptr()), C.c_void_p(upast.data_ptr()),
                                           C.c_void_p(stream), C.byref(d))
    N.check(st)
    return {k: getattr(d, k) for k in KEYS} | {"nan_detected": d.nan_detected, "defect_faces": d.defect_faces}


# 40x36x28 = 40 320 cells needs 158 reduction blocks of 256 threads; 96^3 =
# 884 736 cells is above 1184 x 256, so the grid is capped at the scratch
# array's 1184 blocks, each thread sums several cells and the fold runs over
# the whole array.
GRIDS = {"small": (40, 36, 28), "capped": (96, 96, 96)}


@pytest.mark.parametrize("grid", list(GRIDS), ids=list(GRIDS))
@pytest.mark.parametrize("precision", [L.Precision.FP64, L.Precision.FP32], ids=["fp64", "fp32"])
def test_noalloc_flow_reduce_matches_lbman_reduce_on_two_calls(precision, grid):
    import torch

    nx, ny, nz = GRIDS[grid]
    p = L.Params(nx=nx, ny=ny, nz=nz, ALPHA=0.01)
    V = p.V
    dtype = torch.float64 if precision == L.Precision.FP64 else torch.float32
    sim = L.Simulation(p, L.ChannelConfig(), precision)
    sim.init_seeded(17, 0.5, 1e-3)
    stream = torch.cuda.current_stream().cuda_stream
    upast = torch.zeros(3 * V, dtype=dtype, device="cuda")  # caller-owned, like AnalysisFields::u*_past_
    for call in range(2):
        sim.step(5)
        ref = sim.reduce(N.DIAG_FLOW)
        host = sim.download()
        rho = torch.tensor(host["rho"], dtype=dtype, device="cuda")
        u = torch.tensor(host["u"], dtype=dtype, device="cuda")
        got = _noalloc(V, precision, rho, u, upast, stream)
        for k in KEYS:
            assert abs(got[k] - ref[k]) <= 1e-12 * max(abs(ref[k]), 1e-300), (call, k, got[k], ref[k])
        assert got["nan_detected"] == 0 and got["defect_faces"] == -1
        # upast now holds this call's velocity, as lbman_reduce keeps its own copy
        np.testing.assert_array_equal(upast.cpu().numpy(), u.cpu().numpy())
    assert got["rel_change_num"] > 0.0
    sim.close()


def test_noalloc_rejects_sizes_beyond_the_maximum():
    import torch

    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    d = N.lbman_diag()
    args = (C.c_void_p(x.data_ptr()),) * 3 + (None, C.byref(d))
    assert N.lib().lbman_flow_reduce_noalloc(2 ** 31, L.Precision.FP64, *args) == N.ERR_ARG
    assert "LBMAN_NOALLOC_MAX_CELLS" in N.lib().lbman_last_error().decode()
    assert N.lib().lbman_flow_reduce_noalloc(0, L.Precision.FP64, *args) == N.ERR_ARG
    assert N.lib().lbman_flow_reduce_noalloc(8, L.Precision.FP16, *args) == N.ERR_ARG
