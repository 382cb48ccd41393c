"""Disclination lines against the reference's own DefectFinder output.

CPU: plaquette flags from the reference's director field in each golden
fixture (oracle/defects.py restates the winding test) go through the
library's host graph builder (lbman_defect_graph); the flagged-face and
disclination counts must equal the reference's.
GPU: the same through lbman_defect_lines on the FP64 GPU state.
"""
import numpy as np
import pytest

import lbman3d_b200 as L
from golden_util import load, names
from oracle import defects as D

CASES = [n for n in names() if int(load(n)["s0_defect_faces"]) >= 0]


def _qper(faces):
    return [f[0] == 0 for f in faces]


@pytest.mark.parametrize("name", CASES)
def test_graph_from_reference_director_matches_reference(name):
    g = load(name)
    nx, ny, nz = g["grid"]
    for k in range(len(g["steps"])):
        fx, fy, fz = D.winding_flags(g[f"s{k}_director"], nx, ny, nz)
        info, pts, off = L._native.defect_graph(nx, ny, nz, _qper(g["faces"]), fx, fy, fz)
        assert info["faces"] == int(g[f"s{k}_defect_faces"]), (name, k)
        assert info["lines"] == int(g[f"s{k}_disclinations"]), (name, k)
        assert off[0] == 0 and off[-1] == info["points"] and np.all(np.diff(off) >= 1)
        assert pts.shape == (info["points"], 3)
        assert np.all(pts >= 0) and np.all(pts[:, 0] <= nx) and np.all(pts[:, 2] <= nz)


def test_graph_rejects_thin_boxes():
    z = np.zeros(10, dtype=np.uint8)
    with pytest.raises(L._native.LbmanError):
        L._native.defect_graph(1, 4, 4, [1] * 6, z, z, z)


@pytest.mark.gpu
@pytest.mark.parametrize("name", [n for n in CASES if load(n)["mode"] == "full"])
def test_gpu_defect_lines_match_reference(name):
    from test_gpu_parity import sim_from
    g = load(name)
    sim = sim_from(g["grid"], g["faces"], g["phys"], g["upwind"])
    sim.upload(g["in_rho"], g["in_u"], g["in_q"], None, g["in_force"])
    done = 0
    for k, t in enumerate(g["steps"]):
        sim.step(t - done)
        done = t
        info, pts, off = sim.defect_lines()
        assert info["faces"] == int(g[f"s{k}_defect_faces"]), (name, k)
        assert info["lines"] == int(g[f"s{k}_disclinations"]), (name, k)
    sim.close()
