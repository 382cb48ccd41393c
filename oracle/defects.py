"""NumPy restatement of the reference's plaquette winding test
(DefectFinder::ComputeWindingNumbers, src/analysis/defect_finder.tpp:13-165,
FlipN src/analysis/defect_fields.cc:17-24).  TEST INFRASTRUCTURE ONLY.

Each face of the director lattice is walked n1 -> n2 -> n3 -> n4 -> n1; a
vertex is flipped when its dot product with the previous (possibly flipped)
vertex is <= 0, and the face is flagged when the closing step n4 -> n1
would flip.  Faces that would cross the box boundary are not visited.
Director fields are AoS (cell*3 + component), cell = (z*ny + y)*nx + x.
"""
from __future__ import annotations

import numpy as np


def _flip_chain(n1, n2, n3, n4):
    def fix(a, b):
        d = np.sum(a * b, axis=-1, keepdims=True)
        return np.where(d <= 0.0, -b, b)
    n2 = fix(n1, n2)
    n3 = fix(n2, n3)
    n4 = fix(n3, n4)
    return (np.sum(n4 * n1, axis=-1) <= 0.0).astype(np.uint8)


def winding_flags(director, nx, ny, nz):
    """(def_x, def_y, def_z) uint8 arrays in the reference's DefectFields layout."""
    D = np.asarray(director, dtype=np.float64).reshape(nz, ny, nx, 3)
    # x faces (y-z loops): (y,z) -> (y+1,z) -> (y+1,z+1) -> (y,z+1)
    fx = _flip_chain(D[:-1, :-1, :], D[:-1, 1:, :], D[1:, 1:, :], D[1:, :-1, :])
    # y faces (x-z loops): (x,z) -> (x+1,z) -> (x+1,z+1) -> (x,z+1)
    fy = _flip_chain(D[:-1, :, :-1], D[:-1, :, 1:], D[1:, :, 1:], D[1:, :, :-1])
    # z faces (x-y loops): (x,y) -> (x+1,y) -> (x+1,y+1) -> (x,y+1)
    fz = _flip_chain(D[:, :-1, :-1], D[:, :-1, 1:], D[:, 1:, 1:], D[:, 1:, :-1])
    return fx.ravel(), fy.ravel(), fz.ravel()
