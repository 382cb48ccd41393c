"""Helpers to read the golden fixtures (tests/golden/*.npz)."""
import ast
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["grid"] = tuple(int(v) for v in d["grid"])
    d["faces"] = ast.literal_eval(str(d["faces"]))
    d["phys"] = ast.literal_eval(str(d["phys"]))
    d["upwind"] = bool(d["upwind"])
    d["mode"] = str(d["mode"])
    d["steps"] = [int(s) for s in d["steps"]]
    d["in_force"] = d["in_force"] if d["in_force"].size else None
    return d
