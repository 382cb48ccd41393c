"""ctypes binding of include/lbman3d.h (liblbman3d_b200.so, built in tree).

The shared library is the product: there is no Python or CPU fallback.  If
it is missing, every entry point raises ImportError with the build command.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liblbman3d_b200.so")

OK, ERR_ARG, ERR_CUDA, ERR_DIVERGED, ERR_TIMEOUT, ERR_STATE, ERR_UNSUPPORTED, ERR_NOMEM = range(8)
Q_PERIODIC, Q_NEUMANN, Q_ANCHORING = 0, 1, 2
U_PERIODIC, U_NOSLIP, U_MOVING, U_SPECULAR = 0, 1, 2, 3
CENTRED, UPWIND = 0, 1
FP64, FP32, FP16 = 0, 1, 2
KERNELS_AUTO, KERNELS_SPLIT, KERNELS_FUSED, KERNELS_SPLIT_PAIR = 0, 1, 2, 3
DIAG_FLOW, DIAG_ENERGY, DIAG_DEFECTS, DIAG_ALL = 1, 2, 4, 7
HALO_QU, HALO_F_IN, HALO_F_OUT = 0, 1, 2
HALO_MAX_SPANS = 8
FIELD_Q, FIELD_U, FIELD_F, FIELD_FSTAGE = 0, 1, 2, 3


class lbman_face(C.Structure):
    _fields_ = [("qbc", C.c_int), ("s", C.c_double), ("theta", C.c_double), ("phi", C.c_double),
                ("ubc", C.c_int), ("uw", C.c_double * 3)]


class lbman_config(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("DT", C.c_double), ("kDensity", C.c_double), ("TAUF", C.c_double),
                ("L", C.c_double), ("A", C.c_double), ("B", C.c_double), ("C", C.c_double),
                ("LAMBDA", C.c_double), ("GAMMA", C.c_double), ("ALPHA", C.c_double),
                ("MU", C.c_double), ("advection", C.c_int), ("face", lbman_face * 6),
                ("precision", C.c_int), ("kernels", C.c_int), ("device", C.c_int),
                ("tile_x", C.c_int), ("tile_y", C.c_int), ("zchunk", C.c_int), ("threads", C.c_int)]


class lbman_diag(C.Structure):
    _fields_ = [("mass", C.c_double), ("px", C.c_double), ("py", C.c_double), ("pz", C.c_double),
                ("kinetic_energy", C.c_double), ("rel_change_num", C.c_double),
                ("rel_change_den", C.c_double), ("umax2", C.c_double), ("free_energy", C.c_double),
                ("defect_faces", C.c_int64), ("nan_detected", C.c_int)]


class lbman_shape(C.Structure):
    _fields_ = [("kernels", C.c_int), ("tile_x", C.c_int), ("tile_y", C.c_int), ("zchunk", C.c_int),
                ("threads", C.c_int), ("ms_per_step", C.c_double), ("blocks", C.c_int)]


class lbman_defects(C.Structure):
    _fields_ = [("faces", C.c_int64), ("edges", C.c_int64), ("lines", C.c_int64), ("points", C.c_int64)]


class lbman_halo_span(C.Structure):
    _fields_ = [("field", C.c_int), ("comp", C.c_int), ("plane", C.c_int), ("planes", C.c_int)]


class lbman_stats(C.Structure):
    _fields_ = [("mean_speed", C.c_double), ("rms_speed", C.c_double), ("defect_faces", C.c_int64),
                ("defect_density", C.c_double)]


STATS_MAX_BINS = 8192
CLOSURE_WAIT_DEFAULT = 67108864  # LBMAN_CLOSURE_WAIT_DEFAULT


class LbmanError(RuntimeError):
    """A non-zero status from the C ABI (the reference throws std::runtime_error)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"lbman status {status}: {message}")
        self.status = status


class DivergedError(LbmanError):
    pass


_lib = None

# (name, restype, argtypes) for every entry point declared in include/lbman3d.h
_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)
PROTOTYPES = [
    ("lbman_config_init", C.c_int, [C.POINTER(lbman_config)]),
    ("lbman_status_string", C.c_char_p, [C.c_int]),
    ("lbman_last_error", C.c_char_p, []),
    ("lbman_abi_version", C.c_int, []),
    ("lbman_device_info", C.c_int, [C.c_int, C.c_char_p, C.c_size_t]),
    ("lbman_create", C.c_int, [C.POINTER(lbman_config), C.POINTER(C.c_void_p)]),
    ("lbman_destroy", C.c_int, [C.c_void_p]),
    ("lbman_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("lbman_synchronize", C.c_int, [C.c_void_p]),
    ("lbman_upload", C.c_int, [C.c_void_p, _DP, _DP, _DP, _DP, _DP]),
    ("lbman_init_seeded", C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.c_double]),
    ("lbman_download", C.c_int, [C.c_void_p, _DP, _DP, _DP, _DP, _DP]),
    ("lbman_step", C.c_int, [C.c_void_p, C.c_int]),
    ("lbman_qtensor_step", C.c_int, [C.c_void_p]),
    ("lbman_lbm_step", C.c_int, [C.c_void_p]),
    ("lbman_qtensor_setup", C.c_int, [C.c_void_p]),
    ("lbman_active_force", C.c_int, [C.c_void_p]),
    ("lbman_download_stress", C.c_int, [C.c_void_p, _DP, _DP]),
    ("lbman_upload_stress", C.c_int, [C.c_void_p, _DP, _DP]),
    ("lbman_reduce", C.c_int, [C.c_void_p, C.c_int, C.POINTER(lbman_diag)]),
    ("lbman_steps_done", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    ("lbman_launch_count", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    ("lbman_get_shape", C.c_int, [C.c_void_p, C.POINTER(lbman_shape)]),
    ("lbman_set_shape", C.c_int, [C.c_void_p, C.POINTER(lbman_shape)]),
    ("lbman_autotune", C.c_int, [C.c_void_p, C.c_int, C.POINTER(lbman_shape), C.POINTER(C.c_int)]),
    ("lbman_ensemble_create", C.c_int, [C.POINTER(lbman_config), C.c_int, C.POINTER(C.c_void_p)]),
    ("lbman_ensemble_destroy", C.c_int, [C.c_void_p]),
    ("lbman_ensemble_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("lbman_ensemble_init_seeded", C.c_int, [C.c_void_p, C.c_uint64, C.c_double]),
    ("lbman_ensemble_init_seeded_each", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.c_double]),
    ("lbman_ensemble_upload", C.c_int, [C.c_void_p, C.c_int, _DP, _DP, _DP]),
    ("lbman_ensemble_download", C.c_int, [C.c_void_p, C.c_int, _DP, _DP, _DP, _DP]),
    ("lbman_ensemble_step", C.c_int, [C.c_void_p, C.c_int]),
    ("lbman_ensemble_synchronize", C.c_int, [C.c_void_p]),
    ("lbman_ensemble_set_shape", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("lbman_ensemble_get_shape", C.c_int, [C.c_void_p, C.POINTER(lbman_shape)]),
    ("lbman_ensemble_autotune", C.c_int, [C.c_void_p, C.c_int, C.POINTER(lbman_shape), C.POINTER(C.c_int)]),
    ("lbman_ensemble_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64)]),
    ("lbman_velocity_spectrum", C.c_int, [C.c_void_p, C.c_int, _DP, _DP]),
    ("lbman_q_correlation", C.c_int, [C.c_void_p, C.c_int, _DP, _DP, _DP]),
    ("lbman_statistics", C.c_int, [C.c_void_p, C.POINTER(lbman_stats)]),
    ("lbman_defect_lines", C.c_int, [C.c_void_p, C.POINTER(lbman_defects), _DP, C.c_int64,
                                     C.POINTER(C.c_int64), C.c_int64]),
    ("lbman_defect_graph", C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.POINTER(lbman_defects), _DP, C.c_int64,
                                     C.POINTER(C.c_int64), C.c_int64]),
    ("lbman_closure_selftest", C.c_int, [C.c_int, _DP]),
    ("lbman_closure_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    ("lbman_closure_destroy", C.c_int, [C.c_void_p]),
    ("lbman_closure_param_count", C.c_int, []),
    ("lbman_closure_get_params", C.c_int, [C.c_void_p, _FP]),
    ("lbman_closure_set_params", C.c_int, [C.c_void_p, _FP]),
    ("lbman_closure_get_scales", C.c_int, [C.c_void_p, _FP, _FP, _FP]),
    ("lbman_closure_set_scales", C.c_int, [C.c_void_p, _FP, _FP, _FP]),
    ("lbman_closure_forward", C.c_int, [C.c_void_p, _FP, _FP]),
    ("lbman_closure_gradient", C.c_int, [C.c_void_p, _FP, _FP, _DP, _FP]),
    ("lbman_closure_record", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("lbman_closure_record_box", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    ("lbman_closure_add_rollout_pairs", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                  C.POINTER(C.c_int)]),
    ("lbman_closure_dataset", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("lbman_closure_build_targets", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("lbman_closure_train", C.c_int, [C.c_void_p, C.c_int, C.c_float, C.c_uint64, _DP, _DP]),
    ("lbman_closure_load_snapshot", C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    ("lbman_closure_step", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("lbman_closure_set_options", C.c_int, [C.c_void_p, C.c_float, C.c_float]),
    ("lbman_closure_set_wait_limit", C.c_int, [C.c_void_p, C.c_uint32]),
    ("lbman_create_slab", C.c_int, [C.POINTER(lbman_config), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("lbman_halo_plan", C.c_int, [C.c_int, C.c_int, C.POINTER(lbman_halo_span), C.POINTER(lbman_halo_span),
                                  C.POINTER(C.c_int)]),
    ("lbman_halo_spans", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                   C.POINTER(C.c_size_t), C.POINTER(C.c_int)]),
    ("lbman_halo_done", C.c_int, [C.c_void_p, C.c_int]),
    ("lbman_slab_exchange", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int]),
    ("lbman_slab_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("lbman_flow_reduce_noalloc", C.c_int,
     [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(lbman_diag)]),
]


def lib():
    """Load liblbman3d_b200.so (once).  Raises ImportError if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m lbman3d_b200.build` "
                              "(nvcc, sm_100a). There is no CPU fallback.")
        L = C.CDLL(LIB_PATH)
        for name, res, args in PROTOTYPES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int):
    if status != OK:
        msg = lib().lbman_last_error().decode(errors="replace")
        if status == ERR_DIVERGED:
            raise DivergedError(status, msg)
        raise LbmanError(status, msg)
    return status


def defect_graph(nx, ny, nz, qper6, def_x, def_y, def_z, with_points=True):
    """lbman_defect_graph on host flag arrays: (info dict, points (n,3), offsets)."""
    import numpy as np
    fx, fy, fz = (np.ascontiguousarray(a, dtype=np.uint8) for a in (def_x, def_y, def_z))
    q = (C.c_int * 6)(*[int(bool(v)) for v in qper6])
    info = lbman_defects()
    args = (int(nx), int(ny), int(nz), q, fx.ctypes.data_as(C.c_void_p), fy.ctypes.data_as(C.c_void_p),
            fz.ctypes.data_as(C.c_void_p), C.byref(info))
    check(lib().lbman_defect_graph(*args, None, 0, None, 0))
    if not with_points:
        return {k: getattr(info, k) for k, _ in lbman_defects._fields_}, None, None
    pts = np.zeros(3 * max(info.points, 1))
    off = np.zeros(info.lines + 1, dtype=np.int64)
    check(lib().lbman_defect_graph(*args, pts.ctypes.data_as(_DP), pts.size,
                                   off.ctypes.data_as(C.POINTER(C.c_int64)), off.size))
    return {k: getattr(info, k) for k, _ in lbman_defects._fields_}, pts[:3 * info.points].reshape(-1, 3), off


def fptr(a):
    """float32 C-contiguous numpy array -> float*, None -> NULL."""
    if a is None:
        return None
    if a.dtype.name != "float32" or not a.flags.c_contiguous:
        raise TypeError("buffers must be C-contiguous float32 arrays")
    return a.ctypes.data_as(_FP)


def dptr(a):
    """float64 C-contiguous numpy array -> double*, None -> NULL."""
    if a is None:
        return None
    if a.dtype.name != "float64" or not a.flags.c_contiguous:
        raise TypeError("host buffers must be C-contiguous float64 arrays")
    return a.ctypes.data_as(_DP)
