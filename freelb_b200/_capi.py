"""ctypes declarations for include/flb.h (libflb_b200.so).

The library is loaded from this package directory only; there is no fallback.
If the shared object is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libflb_b200.so")

FLB_OK = 0
ERR_NUMERIC, ERR_TIMEOUT = -5, -4
ROUND_DEFAULT, ROUND_NEAREST, ROUND_STOCHASTIC = -1, 0, 1
ERRORS = {-1: "FLB_ERR_INVALID", -2: "FLB_ERR_CUDA", -3: "FLB_ERR_OOM", -4: "FLB_ERR_TIMEOUT",
          -5: "FLB_ERR_NUMERIC", -6: "FLB_ERR_UNSUPPORTED", -7: "FLB_ERR_STATE"}

STORAGE_FP32, STORAGE_FP16S, STORAGE_FP64, STORAGE_FP32S = 0, 1, 2, 3
MODEL_BGK, MODEL_MRT, MODEL_LES, MODEL_BRINKMAN = 0, 1, 2, 3
OP_NONE, OP_BULK, OP_BOUNCEBACK, OP_MOVINGWALL, OP_FIELD_BGK = 0, 1, 2, 3, 4
DTYPE_F32, DTYPE_F64 = 0, 1
FIELD_RHO, FIELD_VELOCITY, FIELD_ALPHA = 0, 1, 2
MAX_TASKS = 8


class LatticeDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("storage", ctypes.c_int), ("model", ctypes.c_int),
                ("omega", ctypes.c_double), ("smagorinsky", ctypes.c_double),
                ("mrt_rates", ctypes.c_double * 19), ("rho0", ctypes.c_double),
                ("ntasks", ctypes.c_int), ("task_keys", ctypes.c_uint8 * MAX_TASKS),
                ("task_ops", ctypes.c_uint8 * MAX_TASKS)]


class BlockDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("ox", ctypes.c_int), ("oy", ctypes.c_int), ("oz", ctypes.c_int),
                ("omega", ctypes.c_double)]


BLOCKS_INDEPENDENT, BLOCKS_HALO = 0, 1


class Layout(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("pitch_x", ctypes.c_int), ("plane", ctypes.c_size_t),
                ("dir_stride", ctypes.c_size_t), ("elem_bytes", ctypes.c_int)]


class FlbError(RuntimeError):
    def __init__(self, code, fn, msg):
        super().__init__(f"{fn}: {ERRORS.get(code, code)}: {msg}")
        self.code = code


_P = ctypes.c_void_p
_I = ctypes.c_int
# name -> argtypes (all return int unless listed in _RESTYPES)
SIGNATURES = {
    "flb_version": [ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "flb_last_error": [],
    "flb_desc_default": [ctypes.POINTER(LatticeDesc), _I, _I, _I, ctypes.c_double],
    "flb_create": [ctypes.POINTER(LatticeDesc), ctypes.POINTER(_P)],
    "flb_destroy": [_P],
    "flb_memory_bytes": [_P, ctypes.POINTER(ctypes.c_size_t)],
    "flb_upload_flags": [_P, _P, _P],
    "flb_download_flags": [_P, _P, _P],
    "flb_upload_pops": [_P, _P, _I, _P],
    "flb_download_pops": [_P, _P, _I, _P],
    "flb_upload_field": [_P, _I, _P, _I, _P],
    "flb_download_field": [_P, _I, _P, _I, _P],
    "flb_init_equilibrium": [_P, ctypes.c_double, _P],
    "flb_step": [_P, _I, _P],
    "flb_compute_rhou": [_P, ctypes.c_uint8, _P],
    "flb_reduce_conservation": [_P, ctypes.c_uint8, ctypes.POINTER(ctypes.c_double), _P],
    "flb_tolerance_u": [_P, ctypes.c_uint8, ctypes.POINTER(ctypes.c_double), _P],
    "flb_check_finite": [_P, ctypes.POINTER(ctypes.c_uint64), _P],
    "flb_get_layout": [_P, ctypes.POINTER(Layout)],
    "flb_device_pointers": [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P),
                            ctypes.POINTER(_P)],
    "flb_create_blocks": [ctypes.POINTER(LatticeDesc), _I, ctypes.POINTER(BlockDesc), _I,
                          ctypes.POINTER(_P)],
    "flb_block_count": [_P, ctypes.POINTER(_I)],
    "flb_halo_count": [_P, ctypes.POINTER(ctypes.c_longlong)],
    "flb_upload_flags_block": [_P, _I, _P, _P],
    "flb_download_flags_block": [_P, _I, _P, _P],
    "flb_upload_pops_block": [_P, _I, _P, _I, _P],
    "flb_download_pops_block": [_P, _I, _P, _I, _P],
    "flb_upload_field_block": [_P, _I, _I, _P, _I, _P],
    "flb_download_field_block": [_P, _I, _I, _P, _I, _P],
    "flb_set_launch": [_P, _I, _I, _I],
    "flb_get_launch": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "flb_set_wait_limit": [_P, ctypes.c_double],
    "flb_device_status": [_P, _P],
    "flb_test_withhold_tile": [_P, ctypes.c_longlong],
    "flb_set_rounding": [_P, _I],
    "flb_snapshot_bytes": [_P, ctypes.POINTER(ctypes.c_size_t)],
    "flb_snapshot_save": [_P, _P, ctypes.c_size_t, _P],
    "flb_snapshot_restore": [_P, _P, ctypes.c_size_t, _P],
    "flb_get_rounding": [_P, ctypes.POINTER(_I)],
    "flb_autotune": [_P, _I, _P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I),
                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_I)],
    "flb_step_graph": [_P, _I, _P],
    "flb_objective_u2": [_P, ctypes.POINTER(ctypes.c_double), _P],
    "flb_adjoint_forward": [_P, _I, _I, ctypes.POINTER(ctypes.c_double), _P],
    "flb_adjoint_backward": [_P, _P, ctypes.POINTER(ctypes.c_double),
                             ctypes.POINTER(ctypes.c_double), _P],
    "flb_adjoint_release": [_P],
    "flb_set_tasks": [_P, _I, _P, _P, _I],
    "flb_reduce_conservation_noalloc": [_P, _P, ctypes.POINTER(Layout), _I, ctypes.c_double,
                                        ctypes.c_uint8, ctypes.POINTER(ctypes.c_double), _P],
    "flb_bb_create": [_P, ctypes.c_uint8, ctypes.c_uint8, _I, ctypes.c_double,
                      ctypes.POINTER(_P)],
    "flb_bb_count": [_P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)],
    "flb_bb_apply": [_P, _P, _P],
    "flb_bb_destroy": [_P],
    "flb_periodic_create": [_P, ctypes.POINTER(_I), _I, ctypes.POINTER(_I), _I, ctypes.c_uint8,
                            ctypes.POINTER(_P)],
    "flb_periodic_count": [_P, ctypes.POINTER(ctypes.c_longlong),
                           ctypes.POINTER(ctypes.c_longlong)],
    "flb_periodic_apply": [_P, _P, _P],
    "flb_periodic_destroy": [_P],
    "flb_set_halo_mode": [_P, _I],
    "flb_exchange_plan": [_I, ctypes.POINTER(BlockDesc), ctypes.POINTER(_I), _I, _I, _I,
                          ctypes.POINTER(_I), ctypes.POINTER(_I),
                          ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)],
    "flb_exchange_create": [_P, _I, ctypes.POINTER(BlockDesc), ctypes.POINTER(_I), _I,
                            ctypes.POINTER(_P)],
    "flb_exchange_peers": [_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I),
                           ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)],
    "flb_exchange_pack": [_P, _P, _I, _P, _P],
    "flb_exchange_unpack": [_P, _P, _I, _P, _P],
    "flb_exchange_destroy": [_P],
    "flb_vtk_field_base64": [_P, _I, _I, _I, _I, _I, ctypes.c_double, ctypes.c_double,
                             ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), _P],
}
VTK_FLAG = 16
HALO_NORMAL, HALO_FULL = 0, 1
BB_NORMAL, BB_MOVINGWALL, BB_ANTI_SIMPLE, BB_ANTI_O1, BB_ANTI_O2, BB_ANTI_PRESSURE = range(6)
_RESTYPES = {"flb_last_error": ctypes.c_char_p}

_lib = None


def load():
    """Load libflb_b200.so (raises if it is absent: there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m freelb_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib


def call(name, *args):
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != FLB_OK:
        raise FlbError(rc, name, lib.flb_last_error().decode())
    return rc
