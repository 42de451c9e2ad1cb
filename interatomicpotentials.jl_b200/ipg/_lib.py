"""ctypes binding of libipg.so (declarations in include/ipg.h).

The library is built in-tree by ``interatomicpotentials.jl_b200/build.py``.  There is no
CPU fallback: if the library is missing, or no sm_100 device is present, calls raise
``IPGError``.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libipg.so")

IPG_OK = 0
STATUS = {
    -1: "IPG_ERR_ARG", -2: "IPG_ERR_CUDA", -3: "IPG_ERR_NOMEM", -4: "IPG_ERR_CAPACITY",
    -6: "IPG_ERR_NONFINITE", -7: "IPG_ERR_SPECIES", -8: "IPG_ERR_UNSUPPORTED", -9: "IPG_ERR_NODEVICE",
}

PAIR_KIND = {"LJ": 1, "BM": 2, "COUL": 3, "MORSE": 4, "ZBL": 5, "MOCK_R2": 6}
WANT_E, WANT_F, WANT_W = 1, 2, 4
PAIR_GRAPH = 8  # ipg_pair_eval_dev: replay a CUDA graph of the evaluation
DESC_B, DESC_DB, DESC_W = 1, 2, 4
NLIST_HALF, NLIST_FULL, NLIST_LITERAL_SQRT = 0, 1, 0x100
SNAP_PLAIN, SNAP_ADJOINT = 0, 1
MAX_SNAP_SPECIES = 8
MAX_PAIR_TERMS = 16

# Every symbol include/ipg.h declares.
API_SYMBOLS = (
    "ipg_create", "ipg_destroy", "ipg_last_error", "ipg_set_stream", "ipg_version",
    "ipg_launch_count", "ipg_timing_enable", "ipg_timing_read", "ipg_neighbor_build", "ipg_neighbor_count", "ipg_nlist_size", "ipg_nlist_export", "ipg_nlist_free",
    "ipg_pair_eval", "ipg_pair_eval_dev", "ipg_pair_eval_noalloc", "ipg_snap_create", "ipg_snap_destroy", "ipg_snap_ncoeff",
    "ipg_snap_descriptors", "ipg_snap_energy_forces", "ipg_snap_energy_forces_dev", "ipg_snap_vjp_beta",
    "ipg_snap_vjp", "ipg_snap_autotune", "ipg_snap_batch_descriptors", "ipg_snap_set_skin", "ipg_snap_skin_stats",
    "ipg_snap_batch_energy_forces", "ipg_snap_batch_energy_forces_dev", "ipg_snap_batch_loss_grad",
    "ipg_snap_batch_loss_grad_dev",
)


class IPGError(RuntimeError):
    def __init__(self, status, message=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {message}")


class PairTerm(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("coeff", C.c_double), ("rcut", C.c_double),
                ("species_mask", C.c_uint64), ("params", C.c_double * 8)]


class SnapParams(C.Structure):
    _fields_ = [("twojmax", C.c_int32), ("nspecies", C.c_int32), ("rcutfac", C.c_double), ("rmin0", C.c_double),
                ("rfac0", C.c_double), ("radii", C.c_double * MAX_SNAP_SPECIES),
                ("weight", C.c_double * MAX_SNAP_SPECIES), ("chem_flag", C.c_int32), ("bzero_flag", C.c_int32),
                ("bnorm_flag", C.c_int32), ("switch_flag", C.c_int32), ("wselfall_flag", C.c_int32),
                ("literal_sqrt_radius", C.c_int32), ("quadratic_flag", C.c_int32), ("literal_chem_z", C.c_int32)]


_lib = None


def lib():
    """Loads libipg.so once.  Raises IPGError when it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise IPGError(-9, f"{LIB_PATH} is missing; build it with interatomicpotentials.jl_b200/build.py")
    L = C.CDLL(LIB_PATH)
    i32, i64, u32, d, vp = C.c_int32, C.c_int64, C.c_uint32, C.c_double, C.c_void_p
    sig = {
        "ipg_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
        "ipg_destroy": (C.c_int, [vp]),
        "ipg_last_error": (C.c_char_p, [vp]),
        "ipg_set_stream": (C.c_int, [vp, vp]),
        "ipg_version": (C.c_int, []),
        "ipg_launch_count": (C.c_int, [vp, C.POINTER(i64)]),
        "ipg_timing_enable": (C.c_int, [vp, C.c_int]),
        "ipg_timing_read": (C.c_int, [vp, C.c_char_p, C.POINTER(d), C.POINTER(i64)]),
        "ipg_neighbor_build": (C.c_int, [vp, i64, vp, vp, vp, i32, vp, i32, C.POINTER(vp)]),
        "ipg_nlist_size": (C.c_int, [vp, C.POINTER(i64)]),
        "ipg_neighbor_count": (C.c_int, [vp, i64, vp, vp, vp, i32, vp, i32, C.POINTER(i64)]),
        "ipg_nlist_export": (C.c_int, [vp, vp, vp, vp]),
        "ipg_nlist_free": (C.c_int, [vp]),
        "ipg_pair_eval": (C.c_int, [vp, i64, vp, vp, vp, vp, i32, vp, vp, vp, u32]),
        "ipg_pair_eval_dev": (C.c_int, [vp, i64, vp, vp, vp, vp, i32, vp, vp, vp, u32]),
        "ipg_pair_eval_noalloc": (C.c_int, [vp, i64, vp, vp, vp, vp, i32, vp, vp, vp, u32]),
        "ipg_snap_create": (C.c_int, [vp, vp, C.POINTER(vp)]),
        "ipg_snap_destroy": (C.c_int, [vp]),
        "ipg_snap_ncoeff": (C.c_int, [vp, C.POINTER(i32)]),
        "ipg_snap_descriptors": (C.c_int, [vp, i64, vp, vp, vp, vp, vp, vp, u32]),
        "ipg_snap_energy_forces": (C.c_int, [vp, i64, vp, vp, vp, vp, d, i32, vp, vp, vp]),
        "ipg_snap_energy_forces_dev": (C.c_int, [vp, i64, vp, vp, vp, vp, d, i32, vp, vp, vp]),
        "ipg_snap_vjp_beta": (C.c_int, [vp, i64, vp, vp, vp, d, vp, vp, vp]),
        "ipg_snap_vjp": (C.c_int, [vp, i64, vp, vp, vp, vp, d, vp, vp, vp, vp]),
        "ipg_snap_autotune": (C.c_int, [vp, i64, vp, vp, vp, vp, C.c_char_p, C.c_char_p, i32]),
        "ipg_snap_batch_descriptors": (C.c_int, [vp, i32, vp, vp, vp, vp, vp, vp, vp]),
        "ipg_snap_set_skin": (C.c_int, [vp, d]),
        "ipg_snap_skin_stats": (C.c_int, [vp, C.POINTER(i64), C.POINTER(i64)]),
        "ipg_snap_batch_energy_forces": (C.c_int, [vp, i32, vp, vp, vp, vp, vp, d, i32, vp, vp, vp]),
        "ipg_snap_batch_energy_forces_dev": (C.c_int, [vp, i32, vp, vp, vp, vp, vp, d, i32, i32, vp, vp, vp]),
        "ipg_snap_batch_loss_grad": (C.c_int, [vp, i32, vp, vp, vp, vp, vp, d, vp, vp, vp]),
        "ipg_snap_batch_loss_grad_dev": (C.c_int, [vp, i32, vp, vp, vp, vp, vp, d, vp, i32, vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status, ctx=None):
    if status != IPG_OK:
        msg = ""
        if ctx is not None:
            m = lib().ipg_last_error(ctx)
            msg = m.decode() if m else ""
        raise IPGError(status, msg)
