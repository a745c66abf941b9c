"""ctypes declarations of the C ABI in ``include/ffs_lbm.h``.

``load()`` opens the in-tree ``libffs_lbm.so`` (built by ``freeflow_b200.build``)
and fails loudly if it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libffs_lbm.so")

FFS_OK = 0
STATUS_NAMES = {0: "ok", 1: "invalid argument", 2: "out of device memory", 3: "CUDA error",
                4: "capacity exceeded", 5: "unsupported"}

STORAGE = {"f32": 0, "fp32": 0, "float32": 0, "f16": 1, "fp16": 1, "float16": 1, "bf16": 2, "bfloat16": 2}
LAYOUT_AOS, LAYOUT_SOA = 0, 1
MEM_HOST, MEM_DEVICE = 0, 1
BUF_CURRENT, BUF_NEXT, BUF_A, BUF_B, BUF_BOTH = 0, 1, 2, 3, 4

STATUS_NONFINITE = 1
STATUS_LINK_OVERFLOW = 2
STATUS_FORCE_RANGE = 4
STATUS_BAD_ELEMENT = 8

# fixed scratch of ffs_lbm_step_noalloc
NOALLOC_MAX_VERTICES = 32768
NOALLOC_MAX_LINK_CELLS = 16384

# every entry point include/ffs_lbm.h declares
EXPORTS = (
    "ffs_lbm_create", "ffs_lbm_destroy", "ffs_lbm_set_flags", "ffs_lbm_get_flags", "ffs_lbm_initialize",
    "ffs_lbm_set_moments", "ffs_lbm_get_moments", "ffs_lbm_reserve_surface", "ffs_lbm_step",
    "ffs_lbm_step_noalloc",
    "ffs_lbm_fill_solid", "ffs_lbm_get_status", "ffs_lbm_get_info", "ffs_lbm_debug_links",
    "ffs_lbm_profile_enable", "ffs_lbm_profile_read",
    "ffs_status_string", "ffs_last_error", "ffs_abi_version",
)


class Profile(C.Structure):
    _fields_ = [("ms", C.c_double * 4), ("launches", C.c_int64 * 4)]


PROFILE_STAGES = ("detect_links", "dense", "link_cells", "finalize_forces")


class LbmDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("fluid_viscosity", C.c_double), ("fluid_density", C.c_double),
        ("fluid_dx", C.c_double), ("dt", C.c_double),
        ("boundary_velocities", C.c_float * 6),
        ("storage", C.c_int), ("periodic_mask", C.c_int), ("ref_half_populations", C.c_int),
    ]


class Surface(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("vertices", C.c_void_p), ("velocities", C.c_void_p), ("elements", C.c_void_p),
        ("num_vertices", C.c_int), ("num_elements", C.c_int),
        ("forces", C.c_void_p), ("forces64", C.c_void_p),
    ]


_LIB = None


class FfsError(RuntimeError):
    pass


def load():
    """Open libffs_lbm.so and declare its signatures (raises if absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise FfsError(f"{LIB_PATH} is missing: build it with `python -m freeflow_b200.build` "
                       "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64 = C.c_void_p, C.c_int, C.c_int64
    sig = {
        "ffs_lbm_create": [C.POINTER(LbmDesc), C.POINTER(vp)],
        "ffs_lbm_destroy": [vp],
        "ffs_lbm_set_flags": [vp, vp, i32, vp],
        "ffs_lbm_get_flags": [vp, vp, i32, vp],
        "ffs_lbm_initialize": [vp, vp],
        "ffs_lbm_set_moments": [vp, vp, i32, i32, i32, vp],
        "ffs_lbm_get_moments": [vp, vp, i32, i32, i32, vp],
        "ffs_lbm_reserve_surface": [vp, i32, i32],
        "ffs_lbm_step": [vp, C.POINTER(Surface), vp],
        "ffs_lbm_step_noalloc": [vp, C.POINTER(Surface), vp],
        "ffs_lbm_fill_solid": [vp, C.POINTER(Surface), vp],
        "ffs_lbm_get_status": [vp, C.POINTER(C.c_uint32), i32, vp],
        "ffs_lbm_get_info": [vp, C.POINTER(i64), C.POINTER(i32), C.POINTER(i32), C.POINTER(C.c_double),
                             C.POINTER(C.c_double)],
        "ffs_lbm_debug_links": [vp, C.POINTER(Surface), vp, vp, i64, C.POINTER(i64), vp],
        "ffs_lbm_profile_enable": [vp, i32],
        "ffs_lbm_profile_read": [vp, C.POINTER(Profile), i32],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = i32
    L.ffs_status_string.argtypes = [i32]
    L.ffs_status_string.restype = C.c_char_p
    L.ffs_last_error.argtypes = []
    L.ffs_last_error.restype = C.c_char_p
    L.ffs_abi_version.argtypes = []
    L.ffs_abi_version.restype = i32
    _LIB = L
    return L


def check(status: int, what: str = "") -> None:
    if status != FFS_OK:
        L = load()
        msg = L.ffs_last_error().decode(errors="replace")
        raise FfsError(f"{what}: {STATUS_NAMES.get(status, status)}: {msg}")
