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

# every entry point include/ffs_lbm.h and include/ffs_pool.h declare
EXPORTS = (
    "ffs_lbm_create", "ffs_lbm_destroy", "ffs_lbm_set_flags", "ffs_lbm_get_flags", "ffs_lbm_initialize",
    "ffs_lbm_set_moments", "ffs_lbm_get_moments", "ffs_lbm_reserve_surface", "ffs_lbm_step",
    "ffs_lbm_step_noalloc", "ffs_lbm_step_coupled",
    "ffs_lbm_fill_solid", "ffs_lbm_get_status", "ffs_lbm_get_info", "ffs_lbm_debug_links",
    "ffs_lbm_profile_enable", "ffs_lbm_profile_read",
    "ffs_status_string", "ffs_last_error", "ffs_abi_version",
    "ffs_pool_create", "ffs_pool_destroy", "ffs_pool_episode_bytes", "ffs_pool_admit", "ffs_pool_evict",
    "ffs_pool_set_action", "ffs_pool_set_actions", "ffs_pool_advance", "ffs_pool_collect", "ffs_pool_collect_many",
    "ffs_pool_get_moments", "ffs_pool_tune",
    "ffs_pool_get_info", "ffs_swimmer_surface",
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
        ("ref_2d_wall_stream", C.c_int),
    ]


class Surface(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("vertices", C.c_void_p), ("velocities", C.c_void_p), ("elements", C.c_void_p),
        ("num_vertices", C.c_int), ("num_elements", C.c_int),
        ("forces", C.c_void_p), ("forces64", C.c_void_p),
    ]


class VolumeSurface(C.Structure):
    """ffs_volume_surface: a surface given through its volume mesh's arrays and the
    surface-to-volume vertex map."""
    _fields_ = [
        ("dim", C.c_int), ("num_volume_vertices", C.c_int),
        ("volume_positions", C.c_void_p), ("volume_velocities", C.c_void_p), ("volume_forces", C.c_void_p),
        ("num_vertices", C.c_int), ("num_elements", C.c_int),
        ("surface_to_volume", C.c_void_p), ("elements", C.c_void_p),
        ("surface_positions", C.c_void_p), ("surface_velocities", C.c_void_p),
    ]


class PoolDesc(C.Structure):
    _fields_ = [("storage", C.c_int), ("budget_bytes", C.c_int64), ("max_episodes", C.c_int),
                ("substeps", C.c_int), ("num_actions", C.c_int), ("max_link_cells", C.c_int),
                ("stream", C.c_void_p)]


class Swimmer(C.Structure):
    _fields_ = [("num_vertices", C.c_int), ("num_elements", C.c_int),
                ("rest", C.c_void_p), ("elements", C.c_void_p), ("amplitude", C.c_void_p),
                ("sin_kx", C.c_void_p), ("cos_kx", C.c_void_p), ("segment", C.c_void_p),
                ("omega", C.c_double), ("t0", C.c_double)]


class EpisodeDesc(C.Structure):
    _fields_ = [("grid", LbmDesc), ("flags", C.c_void_p), ("swimmer", Swimmer)]


class PoolOutput(C.Structure):
    _fields_ = [("energy", C.c_double), ("force", C.c_double * 2), ("torque", C.c_double),
                ("status", C.c_uint32), ("pad", C.c_uint32)]


class PoolInfo(C.Structure):
    _fields_ = [("budget_bytes", C.c_int64), ("free_bytes", C.c_int64), ("largest_free_bytes", C.c_int64),
                ("active_episodes", C.c_int), ("tiles", C.c_int), ("tile_x", C.c_int), ("tile_y", C.c_int),
                ("advances", C.c_int64), ("graph_builds", C.c_int64), ("cells", C.c_int64),
                ("tuned_cells", C.c_int64), ("dense_ms", C.c_double), ("strip", C.c_int), ("pad", C.c_int)]


POOL_MAX_ACTIONS = 16
POOL_MAX_SUBSTEPS = 64

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
        "ffs_lbm_step_coupled": [vp, C.POINTER(VolumeSurface), vp],
        "ffs_lbm_fill_solid": [vp, C.POINTER(Surface), vp],
        "ffs_lbm_get_status": [vp, C.POINTER(C.c_uint32), i32, vp],
        "ffs_lbm_get_info": [vp, C.POINTER(i64), C.POINTER(i32), C.POINTER(i32), C.POINTER(C.c_double),
                             C.POINTER(C.c_double)],
        "ffs_lbm_debug_links": [vp, C.POINTER(Surface), vp, vp, i64, C.POINTER(i64), vp],
        "ffs_lbm_profile_enable": [vp, i32],
        "ffs_lbm_profile_read": [vp, C.POINTER(Profile), i32],
        "ffs_pool_create": [C.POINTER(PoolDesc), C.POINTER(vp)],
        "ffs_pool_destroy": [vp],
        "ffs_pool_episode_bytes": [vp, C.POINTER(EpisodeDesc), C.POINTER(i64)],
        "ffs_pool_admit": [vp, C.POINTER(EpisodeDesc), C.POINTER(i32)],
        "ffs_pool_evict": [vp, i32],
        "ffs_pool_set_action": [vp, i32, vp, i32],
        "ffs_pool_set_actions": [vp, i32, vp, vp],
        "ffs_pool_collect_many": [vp, i32, vp, vp],
        "ffs_pool_advance": [vp],
        "ffs_pool_collect": [vp, i32, C.POINTER(PoolOutput), vp],
        "ffs_pool_get_moments": [vp, i32, vp],
        "ffs_pool_tune": [vp],
        "ffs_pool_get_info": [vp, C.POINTER(PoolInfo)],
        "ffs_swimmer_surface": [C.POINTER(Swimmer), vp, i32, i64, C.c_double, vp, vp],
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
