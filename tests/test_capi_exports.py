"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU)."""
import ctypes
import os
import re

from freeflow_b200 import _capi
from freeflow_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = set()
    for h in ("ffs_lbm.h", "ffs_pool.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(ffs_\w+)\s*\(", src))
    return sorted(names)


def test_library_builds_and_loads():
    path = B.build()
    assert os.path.exists(path)
    lib = ctypes.CDLL(path)
    assert lib is not None


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(B.build())
    names = declared_entry_points()
    assert names, "no entry points found in the header"
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_capi.EXPORTS) == names


def test_abi_version_and_status_strings():
    L = _capi.load()
    assert L.ffs_abi_version() == 4
    assert L.ffs_status_string(0) == b"ok"
    assert L.ffs_status_string(1) == b"invalid argument"


def test_invalid_descriptor_is_rejected_without_gpu_work():
    L = _capi.load()
    d = _capi.LbmDesc()
    d.dim = 4
    h = ctypes.c_void_p()
    assert L.ffs_lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1
    assert b"dim" in L.ffs_last_error()
    assert L.ffs_lbm_create(None, ctypes.byref(h)) == 1


def test_oversized_and_malformed_grids_are_rejected_before_any_device_work():
    L = _capi.load()
    h = ctypes.c_void_p()
    d = _capi.LbmDesc()
    d.dim, d.nx, d.ny, d.nz = 3, 2048, 2048, 1024       # 2^32 cells
    d.fluid_viscosity, d.fluid_dx, d.dt = 0.01, 1.0, 1.0
    assert L.ffs_lbm_create(ctypes.byref(d), ctypes.byref(h)) == 5   # FFS_ERR_UNSUPPORTED
    assert b"2^31" in L.ffs_last_error()
    d.nx = 0
    assert L.ffs_lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d.nx, d.nz, d.fluid_viscosity = 8, 8, 0.0
    assert L.ffs_lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d.fluid_viscosity, d.storage = 0.01, 7
    assert L.ffs_lbm_create(ctypes.byref(d), ctypes.byref(h)) == 1


def test_pool_descriptor_checks_need_no_device():
    L = _capi.load()
    h = ctypes.c_void_p()
    d = _capi.PoolDesc()
    d.storage, d.budget_bytes, d.max_episodes, d.substeps, d.num_actions = 1, 1 << 20, 0, 10, 8
    assert L.ffs_pool_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d.max_episodes, d.substeps = 4, 65
    assert L.ffs_pool_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d.substeps, d.num_actions = 10, 17
    assert L.ffs_pool_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d.num_actions, d.budget_bytes = 8, 0
    assert L.ffs_pool_create(ctypes.byref(d), ctypes.byref(h)) == 1


def test_step_entry_points_reject_null_arguments_without_device_work():
    L = _capi.load()
    vs = _capi.VolumeSurface()
    s = _capi.Surface()
    assert L.ffs_lbm_step_coupled(None, ctypes.byref(vs), None) == 1
    assert b"null" in L.ffs_last_error()
    assert L.ffs_lbm_step(None, ctypes.byref(s), None) == 1
    assert L.ffs_lbm_step_noalloc(None, ctypes.byref(s), None) == 1


def test_ctypes_structs_match_the_c_header(tmp_path):
    """The ctypes mirrors of the ABI structs have the C layout: a C program built
    against include/ffs_lbm.h and include/ffs_pool.h prints sizeof and every
    field's offsetof."""
    import shutil
    import subprocess

    import pytest

    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    structs = {"ffs_surface": _capi.Surface, "ffs_volume_surface": _capi.VolumeSurface, "ffs_lbm_desc": _capi.LbmDesc,
               "ffs_profile": _capi.Profile, "ffs_pool_desc": _capi.PoolDesc, "ffs_swimmer": _capi.Swimmer,
               "ffs_episode_desc": _capi.EpisodeDesc, "ffs_pool_output": _capi.PoolOutput,
               "ffs_pool_info": _capi.PoolInfo}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "ffs_lbm.h"', '#include "ffs_pool.h"',
             "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = str(tmp_path / "layout")
    r = subprocess.run(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "include"), str(src), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = dict(line.split() for line in subprocess.run([exe], capture_output=True, text=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, f"{cname}.{fname}"


def test_volume_surface_struct_plumbing_on_the_host():
    """VolumeSurface fills every ffs_volume_surface field from its tensors (built on
    the CPU here; no library call is made)."""
    import numpy as np

    from freeflow_b200 import VolumeSurface

    rng = np.random.default_rng(0)
    vp = rng.standard_normal((10, 3)).astype(np.float32)
    vv = rng.standard_normal((10, 3)).astype(np.float32)
    smap = np.array([7, 2, 5, 0], np.uint32)
    elems = np.array([[0, 1, 2], [1, 2, 3]], np.uint32)
    vs = VolumeSurface(vp, vv, smap, elems, device="cpu")
    s = vs.c_struct()
    assert (s.dim, s.num_volume_vertices, s.num_vertices, s.num_elements) == (3, 10, 4, 2)
    for name in ("volume_positions", "volume_velocities", "volume_forces", "surface_to_volume", "elements",
                 "surface_positions", "surface_velocities"):
        assert getattr(s, name), name
    assert s.volume_positions == vs.volume_positions.data_ptr()
    assert np.array_equal(vs.surface_to_volume.numpy().view(np.uint32), smap)
    assert vs.surface_positions.shape == (4, 3) and vs.volume_forces.shape == (10, 3)
    moved = vp + 1.0
    vs.update(moved, None)
    assert np.array_equal(vs.volume_positions.numpy(), moved) and np.array_equal(vs.volume_velocities.numpy(), vv)
    assert not np.array_equal(vp, moved)          # the caller's array is not aliased
