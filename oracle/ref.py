"""ctypes wrapper around the reference's own fluid step (``_ref/libffs_ref.so``).

TEST INFRASTRUCTURE ONLY, like ``oracle.py``: the GPU tests run it next to the
product to pin both the product and the CPU restatement to the reference.

The library is the reference's unmodified ``FsiCoupling2D/3D.cu``,
``LbmUtilsFunc.cu``, ``LbmConstants.cu`` and ``LbmFlowField2D/3D.cpp``,
compiled for sm_100a by ``make ref`` in this directory (stand-in headers in
``ref_shim/``), so it needs a GPU.  ``RefStep`` mirrors ``Oracle``: moments
in the reference's AoS layout, ``step(vertices, velocities, elements,
forces)`` with float64 ``forces`` accumulated (+=).  The reference has no
periodic axes and no per-grid inlet velocities (inlet nodes keep their
initial moments), so neither is a parameter.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libffs_ref.so")
_LIB = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        L = C.CDLL(LIB_PATH)
        vp, i32, f64 = C.c_void_p, C.c_int, C.c_double
        L.ffr_create.restype = vp
        L.ffr_create.argtypes = [i32, i32, i32, i32, f64, f64, f64, f64]
        L.ffr_destroy.argtypes = [vp]
        L.ffr_set_flags.argtypes = [vp, vp]
        L.ffr_set_moments.argtypes = [vp, vp]
        L.ffr_get_moments.argtypes = [vp, vp]
        L.ffr_step.argtypes = [vp, vp, vp, vp, i32, i32, vp]
        L.ffr_get_hits.argtypes = [vp, vp]
        L.ffr_last_error.restype = C.c_char_p
        _LIB = L
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class RefStep:
    """One flow field of the reference (LbmFlowField2D/3D) stepped by its own
    solveLbmAndFsiStep2D/3D sequence."""

    def __init__(self, dim, nx, ny, nz=1, viscosity=0.01, density=1000.0, dx=1.0, dt=1.0):
        self.dim, self.nx, self.ny, self.nz = dim, nx, ny, (1 if dim == 2 else nz)
        self.nm = 6 if dim == 2 else 10
        self._h = lib().ffr_create(dim, nx, ny, self.nz, viscosity, density, dx, dt)
        if not self._h:
            raise RuntimeError("reference flow field: " + lib().ffr_last_error().decode())

    @property
    def ncell(self):
        return self.nx * self.ny * self.nz

    def _ck(self, rc, what):
        if rc:
            raise RuntimeError(f"reference {what}: " + lib().ffr_last_error().decode())

    def close(self):
        if self._h:
            lib().ffr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_flags(self, flags):
        f = np.ascontiguousarray(flags, dtype=np.uint8).reshape(-1)
        assert f.size == self.ncell
        self._ck(lib().ffr_set_flags(self._h, _ptr(f)), "set_flags")

    def set_moments(self, m):
        a = np.ascontiguousarray(m, dtype=np.float32).reshape(-1)
        assert a.size == self.ncell * self.nm
        self._ck(lib().ffr_set_moments(self._h, _ptr(a)), "set_moments")

    def get_moments(self):
        a = np.zeros(self.ncell * self.nm, dtype=np.float32)
        self._ck(lib().ffr_get_moments(self._h, _ptr(a)), "get_moments")
        return a.reshape(self.ncell, self.nm).astype(np.float64)

    def hits(self):
        """The reference's hit index of the last step, (ncell, Q) uint32
        (0xFFFFFFFF: no link; else depth_q16 << 16 | element)."""
        q = 9 if self.dim == 2 else 27
        a = np.zeros(self.ncell * q, dtype=np.uint32)
        self._ck(lib().ffr_get_hits(self._h, _ptr(a)), "get_hits")
        return a.reshape(self.ncell, q)

    def step(self, vertices=None, velocities=None, elements=None, forces=None):
        if elements is None or len(elements) == 0:
            self._ck(lib().ffr_step(self._h, None, None, None, 0, 0, None), "step")
            return
        V = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1)
        U = np.ascontiguousarray(velocities, dtype=np.float32).reshape(-1)
        E = np.ascontiguousarray(elements, dtype=np.uint32).reshape(-1)
        F = np.zeros(V.size, dtype=np.float32)
        self._ck(lib().ffr_step(self._h, _ptr(V), _ptr(U), _ptr(E), V.size // self.dim, E.size // self.dim,
                                _ptr(F)), "step")
        if forces is not None:
            forces += F.astype(np.float64)
