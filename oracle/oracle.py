"""ctypes wrapper around the CPU oracle (``libffs_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``.  The product path never touches it.

Two builds of the same restatement are exposed:

* ``Oracle(..., precision="ref32")`` follows the reference's FP32 arithmetic
  (op order, double-literal promotions, the binary16 D2Q9 population tile when
  ``half_pops=True``);
* ``Oracle(..., precision="phys64")`` runs the same update in FP64.

The restatement is pinned to the reference's own step: ``ref.py`` runs the
reference's unmodified CUDA sources (built into ``_ref/`` by ``make ref``) on
the GPU, and the GPU tests compare this oracle and the product against it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> str:
    """Compile the oracle with its Makefile; returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "libffs_oracle.so")


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "libffs_oracle.so")
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    vp, i32, f64 = C.c_void_p, C.c_int, C.c_double
    for pre in ("ffo32_", "ffo64_"):
        f = getattr(L, pre + "create")
        f.restype = vp
        f.argtypes = [i32, i32, i32, i32, f64, f64, f64, f64, vp, i32, i32]
        getattr(L, pre + "destroy").argtypes = [vp]
        getattr(L, pre + "set_flags").argtypes = [vp, vp]
        getattr(L, pre + "get_flags").argtypes = [vp, vp]
        getattr(L, pre + "initialize").argtypes = [vp]
        getattr(L, pre + "set_moments").argtypes = [vp, vp, i32]
        getattr(L, pre + "get_moments").argtypes = [vp, vp, i32]
        f = getattr(L, pre + "step")
        f.restype = i32
        f.argtypes = [vp, vp, vp, vp, i32, i32, vp]
        getattr(L, pre + "num_links").restype = C.c_longlong
        getattr(L, pre + "num_links").argtypes = [vp]
        getattr(L, pre + "get_links").argtypes = [vp, vp, vp]
        getattr(L, pre + "get_cf").restype = f64
        getattr(L, pre + "get_cf").argtypes = [vp]
        getattr(L, pre + "get_omega").restype = f64
        getattr(L, pre + "get_omega").argtypes = [vp]
        getattr(L, pre + "fill_solid2").argtypes = [vp, vp, vp, i32]
        getattr(L, pre + "reconstruct").argtypes = [i32, vp, vp, i32]
        getattr(L, pre + "reconstruct_at").restype = f64
        getattr(L, pre + "reconstruct_at").argtypes = [i32, vp, i32]
        getattr(L, pre + "collide_pops").argtypes = [i32, vp, f64, vp]
    L.ffo_fill_solid3.argtypes = [vp, i32, i32, i32, C.c_float, vp, i32, vp, i32]
    L.ffo_inside3_ref.restype = i32
    L.ffo_inside3_ref.argtypes = [vp, vp, i32, C.c_float, C.c_float, C.c_float]
    L.ffo_set_threads.argtypes = [i32]
    L.ffo_get_threads.restype = i32
    L.ffo_round_half.restype = C.c_float
    L.ffo_round_half.argtypes = [C.c_float]
    _LIB = L
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def set_threads(n: int) -> None:
    lib().ffo_set_threads(int(n))


def get_threads() -> int:
    return int(lib().ffo_get_threads())


def reconstruct(dim: int, m, precision="phys64", half_pops=False) -> np.ndarray:
    m = np.ascontiguousarray(m, dtype=np.float64)
    q = 9 if dim == 2 else 27
    out = np.zeros(q, dtype=np.float64)
    pre = "ffo32_" if precision == "ref32" else "ffo64_"
    getattr(lib(), pre + "reconstruct")(dim, _ptr(m), _ptr(out), int(half_pops))
    return out


def reconstruct_at(dim: int, m, i: int, precision="phys64") -> float:
    m = np.ascontiguousarray(m, dtype=np.float64)
    pre = "ffo32_" if precision == "ref32" else "ffo64_"
    return float(getattr(lib(), pre + "reconstruct_at")(dim, _ptr(m), int(i)))


def collide_pops(dim: int, pops, omega: float, precision="phys64") -> np.ndarray:
    p = np.ascontiguousarray(pops, dtype=np.float64)
    out = np.zeros(6 if dim == 2 else 10, dtype=np.float64)
    pre = "ffo32_" if precision == "ref32" else "ffo64_"
    getattr(lib(), pre + "collide_pops")(dim, _ptr(p), float(omega), _ptr(out))
    return out


def fill_solid3(flags, nx: int, ny: int, nz: int, cl: float, vertices, elements) -> np.ndarray:
    """The product's D3Q27 solid fill restated (ffo_fill_solid3): returns the
    new flag array; Fluid/SolidDynamic cells inside the closed triangle mesh
    become SolidDynamic, the others Fluid; every other flag is kept."""
    f = np.array(flags, dtype=np.uint8, copy=True).reshape(-1)
    V = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1)
    E = np.ascontiguousarray(elements, dtype=np.uint32).reshape(-1)
    lib().ffo_fill_solid3(_ptr(f), nx, ny, nz, float(cl), _ptr(V), V.size // 3, _ptr(E), E.size // 3)
    return f


def inside3_ref(vertices, elements, p) -> bool:
    """The reference's SolidGeometryProxy_Device<3>::isInside for one point."""
    V = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1)
    E = np.ascontiguousarray(elements, dtype=np.uint32).reshape(-1)
    return bool(lib().ffo_inside3_ref(_ptr(V), _ptr(E), E.size // 3, float(p[0]), float(p[1]), float(p[2])))


class Oracle:
    """One fluid grid on the CPU, stepped like solveLbmAndFsiStep2D/3D.

    Moments use the reference layout: AoS, x fastest, 6 (D2Q9) or 10 (D3Q27)
    values per cell in the order [rho, ux, uy, pixx, piyy, pixy] /
    [rho, ux, uy, uz, pixx, piyy, pizz, pixy, piyz, pixz].
    """

    def __init__(self, dim, nx, ny, nz=1, viscosity=0.01, density=1000.0, dx=1.0, dt=1.0,
                 boundary_velocities=None, periodic=0, half_pops=False, precision="ref32", wall_stream=False):
        self.dim, self.nx, self.ny = dim, nx, ny
        self.nz = 1 if dim == 2 else nz
        self.nm = 6 if dim == 2 else 10
        self.q = 9 if dim == 2 else 27
        self.pre = "ffo32_" if precision == "ref32" else "ffo64_"
        bc = np.zeros(6, dtype=np.float32)
        if boundary_velocities is not None:
            v = np.asarray(boundary_velocities, dtype=np.float32)
            bc[: len(v)] = v
        L = lib()
        self._h = getattr(L, self.pre + "create")(dim, nx, ny, self.nz, viscosity, density, dx, dt,
                                                  _ptr(bc), int(periodic),
                                                  int(bool(half_pops)) | (int(bool(wall_stream)) << 1))
        if not self._h:
            raise ValueError("invalid grid description")

    def _f(self, name):
        return getattr(lib(), self.pre + name)

    def close(self):
        if self._h:
            self._f("destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ncell(self):
        return self.nx * self.ny * self.nz

    @property
    def cf(self):
        return float(self._f("get_cf")(self._h))

    @property
    def omega(self):
        return float(self._f("get_omega")(self._h))

    def set_flags(self, flags):
        f = np.ascontiguousarray(flags, dtype=np.uint8).reshape(-1)
        assert f.size == self.ncell
        self._f("set_flags")(self._h, _ptr(f))

    def get_flags(self):
        f = np.zeros(self.ncell, dtype=np.uint8)
        self._f("get_flags")(self._h, _ptr(f))
        return f

    def initialize(self):
        self._f("initialize")(self._h)

    def set_moments(self, m, which=4):
        a = np.ascontiguousarray(m, dtype=np.float64).reshape(-1)
        assert a.size == self.ncell * self.nm
        self._f("set_moments")(self._h, _ptr(a), int(which))

    def get_moments(self, which=0):
        a = np.zeros(self.ncell * self.nm, dtype=np.float64)
        self._f("get_moments")(self._h, _ptr(a), int(which))
        return a.reshape(self.ncell, self.nm)

    def step(self, vertices=None, velocities=None, elements=None, forces=None):
        if elements is None or len(elements) == 0:
            self._f("step")(self._h, None, None, None, 0, 0, _ptr(forces) if forces is not None else None)
            return
        V = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1)
        U = np.ascontiguousarray(velocities, dtype=np.float32).reshape(-1)
        E = np.ascontiguousarray(elements, dtype=np.uint32).reshape(-1)
        nv = V.size // self.dim
        ne = E.size // self.dim
        if forces is not None:
            assert forces.dtype == np.float64 and forces.flags.c_contiguous and forces.size == nv * self.dim
        self._f("step")(self._h, _ptr(V), _ptr(U), _ptr(E), nv, ne, _ptr(forces) if forces is not None else None)

    def links(self):
        n = int(self._f("num_links")(self._h))
        cq = np.zeros(n, dtype=np.uint64)
        key = np.zeros(n, dtype=np.uint64)
        if n:
            self._f("get_links")(self._h, _ptr(cq), _ptr(key))
        return cq, key

    def fill_solid(self, vertices, elements):
        V = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1)
        E = np.ascontiguousarray(elements, dtype=np.uint32).reshape(-1)
        self._f("fill_solid2")(self._h, _ptr(V), _ptr(E), E.size // 2)
