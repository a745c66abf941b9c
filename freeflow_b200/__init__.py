"""freeflow_b200 -- B200-native moment-encoded LBM fluid step of FreeFlow.

The product is ``libffs_lbm.so`` (hand-written sm_100a CUDA behind the C ABI in
``include/ffs_lbm.h``).  This package holds its build recipe, the ctypes
binding, and host-side mirrors of the reference's Python interface.
"""
from . import _capi
from ._capi import FfsError, load
from .grid import DeviceSurface, FluidGrid, VolumeSurface

__all__ = ["FluidGrid", "DeviceSurface", "VolumeSurface", "FfsError", "load", "_capi"]
