"""dtmaxwell4_b200 -- B200-native FDTD engine for the DTmaxwell4 leapfrog E/H path.

The compute path is hand-written sm_100a CUDA behind a C ABI (include/dtmx.h,
libdtmx.so); this package is the Python host side: ctypes structs (abi),
the Simulation wrapper (engine), scenario builders (scenarios) and the
DTmxw drop-in module mirroring the reference's SWIG surface (DTmxw).
"""
from . import abi
from .engine import Simulation, DtmxError, load, LIB_PATH, EXPORTS

__all__ = ["abi", "Simulation", "DtmxError", "load", "LIB_PATH", "EXPORTS"]
