"""Drop-in for the reference's SWIG module ``DTmxw`` (mxw.i:1-36).

Same surface as the SWIG build: ``cvar`` holds the run constants
(``GridNx/GridNy/GridNz``, ``ds, da, dv, dt``, ``Np``, ``NyBloch``,
``Npmlx/Npmly/Npmlz``, ``Tsteps``) and the ``shotpoint`` (a ``TFSFsrc`` with
the reference's field names and ``set(c, imp, lmb)`` / ``check()``);
``_main(argv)`` runs the headless driver.  The reference's ``run.py`` works
unchanged with ``sys.modules['DTmxw']`` pointing at this module.

Unlike the SWIG build, the grid is not fixed at compile time: ``Np, Na, Nv``
(rags along x, y and cells along z), ``Ns`` and ``Ntime`` are attributes of
``cvar`` and ``GridNx = 3 Np``, ``GridNy = 3 Na``, ``GridNz = Nv`` follow them.
"""
import ctypes as C
import math
import struct

from . import engine


def _ftype(v):
    """A value stored in one of the reference's ftype (float) variables."""
    return struct.unpack("f", struct.pack("f", float(v)))[0]


class TFSFsrc(C.Structure):
    """TFSFsrc (py_consts.h:73-91) -- the dipole shotpoint.  Its real fields
    are the reference's ftype (float): an assignment, and TFSFsrc::set, round
    the value to float as the SWIG-wrapped struct does."""
    _fields_ = [
        ("tStop", C.c_double),
        ("srcXs", C.c_double), ("srcXa", C.c_double), ("srcXv", C.c_double), ("sphR", C.c_double),
        ("BoxMs", C.c_double), ("BoxPs", C.c_double), ("BoxMa", C.c_double), ("BoxPa", C.c_double),
        ("BoxMv", C.c_double), ("BoxPv", C.c_double),
        ("V_max", C.c_double),
        ("start", C.c_int),
        ("wavelength", C.c_double), ("w", C.c_double), ("k", C.c_double), ("Omega", C.c_double),
        ("kEnv", C.c_double), ("theta", C.c_double), ("phi", C.c_double),
        ("cSrc", C.c_double), ("Imp", C.c_double),
        ("t0", C.c_double), ("tw", C.c_double), ("T", C.c_double),
    ]

    def __setattr__(self, name, value):
        if name in _REAL_FIELDS:
            value = _ftype(value)
        super().__setattr__(name, value)

    def set(self, c, imp, lmb):
        """TFSFsrc::set (signal.hpp:99-115)."""
        L = engine.load()
        L.dtmx_tfsfsrc_set.restype = None
        L.dtmx_tfsfsrc_set.argtypes = [C.POINTER(TFSFsrc), C.c_double, C.c_double, C.c_double]
        L.dtmx_tfsfsrc_set(C.byref(self), c, imp, lmb)
        for name in _REAL_FIELDS:
            setattr(self, name, getattr(self, name))

    def check(self):
        """TFSFsrc::check (signal.hpp:116-133); the shotpoint line prints srcXv
        twice, as the reference does."""
        print("TF/SF source: Box(s,v,a) |%g-%g|x|%g-%g|x|%g-%g|" % (self.BoxMs, self.BoxPs, self.BoxMv, self.BoxPv,
                                                                   self.BoxMa, self.BoxPa))
        print("TF/SF source: Shotpoint(s,v,a) = %g,%g,%g" % (self.srcXs, self.srcXv, self.srcXv))
        print("TF/SF source: wavelength = %g, kEnv=%g, tStop=%g" % (self.wavelength, self.kEnv, self.tStop))
        print("TF/SF stops after %d steps" % int(self.tStop / cvar.dt))


_REAL_FIELDS = tuple(n for n, t in TFSFsrc._fields_ if t is C.c_double)


class RefGlobals(C.Structure):
    _fields_ = [("Np", C.c_int), ("Na", C.c_int), ("Nv", C.c_int), ("Ns", C.c_int), ("Ntime", C.c_int),
                ("ds", C.c_double), ("da", C.c_double), ("dv", C.c_double), ("dt", C.c_double),
                ("Tsteps", C.c_int), ("Npmlx", C.c_int), ("Npmly", C.c_int), ("Npmlz", C.c_int)]


class _CVar:
    """Module globals of the SWIG build (``DTmxw.cvar``)."""

    def __init__(self):
        # py_consts.h defaults: 600 x 300 x 640 cells, window of 25 rags
        self.Np, self.Na, self.Nv = 200, 100, 640
        self.Ns = 25
        self.Ntime = self.Ns - 3                 # params.h:50-52
        self.NyBloch = 1
        self.Npmlx, self.Npmly, self.Npmlz = 10, 10, 32
        # const ftype ds=0.005, da, dv, dt=0.002 (py_consts.h:71): float values
        self.ds = self.da = self.dv = _ftype(0.005)
        self.dt = _ftype(0.002)
        self.Tsteps = self.Ntime * 10             # DTmxw.cu:730
        self.shotpoint = TFSFsrc()

    @property
    def GridNx(self):
        return 3 * self.Np

    @property
    def GridNy(self):
        return 3 * self.Na

    @property
    def GridNz(self):
        return self.Nv

    def globals(self):
        return RefGlobals(self.Np, self.Na, self.Nv, self.Ns, self.Ntime, self.ds, self.da, self.dv, self.dt,
                          int(self.Tsteps), int(self.Npmlx), int(self.Npmly), int(self.Npmlz))


cvar = _CVar()


def _main(argv):
    """Headless _main (DTmxw.cu:731-834): argv as the SWIG typemap receives it."""
    L = engine.load()
    L.dtmx_ref_main.argtypes = [C.POINTER(RefGlobals), C.POINTER(TFSFsrc), C.c_int, C.POINTER(C.c_char_p)]
    L.dtmx_ref_main.restype = C.c_int
    args = [str(a).encode() for a in argv]
    arr = (C.c_char_p * (len(args) + 1))(*args, None)
    g = cvar.globals()
    return L.dtmx_ref_main(C.byref(g), C.byref(cvar.shotpoint), len(args), arr)


def reference_materials(g=None):
    """Material table and per-E-component index arrays of the reference geometry."""
    import numpy as np
    from . import abi
    g = g or cvar.globals()
    L = engine.load()
    L.dtmx_ref_materials.argtypes = [C.POINTER(RefGlobals), C.c_void_p, C.c_void_p, C.c_void_p]
    L.dtmx_ref_material_table.argtypes = [C.POINTER(abi.Material), C.c_int]
    shape = (3 * g.Np, 3 * g.Na, g.Nv)
    idx = [np.zeros(shape, np.uint8) for _ in range(3)]
    L.dtmx_ref_materials(C.byref(g), idx[0].ctypes.data, idx[1].ctypes.data, idx[2].ctypes.data)
    tab = (abi.Material * 8)()
    n = L.dtmx_ref_material_table(tab, 8)
    return list(tab[:n]), idx
