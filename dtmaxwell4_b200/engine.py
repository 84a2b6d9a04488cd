"""Python host API over the CUDA engine's C ABI (libdtmx.so, include/dtmx.h).

There is no CPU fallback: if the shared library or a CUDA device is missing,
constructing a Simulation raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdtmx.so")
_lib = None

# every symbol declared in include/dtmx.h
EXPORTS = (
    "dtmx_version", "dtmx_error_string", "dtmx_create", "dtmx_destroy", "dtmx_last_error",
    "dtmx_set_materials", "dtmx_add_point_source", "dtmx_set_tfsf", "dtmx_add_probe",
    "dtmx_read_probes", "dtmx_add_dft_plane", "dtmx_read_dft", "dtmx_step", "dtmx_sync",
    "dtmx_get_step", "dtmx_get_field", "dtmx_set_field", "dtmx_field_device_ptr",
    "dtmx_check_finite", "dtmx_kernel_launches", "dtmx_set_engine", "dtmx_set_xchunk", "dtmx_park", "dtmx_unpark", "dtmx_set_park_pool", "dtmx_plane_state_floats", "dtmx_read_planes", "dtmx_write_planes", "dtmx_copy_planes", "dtmx_set_tile_rows", "dtmx_get_engine", "dtmx_get_stream",
    "dtmx_set_profiling", "dtmx_read_profile", "dtmx_abi_sizes", "dtmx_count_nonfinite_noalloc",
    "dtmx_tfsfsrc_set", "dtmx_ref_main", "dtmx_ref_materials", "dtmx_ref_material_table",
    "dtmx_set_design", "dtmx_forward_adjoint", "dtmx_batch_forward_adjoint", "dtmx_autotune",
    "dtmx_write_arr", "dtmx_save_state", "dtmx_load_state",
    "dtmx_add_dft_patch", "dtmx_add_flux_box", "dtmx_read_flux", "dtmx_flux_faces",
    "dtmx_set_adjoint_memory", "dtmx_ntff", "dtmx_set_wait_limit",
)


class DtmxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("dtmx error %d (%s): %s" % (code, _errstr(code), msg))
        self.code = code


def load():
    """Load libdtmx.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("libdtmx.so not built: run `python -m dtmaxwell4_b200.build` (%s)" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    vp, ip = C.c_void_p, C.c_int
    L.dtmx_version.restype = ip
    L.dtmx_error_string.restype = C.c_char_p
    L.dtmx_error_string.argtypes = [ip]
    L.dtmx_create.argtypes = [C.POINTER(abi.Config), C.POINTER(vp)]
    L.dtmx_destroy.argtypes = [vp]
    L.dtmx_destroy.restype = None
    L.dtmx_last_error.argtypes = [vp]
    L.dtmx_last_error.restype = C.c_char_p
    L.dtmx_set_materials.argtypes = [vp, C.POINTER(abi.Material), ip, vp, vp, vp]
    L.dtmx_add_point_source.argtypes = [vp, C.POINTER(abi.PointSource)]
    L.dtmx_set_tfsf.argtypes = [vp, C.POINTER(abi.TFSF)]
    L.dtmx_add_probe.argtypes = [vp, ip, ip, ip, ip, ip, C.POINTER(ip)]
    L.dtmx_read_probes.argtypes = [vp, vp, ip, C.POINTER(ip)]
    L.dtmx_add_dft_plane.argtypes = [vp, ip, ip, ip, ip, vp, C.POINTER(ip)]
    L.dtmx_read_dft.argtypes = [vp, ip, vp, C.c_size_t]
    L.dtmx_add_dft_patch.argtypes = [vp, ip, ip, ip, ip, ip, ip, ip, ip, vp, C.POINTER(ip)]
    L.dtmx_add_flux_box.argtypes = [vp, C.POINTER(ip), C.POINTER(ip), ip, vp, C.POINTER(ip)]
    L.dtmx_read_flux.argtypes = [vp, ip, vp, C.c_size_t]
    L.dtmx_flux_faces.argtypes = [vp, ip, C.POINTER(ip)]
    L.dtmx_set_adjoint_memory.argtypes = [vp, C.c_int64]
    L.dtmx_ntff.argtypes = [vp, ip, ip, vp, vp, vp, vp, C.c_size_t]
    L.dtmx_step.argtypes = [vp, ip]
    L.dtmx_sync.argtypes = [vp]
    L.dtmx_get_step.argtypes = [vp, C.POINTER(C.c_int64)]
    L.dtmx_get_field.argtypes = [vp, ip, vp]
    L.dtmx_set_field.argtypes = [vp, ip, vp]
    L.dtmx_field_device_ptr.argtypes = [vp, ip, C.POINTER(vp), C.POINTER(C.c_int64)]
    L.dtmx_check_finite.argtypes = [vp]
    L.dtmx_kernel_launches.argtypes = [vp, C.POINTER(C.c_int64)]
    L.dtmx_set_engine.argtypes = [vp, ip, ip]
    L.dtmx_set_xchunk.argtypes = [vp, ip]
    L.dtmx_park.argtypes = [vp]
    L.dtmx_set_park_pool.argtypes = [ip, C.c_int64]
    L.dtmx_plane_state_floats.argtypes = [vp, C.POINTER(C.c_size_t)]
    L.dtmx_read_planes.argtypes = [vp, ip, ip, vp]
    L.dtmx_write_planes.argtypes = [vp, ip, ip, vp]
    L.dtmx_copy_planes.argtypes = [vp, ip, vp, ip, ip]
    L.dtmx_unpark.argtypes = [vp]
    L.dtmx_set_tile_rows.argtypes = [vp, ip]
    L.dtmx_get_engine.argtypes = [vp, C.POINTER(ip), C.POINTER(ip), C.POINTER(ip), C.POINTER(ip)]
    L.dtmx_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.dtmx_set_profiling.argtypes = [vp, ip]
    L.dtmx_read_profile.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    L.dtmx_abi_sizes.argtypes = [C.POINTER(C.c_int64)]
    L.dtmx_set_design.argtypes = [vp, C.POINTER(ip), C.POINTER(ip), vp]
    L.dtmx_forward_adjoint.argtypes = [vp, ip, ip, ip, C.c_double, C.POINTER(C.c_double), vp]
    L.dtmx_write_arr.argtypes = [vp, ip, C.c_char_p]
    L.dtmx_save_state.argtypes = [vp, C.c_char_p]
    L.dtmx_load_state.argtypes = [vp, C.c_char_p]
    L.dtmx_autotune.argtypes = [vp, ip, C.POINTER(ip), C.POINTER(ip), C.POINTER(ip), C.POINTER(C.c_double)]
    L.dtmx_batch_forward_adjoint.argtypes = [C.POINTER(vp), ip, ip, ip, C.POINTER(ip), C.POINTER(C.c_double),
                                             C.POINTER(C.c_double), C.POINTER(vp)]
    L.dtmx_count_nonfinite_noalloc.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int64, C.POINTER(C.c_int64)]
    L.dtmx_set_wait_limit.argtypes = [vp, C.c_int64]
    _lib = L
    return L


def _errstr(code):
    try:
        return load().dtmx_error_string(code).decode()
    except OSError:
        return "?"


class Simulation:
    """One FDTD simulation context on the current CUDA device."""

    def __init__(self, cfg):
        self._L = load()
        self.cfg = cfg
        h = C.c_void_p()
        rc = self._L.dtmx_create(C.byref(cfg), C.byref(h))
        if rc != abi.OK:
            msg = self._L.dtmx_last_error(h).decode() if h.value else ""
            if h.value:
                self._L.dtmx_destroy(h)
            raise DtmxError(rc, msg or "dtmx_create rejected the configuration")
        self._h = h
        self.shape = (cfg.nx, cfg.ny, cfg.nz)
        self._dft = []
        self._flux = []
        self._nprobes = 0
        self.probe_list = []

    def _ck(self, rc):
        if rc != abi.OK:
            raise DtmxError(rc, self._L.dtmx_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.dtmx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- set-up
    def set_materials(self, table, idx_x, idx_y=None, idx_z=None):
        arr = (abi.Material * len(table))(*table)
        keep = [np.ascontiguousarray(a, dtype=np.uint8).reshape(-1) if a is not None else None for a in (idx_x, idx_y, idx_z)]
        for a in keep:
            if a is not None and a.size != self.cfg.nx * self.cfg.ny * self.cfg.nz:
                raise ValueError("material index array has the wrong size")
        ptrs = [a.ctypes.data if a is not None else None for a in keep]
        self._ck(self._L.dtmx_set_materials(self._h, arr, len(table), *ptrs))

    def add_point_source(self, src):
        self._ck(self._L.dtmx_add_point_source(self._h, C.byref(src)))

    def set_tfsf(self, t):
        self._ck(self._L.dtmx_set_tfsf(self._h, C.byref(t)))

    def add_probe(self, comp, i, j, k, mode=abi.PROBE_NODE):
        pid = C.c_int(-1)
        self._ck(self._L.dtmx_add_probe(self._h, comp, i, j, k, mode, C.byref(pid)))
        self._nprobes += 1
        self.probe_list.append((comp, i, j, k, mode))
        return pid.value

    def add_dft_plane(self, axis, index, comp_mask, omegas):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        did = C.c_int(-1)
        self._ck(self._L.dtmx_add_dft_plane(self._h, axis, index, comp_mask, len(om), om.ctypes.data, C.byref(did)))
        n = list(self.shape)
        del n[axis]
        self._dft.append((bin(comp_mask).count("1"), len(om), n[0], n[1]))
        return did.value

    def add_dft_patch(self, axis, index, lo1, n1, lo2, n2, comp_mask, omegas):
        """Running DFT on an n1 x n2 window of the plane {axis = index}."""
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        did = C.c_int(-1)
        self._ck(self._L.dtmx_add_dft_patch(self._h, axis, index, lo1, n1, lo2, n2, comp_mask, len(om),
                                            om.ctypes.data, C.byref(did)))
        self._dft.append((bin(comp_mask).count("1"), len(om), n1, n2))
        return did.value

    def add_flux_box(self, lo, hi, omegas):
        """Six face DFT windows of a power flux box (dtmx_add_flux_box); returns its id."""
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        lo3 = (C.c_int * 3)(*[int(v) for v in lo])
        hi3 = (C.c_int * 3)(*[int(v) for v in hi])
        fid = C.c_int(-1)
        self._ck(self._L.dtmx_add_flux_box(self._h, lo3, hi3, len(om), om.ctypes.data, C.byref(fid)))
        faces = (C.c_int * 6)()
        self._ck(self._L.dtmx_flux_faces(self._h, fid.value, faces))
        for a in range(3):
            n = [hi[q] - lo[q] for q in range(3) if q != a]
            for _ in range(2):
                self._dft.append((4, len(om), n[0], n[1]))              # the face window (flux)
                self._dft.append((4, len(om), n[0] + 1, n[1] + 1))      # far field: E and H of the face plane
                self._dft.append((2, len(om), n[0] + 1, n[1] + 1))      # far field: H one plane further
        self._flux.append((len(om), list(faces)))
        return fid.value

    def flux_faces(self, fid):
        return list(self._flux[fid][1])

    def read_flux(self, fid):
        """(faces[6, nfreq], total[nfreq]): outward FP64 flux of each face and their sum."""
        nf = self._flux[fid][0]
        out = np.zeros(7 * nf, dtype=np.float64)
        self._ck(self._L.dtmx_read_flux(self._h, fid, out.ctypes.data, out.size))
        return out[: 6 * nf].reshape(6, nf), out[6 * nf:]

    def far_field(self, fid, theta, phi, origin=None):
        """Near-to-far-field transform of flux box fid at directions (theta, phi):
        returns (U[ndir, nfreq], E_theta[ndir, nfreq], E_phi[ndir, nfreq]) with
        r E as complex values (exp(-i k r) dropped); see dtmx_ntff."""
        th = np.ascontiguousarray(np.ravel(theta), dtype=np.float64)
        ph = np.ascontiguousarray(np.ravel(phi), dtype=np.float64)
        if th.shape != ph.shape:
            raise ValueError("theta and phi must have the same size")
        nf = self._flux[fid][0]
        out = np.zeros((th.size, nf, 5), dtype=np.float64)
        org = None
        if origin is not None:
            org = np.ascontiguousarray(origin, dtype=np.float64)
        self._ck(self._L.dtmx_ntff(self._h, fid, th.size, th.ctypes.data, ph.ctypes.data,
                                   None if org is None else org.ctypes.data, out.ctypes.data, out.size))
        return out[..., 0], out[..., 1] + 1j * out[..., 2], out[..., 3] + 1j * out[..., 4]

    def set_engine(self, engine, time_block=0):
        self._ck(self._L.dtmx_set_engine(self._h, engine, time_block))

    def park(self):
        """Move the device state to pinned host memory and free the device
        memory (contexts made with make_config(..., parkable=True))."""
        self._ck(self._L.dtmx_park(self._h))

    def unpark(self):
        """Bring a parked context's state back to the device."""
        self._ck(self._L.dtmx_unpark(self._h))

    def plane_state_floats(self):
        """Floats of time-stepping state per x plane (dtmx_plane_state_floats)."""
        n = C.c_size_t(0)
        self._ck(self._L.dtmx_plane_state_floats(self._h, C.byref(n)))
        return n.value

    def read_planes(self, x0, nplanes, out=None):
        """The state of planes [x0, x0 + nplanes) as one float32 array
        (section-major, dtmx_read_planes); out: a buffer to fill (pinned
        memory makes the copies asynchronous to the host)."""
        n = self.plane_state_floats() * int(nplanes)
        if out is None:
            out = np.empty(n, dtype=np.float32)
        if out.dtype != np.float32 or out.size < n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float32 array of %d values" % n)
        self._ck(self._L.dtmx_read_planes(self._h, int(x0), int(nplanes), out.ctypes.data))
        return out[:n]

    def write_planes(self, x0, nplanes, state):
        """Store a read_planes array back into planes [x0, x0 + nplanes)."""
        a = np.ascontiguousarray(state, dtype=np.float32)
        if a.size != self.plane_state_floats() * int(nplanes):
            raise ValueError("plane state of the wrong size")
        self._ck(self._L.dtmx_write_planes(self._h, int(x0), int(nplanes), a.ctypes.data))

    def copy_planes(self, x0, src, src_x0, nplanes):
        """Planes [src_x0, src_x0 + nplanes) of Simulation src into planes
        [x0, ...) of this one, either of them parked (dtmx_copy_planes)."""
        self._ck(self._L.dtmx_copy_planes(self._h, int(x0), src._h, int(src_x0), int(nplanes)))

    def set_xchunk(self, planes):
        """Planes of the x walk per CTA (0: automatic)."""
        self._ck(self._L.dtmx_set_xchunk(self._h, planes))

    def set_tile_rows(self, rows):
        """Tile height of the single-sweep engine (16 or 8; 0: 16)."""
        self._ck(self._L.dtmx_set_tile_rows(self._h, rows))

    def engine_config(self):
        """(engine, time_block, xchunk, tile_rows) that dtmx_step uses."""
        v = [C.c_int() for _ in range(4)]
        self._ck(self._L.dtmx_get_engine(self._h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    # ---- differentiation
    def set_design(self, lo, eps):
        """Per-node permittivity (shape (3, n0, n1, n2)) of the E components
        over the cell box starting at lo."""
        eps = np.ascontiguousarray(eps, dtype=np.float32)
        assert eps.ndim == 4 and eps.shape[0] == 3
        self._design = (tuple(int(v) for v in lo), eps.shape[1:])
        self._ck(self._L.dtmx_set_design(self._h, (C.c_int * 3)(*self._design[0]), (C.c_int * 3)(*eps.shape[1:]),
                                         eps.ctypes.data))

    def forward_adjoint(self, nsteps, plane_x, omega, checkpoint_every=100):
        """Advance nsteps; return (J, dJ/d eps) of the Poynting-flux objective."""
        grad = np.zeros((3,) + tuple(self._design[1]), np.float32)
        J = C.c_double()
        self._ck(self._L.dtmx_forward_adjoint(self._h, int(nsteps), int(checkpoint_every), int(plane_x), float(omega),
                                              C.byref(J), grad.ctypes.data))
        return J.value, grad

    def set_adjoint_memory(self, nbytes):
        """Budget for the recorded design-region history of forward_adjoint
        (0: always checkpoint and recompute; negative: a quarter of free memory)."""
        self._ck(self._L.dtmx_set_adjoint_memory(self._h, int(nbytes)))

    def write_arr(self, comp, path):
        """Field snapshot in the reference's .arr layout (see read_arr)."""
        self._ck(self._L.dtmx_write_arr(self._h, comp, os.fsencode(path)))

    def save_state(self, path):
        self._ck(self._L.dtmx_save_state(self._h, os.fsencode(path)))

    def load_state(self, path):
        self._ck(self._L.dtmx_load_state(self._h, os.fsencode(path)))

    def autotune(self, trial_steps=20):
        """Pick the fastest engine configuration; returns (engine, time_block, xchunk, ms_per_step)."""
        e, t, x, ms = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        self._ck(self._L.dtmx_autotune(self._h, int(trial_steps), C.byref(e), C.byref(t), C.byref(x), C.byref(ms)))
        return e.value, t.value, x.value, ms.value

    # ---- run
    def step(self, n):
        self._ck(self._L.dtmx_step(self._h, int(n)))

    def sync(self):
        self._ck(self._L.dtmx_sync(self._h))

    def set_wait_limit(self, polls):
        """Bound of the device-side waits (polls); <= 0 restores the default."""
        self._ck(self._L.dtmx_set_wait_limit(self._h, int(polls)))

    @property
    def nstep(self):
        v = C.c_int64()
        self._ck(self._L.dtmx_get_step(self._h, C.byref(v)))
        return v.value

    def launches(self):
        v = C.c_int64()
        self._ck(self._L.dtmx_kernel_launches(self._h, C.byref(v)))
        return v.value

    def check_finite(self):
        rc = self._L.dtmx_check_finite(self._h)
        if rc == abi.ERR_NONFINITE:
            return False
        self._ck(rc)
        return True

    # ---- data
    def get_field(self, comp, out=None):
        if out is None:
            out = np.empty(self.shape, dtype=np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.shape == self.shape
        self._ck(self._L.dtmx_get_field(self._h, comp, out.ctypes.data))
        return out

    def set_field(self, comp, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32)
        assert a.shape == self.shape
        self._ck(self._L.dtmx_set_field(self._h, comp, a.ctypes.data))

    def read_probes(self, max_samples=None):
        if max_samples is None:
            max_samples = max(1, self.cfg.probe_capacity or 4096)
        out = np.zeros((max(self._nprobes, 1), max_samples), dtype=np.float32)
        ns = C.c_int(0)
        self._ck(self._L.dtmx_read_probes(self._h, out.ctypes.data, max_samples, C.byref(ns)))
        return out[: self._nprobes, : ns.value]

    def read_dft(self, did):
        ncomp, nf, n1, n2 = self._dft[did]
        out = np.zeros((ncomp, nf, n1, n2, 2), dtype=np.float64)
        self._ck(self._L.dtmx_read_dft(self._h, did, out.ctypes.data, out.size))
        return out[..., 0] + 1j * out[..., 1]

    def stream_handle(self):
        """cudaStream_t of the context (for torch.cuda.ExternalStream)."""
        v = C.c_void_p()
        self._ck(self._L.dtmx_get_stream(self._h, C.byref(v)))
        return v.value

    def device_ptr(self, comp):
        """(device address, element strides (x, y, z)) of a field component."""
        p = C.c_void_p()
        st = (C.c_int64 * 3)()
        self._ck(self._L.dtmx_field_device_ptr(self._h, comp, C.byref(p), st))
        return p.value, (st[0], st[1], st[2])

    def set_profiling(self, on=True):
        self._ck(self._L.dtmx_set_profiling(self._h, 1 if on else 0))

    def read_profile(self):
        a, b, n = C.c_double(), C.c_double(), C.c_int64()
        self._ck(self._L.dtmx_read_profile(self._h, C.byref(a), C.byref(b), C.byref(n)))
        return a.value, b.value, n.value


def set_park_pool(nbytes, device=0):
    """Keep up to nbytes (< 0: no limit, 0: none) of the device memory that
    parking releases on CUDA device `device`, for the next unpark of a block
    of the same size (dtmx_set_park_pool)."""
    L = load()
    rc = L.dtmx_set_park_pool(int(device), int(nbytes))
    if rc:
        raise DtmxError(rc, "dtmx_set_park_pool")


def batch_forward_adjoint(sims, nsteps, plane_x, omega, checkpoint_every=100):
    """dtmx_batch_forward_adjoint over Simulations that have design regions:
    returns ([J], [dJ/d eps])."""
    L = load()
    n = len(sims)
    grads = [np.zeros((3,) + tuple(s._design[1]), np.float32) for s in sims]
    hs = (C.c_void_p * n)(*[s._h for s in sims])
    px = (C.c_int * n)(*[int(v) for v in plane_x])
    om = (C.c_double * n)(*[float(v) for v in omega])
    J = (C.c_double * n)()
    gp = (C.c_void_p * n)(*[g.ctypes.data for g in grads])
    rc = L.dtmx_batch_forward_adjoint(hs, n, int(nsteps), int(checkpoint_every), px, om, J, gp)
    if rc != 0:
        msgs = [L.dtmx_last_error(s._h).decode() for s in sims]
        raise DtmxError(rc, "; ".join(m for m in msgs if m))
    return list(J), grads


def read_arr(path):
    """Read an .arr file (int32 header {12, 0, 0, 0, dim, elsize, n_fastest, ..})
    into an array indexed [x, y, z]."""
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(4), np.int32)
        comment = f.read(int(hdr[0]))
        dim, es = np.frombuffer(f.read(8), np.int32)
        ext = np.frombuffer(f.read(4 * int(dim)), np.int32)
        data = np.frombuffer(f.read(), np.float32 if es == 4 else np.float64)
    del comment
    return data.reshape(tuple(int(v) for v in ext[::-1]))


def abi_sizes():
    out = (C.c_int64 * 6)()
    load().dtmx_abi_sizes(out)
    return tuple(out)


def count_nonfinite_noalloc(device_ptrs, nelem):
    """NaN/Inf count over caller-owned device float arrays, allocating no
    device memory (see dtmx_count_nonfinite_noalloc in include/dtmx.h).
    Returns (status, count)."""
    arr = (C.c_void_p * len(device_ptrs))(*device_ptrs)
    out = C.c_int64(-1)
    rc = load().dtmx_count_nonfinite_noalloc(arr, len(device_ptrs), int(nelem), C.byref(out))
    return rc, out.value
