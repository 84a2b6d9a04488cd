"""ctypes binding of the CPU oracle (oracle/fdtd_oracle.c).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py.  The product package never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from dtmaxwell4_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        for pfx in ("orc64_", "orc32_"):
            g = lambda n: getattr(L, pfx + n)
            g("create").restype = C.c_void_p
            g("create").argtypes = [C.POINTER(abi.Config)]
            g("destroy").argtypes = [C.c_void_p]
            g("set_materials").argtypes = [C.c_void_p, C.POINTER(abi.Material), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
            g("add_point_source").argtypes = [C.c_void_p, C.POINTER(abi.PointSource)]
            g("set_tfsf").argtypes = [C.c_void_p, C.POINTER(abi.TFSF)]
            g("add_probe").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
            g("add_dft_plane").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
            g("step").argtypes = [C.c_void_p, C.c_int]
            g("get_field").argtypes = [C.c_void_p, C.c_int, C.c_void_p]
            g("set_field").argtypes = [C.c_void_p, C.c_int, C.c_void_p]
            g("read_probes").argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
            g("read_dft").argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
            g("set_design").argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p]
            g("plane_state_floats").restype = C.c_size_t
            g("plane_state_floats").argtypes = [C.c_void_p]
            g("read_planes").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
            g("write_planes").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
            g("forward_adjoint").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_double),
                                             C.c_void_p]
        _lib = L
    return _lib


class OracleSim:
    """Same call surface as dtmaxwell4_b200.Simulation, on the CPU oracle."""

    def __init__(self, cfg, precision="f64"):
        self._p = "orc64_" if precision == "f64" else "orc32_"
        self._L = lib()
        self.cfg = cfg
        self._h = self._f("create")(C.byref(cfg))
        if not self._h:
            raise ValueError("oracle rejected the configuration")
        self.shape = (cfg.nx, cfg.ny, cfg.nz)
        self._dft = []
        self._nprobes = 0

    def _f(self, n):
        return getattr(self._L, self._p + n)

    def close(self):
        if self._h:
            self._f("destroy")(self._h)
            self._h = None

    __del__ = close

    def set_materials(self, table, idx_x, idx_y=None, idx_z=None):
        arr = (abi.Material * len(table))(*table)
        keep = [np.ascontiguousarray(a, dtype=np.uint8) if a is not None else None for a in (idx_x, idx_y, idx_z)]
        ptrs = [a.ctypes.data if a is not None else None for a in keep]
        rc = self._f("set_materials")(self._h, arr, len(table), *ptrs)
        if rc:
            raise ValueError("set_materials rc=%d" % rc)

    def add_point_source(self, src):
        self._f("add_point_source")(self._h, C.byref(src))

    def set_tfsf(self, t):
        self._f("set_tfsf")(self._h, C.byref(t))

    def add_probe(self, comp, i, j, k, mode=abi.PROBE_NODE):
        pid = self._f("add_probe")(self._h, comp, i, j, k, mode)
        if pid < 0:
            raise ValueError("add_probe failed")
        self._nprobes += 1
        return pid

    def add_dft_plane(self, axis, index, comp_mask, omegas):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        did = self._f("add_dft_plane")(self._h, axis, index, comp_mask, len(om), om.ctypes.data)
        if did < 0:
            raise ValueError("oracle: too many DFT planes")
        n = list(self.shape)
        del n[axis]
        ncomp = bin(comp_mask).count("1")
        self._dft.append((ncomp, len(om), n[0], n[1]))
        return did

    def step(self, n):
        self._f("step")(self._h, int(n))

    def set_design(self, lo, eps):
        """Per-node permittivity of the three E components over the cell box
        starting at lo; eps has shape (3, n0, n1, n2)."""
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        self._design = (tuple(lo), eps.shape[1:])
        lo_c = (C.c_int * 3)(*lo)
        n_c = (C.c_int * 3)(*eps.shape[1:])
        if self._f("set_design")(self._h, lo_c, n_c, eps.ctypes.data) != 0:
            raise ValueError("bad design region")

    def forward_adjoint(self, nsteps, plane_x, omega):
        """Run nsteps forward, return (J, dJ/d eps) for the Poynting flux
        through the plane x = plane_x at omega (discrete adjoint, FP64)."""
        shape = self._design[1]
        grad = np.zeros((3,) + tuple(shape), np.float64)
        J = C.c_double()
        rc = self._f("forward_adjoint")(self._h, int(nsteps), int(plane_x), float(omega), C.byref(J), grad.ctypes.data)
        if rc != 0:
            raise ValueError("forward_adjoint failed: %d" % rc)
        return J.value, grad

    def get_field(self, comp):
        out = np.empty(self.shape, dtype=np.float64)
        self._f("get_field")(self._h, comp, out.ctypes.data)
        return out

    def set_field(self, comp, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self._f("set_field")(self._h, comp, a.ctypes.data)

    def plane_state_floats(self):
        return int(self._f("plane_state_floats")(self._h))

    def read_planes(self, x0, nplanes, out=None):
        out = np.empty(self.plane_state_floats() * int(nplanes), dtype=np.float64)
        rc = self._f("read_planes")(self._h, int(x0), int(nplanes), out.ctypes.data)
        if rc:
            raise ValueError("read_planes rc=%d" % rc)
        return out

    def write_planes(self, x0, nplanes, state):
        a = np.ascontiguousarray(state, dtype=np.float64)
        if a.size != self.plane_state_floats() * int(nplanes):
            raise ValueError("plane state of the wrong size")
        rc = self._f("write_planes")(self._h, int(x0), int(nplanes), a.ctypes.data)
        if rc:
            raise ValueError("write_planes rc=%d" % rc)

    def read_probes(self, max_samples=100000):
        out = np.zeros((max(self._nprobes, 1), max_samples), dtype=np.float64)
        ns = C.c_int(0)
        self._f("read_probes")(self._h, out.ctypes.data, max_samples, C.byref(ns))
        return out[: self._nprobes, : ns.value]

    def read_dft(self, did):
        ncomp, nf, n1, n2 = self._dft[did]
        out = np.zeros((ncomp, nf, n1, n2, 2), dtype=np.float64)
        rc = self._f("read_dft")(self._h, did, out.ctypes.data, out.size)
        if rc:
            raise ValueError("read_dft rc=%d" % rc)
        return out[..., 0] + 1j * out[..., 1]


def threads():
    return lib().orc64_threads()


FLUX_MASK = {0: (1 << abi.EY) | (1 << abi.EZ) | (1 << abi.HY) | (1 << abi.HZ),
             1: (1 << abi.EX) | (1 << abi.EZ) | (1 << abi.HX) | (1 << abi.HZ),
             2: (1 << abi.EX) | (1 << abi.EY) | (1 << abi.HX) | (1 << abi.HY)}


def add_flux_planes(sim, lo, hi, omegas):
    """Full-plane DFTs of the tangential components on the six faces of a flux
    box (the oracle has no windows: flux_box_from_planes cuts them).  Returns
    {(axis, side): dft id} with side 0 = lo face, 1 = hi face."""
    ids = {}
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        for side, v in enumerate((lo[a], hi[a])):
            ids[(a, side)] = sim.add_dft_plane(a, v, FLUX_MASK[a], omegas)
            # tangential H one plane further along the normal (far-field transform)
            ids[(a, side, "h")] = sim.add_dft_plane(a, v + 1, (1 << (3 + b)) | (1 << (3 + c)), omegas)
    return ids


def flux_box_from_planes(sim, ids, lo, hi, ds=(1.0, 1.0, 1.0)):
    """Outward FP64 flux of each face (x lo, x hi, y lo, y hi, z lo, z hi) and
    their sum, from full-plane oracle DFTs: face normal a, (a, b, c) cyclic,
    sign * d_b d_c * sum over [lo_b, hi_b) x [lo_c, hi_c) of
    Re(E_b conj(H_c) - E_c conj(H_b)).  Returns (faces[6, nfreq], total[nfreq])."""
    faces = []
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        s1, s2 = (1, 2) if a == 0 else ((0, 2) if a == 1 else (0, 1))
        comps = [q for q in range(6) if FLUX_MASK[a] & (1 << q)]
        for side in (0, 1):
            F = sim.read_dft(ids[(a, side)])[:, :, lo[s1]:hi[s1], lo[s2]:hi[s2]]
            Eb, Ec = F[comps.index(b)], F[comps.index(c)]
            Hb, Hc = F[comps.index(3 + b)], F[comps.index(3 + c)]
            s = (Eb * np.conj(Hc) - Ec * np.conj(Hb)).real.sum(axis=(1, 2))
            faces.append((1.0 if side else -1.0) * ds[s1] * ds[s2] * s)
    faces = np.array(faces)
    return faces, faces.sum(axis=0)


def _comp_off(c, x):
    return int(x != c) if c < 3 else int(x == c - 3)


def _ntff_weights(lo, hi, o):
    """Quadrature weights of indices lo..hi over [lo + 1/2, hi + 1/2] for a
    component at index + o/2: midpoints (o = 0) or trapezoid (o = 1)."""
    v = np.arange(lo, hi + 1)
    if o == 0:
        return ((v > lo) & (v <= hi)).astype(np.float64)
    w = ((v > lo) & (v < hi)).astype(np.float64)
    w[0] = w[-1] = 0.5
    return w


def ntff_from_planes(sim, ids, lo, hi, omegas, theta, phi, ds=(1.0, 1.0, 1.0), origin=None):
    """Near-to-far-field transform of a flux box from full-plane oracle DFTs:
    J = n x H, M = -n x E on each face, N = sum J exp(i k rhat.r') dA and
    L = sum M exp(i k rhat.r') dA on the surface of the tangential E (half a
    cell beyond each face plane along its normal; H averaged onto it from the
    face plane and the next one), every term at its component's in-plane Yee
    position, U = k^2/(16 pi^2)(|L_phi + N_theta|^2 + |L_theta - N_phi|^2),
    r E_theta = -i k/(4 pi)(L_phi + N_theta), r E_phi = i k/(4 pi)(L_theta - N_phi).
    Returns (U, E_theta, E_phi), each [ndir, nfreq]."""
    th = np.ravel(np.asarray(theta, dtype=np.float64))
    ph = np.ravel(np.asarray(phi, dtype=np.float64))
    k = np.asarray(omegas, dtype=np.float64)
    rh = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
    org = origin if origin is not None else [(0.5 * (lo[a] + hi[a]) + 0.5) * ds[a] for a in range(3)]
    N = np.zeros((th.size, k.size, 3), np.complex128)
    L = np.zeros_like(N)
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        s1, s2 = (1, 2) if a == 0 else ((0, 2) if a == 1 else (0, 1))
        comps = [q for q in range(6) if FLUX_MASK[a] & (1 << q)]
        dA = ds[s1] * ds[s2]
        for side, w in enumerate((lo[a], hi[a])):
            sgn = 1.0 if side else -1.0
            F = sim.read_dft(ids[(a, side)])[:, :, lo[s1]:hi[s1] + 1, lo[s2]:hi[s2] + 1]
            F2 = sim.read_dft(ids[(a, side, "h")])[:, :, lo[s1]:hi[s1] + 1, lo[s2]:hi[s2] + 1]
            u = np.arange(lo[s1], hi[s1] + 1, dtype=np.float64)[:, None]
            v = np.arange(lo[s2], hi[s2] + 1, dtype=np.float64)[None, :]
            for t, (src, dst, wt) in enumerate(((3 + b, c, sgn), (3 + c, b, -sgn), (b, c, -sgn), (c, b, sgn))):
                idx = {a: np.float64(w), s1: u, s2: v}
                proj = 0.0
                for x in range(3):
                    off = 0.5 if x == a else 0.5 * _comp_off(src, x)
                    px = (idx[x] + off) * ds[x] - org[x]
                    proj = proj + rh[:, x][:, None, None] * px[None]
                phase = np.exp(1j * k[None, :, None, None] * proj[:, None])
                val = F[comps.index(src)]
                if src >= 3:
                    val = 0.5 * (val + F2[0 if src == 3 + min(b, c) else 1])
                qw = (_ntff_weights(lo[s1], hi[s1], _comp_off(src, s1))[:, None] *
                      _ntff_weights(lo[s2], hi[s2], _comp_off(src, s2))[None, :])
                term = wt * dA * (val[None] * qw[None, None] * phase).sum(axis=(2, 3))
                (N if t < 2 else L)[:, :, dst] += term
    tv = np.stack([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)], axis=1)[:, None, :]
    pv = np.stack([-np.sin(ph), np.cos(ph), np.zeros_like(ph)], axis=1)[:, None, :]
    Nt, Np = (N * tv).sum(-1), (N * pv).sum(-1)
    Lt, Lp = (L * tv).sum(-1), (L * pv).sum(-1)
    s = k[None, :] / (4 * np.pi)
    Et = -1j * s * (Lp + Nt)
    Ep = 1j * s * (Lt - Np)
    return np.abs(Et) ** 2 + np.abs(Ep) ** 2, Et, Ep
