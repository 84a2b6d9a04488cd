"""Oracle (test infrastructure only): numpy restatement of the reference's
analytic geometry get_mat_indev (defs.h:128-148) and TFSFsrc::set
(signal.hpp:99-115), in the reference's precision (coordinates computed in
double and stored in float, layer tests in float).  Checks the C driver's
dtmx_ref_materials / dtmx_tfsfsrc_set; never part of the product path.
"""
import math

import numpy as np

ORG, AG, ITO, GLASS = 0, 1, 2, 3
NDT = 3
NPMLX = NPMLY = 10


def mat_indev(ix, iy, iz, Np, Na, ds, da, dv):
    """get_mat_indev (defs.h:128-148) on arrays of half-cell coordinates."""
    f = np.float32
    dx, dy, dz = f(ds), f(da), f(dv)
    x = (ix * 0.5 * np.float64(dx)).astype(f)
    y = (iy * 0.5 * np.float64(dy)).astype(f)
    z = (iz * 0.5 * np.float64(dz)).astype(f)
    Xc = f(0.5 * Np * NDT * np.float64(dx))
    Yc = f(0.5 * Na * NDT * np.float64(dy))
    out = np.full(np.broadcast(x, y, z).shape, GLASS, np.uint8)
    edge = ((x < f((NPMLX * NDT + 100) * dx / f(2))) | (x > f(Np * NDT * dx) - f((NPMLX * NDT + 100) * dx / f(2))) |
            (y < f((NPMLY * NDT + 100) * dy / f(2))) | (y > f(Na * NDT * dy) - f((NPMLY * NDT + 100) * dy / f(2))))
    period, rad, height, shift = f(0.4), f(0.1), f(0.1), f(1e-5)
    # std::round: halves away from zero (np.round rounds halves to even)
    rnd = lambda v: np.sign(v) * np.floor(np.abs(v) + f(0.5))
    xr = (x - Xc) - rnd(((x - Xc) / period).astype(f)).astype(f) * period
    yr = (y - Yc) - rnd(((y - Yc) / period).astype(f)).astype(f) * period
    z1 = (z - (f(0.150) - shift)).astype(f)
    z2 = (z1 - (f(0.180) + shift)).astype(f)
    z3 = (z2 - (f(0.100) + shift)).astype(f)
    hole = (z1 > -height) & ((xr * xr + yr * yr).astype(f) < rad * rad)
    out = np.where(z3 < 0, ITO, out)
    out = np.where(z2 < 0, ORG, out)
    out = np.where(z1 < 0, np.where(hole, ORG, AG), out)
    out = np.where(edge, ORG, out)
    return out.astype(np.uint8)


def material_indices(Np, Na, Nv, ds, da, dv):
    """Per-E-component index arrays: Ex at (2i,2j+1,2k+1), Ey (2i+1,2j,2k+1),
    Ez (2i+1,2j+1,2k) half-cells."""
    i = np.arange(NDT * Np)[:, None, None]
    j = np.arange(NDT * Na)[None, :, None]
    k = np.arange(Nv)[None, None, :]
    offs = ((0, 1, 1), (1, 0, 1), (1, 1, 0))
    return [mat_indev(2 * i + o[0], 2 * j + o[1], 2 * k + o[2], Np, Na, ds, da, dv) for o in offs]


def tfsfsrc_set(c, imp, lmb, ftype=np.float32):
    """TFSFsrc::set (signal.hpp:99-115): the fields it writes.  They are
    ftype (float unless the reference is built with USE_DOUBLE): each
    assignment rounds, later lines read the rounded value, and kEnv = Omega/w
    divides two ftype values."""
    f = ftype
    wl = f(lmb)
    k = f(2 * math.pi / float(wl))
    w = f(c * float(k))
    Omega = f(0.05 * float(w))
    kEnv = Omega / w                     # float / float
    return {n: float(v) for n, v in dict(
        Imp=f(imp), V_max=f(c), cSrc=f(c), wavelength=wl, k=k, w=w, Omega=Omega, kEnv=kEnv,
        theta=f(math.pi), phi=f(math.pi / 2), t0=f(25 * 0.02), tw=f(5 * 0.02), T=f(125 * 0.02)).items()}
