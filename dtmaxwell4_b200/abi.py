"""ctypes mirror of include/dtmx.h (the C ABI of the CUDA engine).

Struct layouts here must match the header field for field; tests/test_cpu.py
checks the sizes against the compiled library.
"""
import ctypes as C

ABI_VERSION = 1

(OK, ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_NONFINITE, ERR_TIMEOUT, ERR_STATE, ERR_UNSUPPORTED, ERR_NODEVICE,
 ERR_TOO_LARGE) = range(10)
NOALLOC_BLOCK_ELEMS = 4096
NOALLOC_MAX_BLOCKS = 4096
NOALLOC_MAX_ELEMS = NOALLOC_BLOCK_ELEMS * NOALLOC_MAX_BLOCKS
EX, EY, EZ, HX, HY, HZ = range(6)
COMP_NAMES = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
GEOM_BOX, GEOM_REFERENCE = 0, 1
ABS_NONE, ABS_CPML, ABS_SPLIT_PML = 0, 1, 2
POLE_LORENTZ, POLE_DRUDE = 0, 1
MAX_POLES = 2
MAX_MATERIALS = 64
WAVE_GAUSS_SINE = 0
TFSF_DIPOLE, TFSF_PLANE_X = 0, 1
PROBE_NODE, PROBE_REFERENCE = 0, 1


class Config(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("order", C.c_int),
        ("geometry", C.c_int),
        ("absorber", C.c_int),
        ("pml", (C.c_int * 2) * 3),
        ("cpml_m", C.c_double), ("cpml_sigma_factor", C.c_double),
        ("cpml_kappa_max", C.c_double), ("cpml_alpha_max", C.c_double),
        ("spml_vmax", C.c_double),
        ("probe_every", C.c_int),
        ("probe_capacity", C.c_int),
        ("parkable", C.c_int),
        ("reserved", C.c_int * 7),
    ]


class Material(C.Structure):
    _fields_ = [
        ("eps", C.c_double * 3),
        ("npoles", C.c_int),
        ("pole_kind", C.c_int * MAX_POLES),
        ("pole", (C.c_double * 4) * MAX_POLES),
        ("eps_inf", C.c_double),
        ("sigma", C.c_double),
        ("gyro_wp", C.c_double), ("gyro_gamma", C.c_double), ("gyro_wc", C.c_double),
        ("reserved", C.c_double * 4),
    ]


class PointSource(C.Structure):
    _fields_ = [
        ("comp", C.c_int), ("i", C.c_int), ("j", C.c_int), ("k", C.c_int),
        ("waveform", C.c_int),
        ("amp", C.c_double), ("f0", C.c_double), ("tau", C.c_double), ("t0", C.c_double),
    ]


class TFSF(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("box_lo", C.c_double * 3), ("box_hi", C.c_double * 3),
        ("c", C.c_double), ("w", C.c_double), ("kenv", C.c_double),
        ("tstop", C.c_double),
        ("ntime", C.c_int),
        ("amp", C.c_double), ("f0", C.c_double), ("tau", C.c_double), ("t0", C.c_double),
        ("x_origin", C.c_double), ("x_cells", C.c_double),
        ("reserved", C.c_double * 2),
    ]


def make_config(nx, ny, nz, dx=1.0, dy=None, dz=None, dt=None, courant=0.5, order=2,
                geometry=GEOM_BOX, absorber=ABS_CPML, pml=10, cpml_m=3.0, cpml_sigma_factor=1.0,
                cpml_kappa_max=1.0, cpml_alpha_max=0.0, spml_vmax=1.0, probe_every=1,
                probe_capacity=0, parkable=False):
    """Build a Config.  dt defaults to courant*dx (c = 1); pml is an int for all
    six faces or a ((xlo,xhi),(ylo,yhi),(zlo,zhi)) tuple."""
    dy = dx if dy is None else dy
    dz = dx if dz is None else dz
    if dt is None:
        dt = courant * min(dx, dy, dz)
    cfg = Config()
    cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
    cfg.dx, cfg.dy, cfg.dz, cfg.dt = dx, dy, dz, dt
    cfg.order = order
    cfg.geometry = geometry
    cfg.absorber = absorber
    if isinstance(pml, int):
        pml = ((pml, pml),) * 3
    for a in range(3):
        for s in range(2):
            cfg.pml[a][s] = int(pml[a][s])
    cfg.cpml_m, cfg.cpml_sigma_factor = cpml_m, cpml_sigma_factor
    cfg.cpml_kappa_max, cfg.cpml_alpha_max = cpml_kappa_max, cpml_alpha_max
    cfg.spml_vmax = spml_vmax
    cfg.probe_every = probe_every
    cfg.probe_capacity = probe_capacity
    cfg.parkable = 1 if parkable else 0
    return cfg


def make_material(eps=1.0, poles=(), eps_inf=1.0, sigma=0.0, gyro=None):
    """eps: scalar or 3-tuple; poles: iterable of (kind, Deps, wp, gp, gp_);
    gyro: (wp, gamma, wc) of a magnetised-Drude current (bias along +z), with
    eps_inf the background permittivity."""
    m = Material()
    if isinstance(eps, (int, float)):
        eps = (eps, eps, eps)
    for c in range(3):
        m.eps[c] = float(eps[c])
    poles = list(poles)
    if len(poles) > MAX_POLES:
        raise ValueError("at most %d poles" % MAX_POLES)
    m.npoles = len(poles)
    for p, (kind, Deps, wp, gp, gp_) in enumerate(poles):
        m.pole_kind[p] = kind
        m.pole[p][0], m.pole[p][1], m.pole[p][2], m.pole[p][3] = Deps, wp, gp, gp_
    m.eps_inf = eps_inf
    m.sigma = sigma
    if gyro is not None:
        m.gyro_wp, m.gyro_gamma, m.gyro_wc = (float(v) for v in gyro)
    return m


def gyro_for(eps_diag, g, omega0, wc_ratio=0.5):
    """Magnetised-Drude parameters (eps_inf, (wp, 0, wc)) whose lossless tensor
    at omega0 has diagonal eps_diag and off-diagonal magnitude g:
    eps_xx = eps_inf - wp^2/(w0^2 - wc^2), |eps_xy| = wp^2 wc / (w0 (w0^2 - wc^2)),
    with wc = wc_ratio * omega0."""
    wc = wc_ratio * omega0
    den = omega0 ** 2 - wc ** 2
    wp2 = g * omega0 * den / wc
    return eps_diag + wp2 / den, (wp2 ** 0.5, 0.0, wc)
