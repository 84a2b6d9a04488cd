"""CPU-only tests: the C ABI library loads and exports every declared symbol;
the oracle reproduces analytic known answers of the update equations."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "dtmx.h")).read()
    return sorted(set(re.findall(r"\b(dtmx_[a-z_0-9]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    from dtmaxwell4_b200 import build, engine
    build.build()
    lib = ctypes.CDLL(engine.LIB_PATH)
    syms = _declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(engine.EXPORTS)


def test_abi_struct_sizes_match_bindings():
    from dtmaxwell4_b200 import DTmxw, abi, engine
    sizes = engine.abi_sizes()
    assert sizes == (ctypes.sizeof(abi.Config), ctypes.sizeof(abi.Material), ctypes.sizeof(abi.PointSource),
                     ctypes.sizeof(abi.TFSF), ctypes.sizeof(DTmxw.TFSFsrc), ctypes.sizeof(DTmxw.RefGlobals))


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from dtmaxwell4_b200 import DtmxError, Simulation, abi
    with pytest.raises(DtmxError) as e:
        Simulation(abi.make_config(16, 16, 16))
    assert e.value.code == abi.ERR_NODEVICE


@pytest.mark.parametrize("order", [2, 4])
def test_oracle_stencil_symbol(order):
    """One H half step from Ez = sin(k(i+1)), H = 0: Hy(i) must equal
    S * 2 cos(k(i+1/2)) * s(k) with s = sin(k/2) (order 2) or
    (27 sin(k/2) - sin(3k/2))/24 (order 4), the symbol of the staggered
    difference; sign: dHy/dt = +dEz/dx."""
    import pyoracle
    from dtmaxwell4_b200 import abi
    n = 24
    S = 0.4
    cfg = abi.make_config(n, n, n, courant=S, order=order, absorber=abi.ABS_NONE, pml=0)
    o = pyoracle.OracleSim(cfg)
    k = 2 * math.pi / 9.0
    i = np.arange(n)[:, None, None]
    ez = np.sin(k * (i + 1)) * np.ones((n, n, n))
    o.set_field(abi.EZ, ez)
    o.step(1)
    hy = o.get_field(abi.HY)
    sym = math.sin(k / 2) if order == 2 else (27 * math.sin(k / 2) - math.sin(1.5 * k)) / 24
    expect = S * 2 * np.cos(k * (i + 0.5)) * sym
    sl = (slice(4, n - 4), slice(4, n - 4), slice(4, n - 4))
    np.testing.assert_allclose(hy[sl], np.broadcast_to(expect, hy.shape)[sl], rtol=0, atol=1e-12)


@pytest.mark.parametrize("order,S", [(2, 0.5), (4, 0.4)])
def test_oracle_numerical_dispersion(order, S):
    """A standing eigenmode advances with the discrete dispersion relation
    sin(w dt/2) = S * s(k) (s as above): after n steps Ez(t) follows
    cos(w n dt) up to the half-step phase of the leapfrog start."""
    import pyoracle
    from dtmaxwell4_b200 import abi
    n = 64
    cfg = abi.make_config(n, 12, 12, courant=S, order=order, absorber=abi.ABS_NONE, pml=0)
    o = pyoracle.OracleSim(cfg)
    k = 2 * math.pi / 16.0
    sym = math.sin(k / 2) if order == 2 else (27 * math.sin(k / 2) - math.sin(1.5 * k)) / 24
    w = 2 * math.asin(S * sym)       # omega*dt
    i = np.arange(n)[:, None, None]
    # eigenmode of the leapfrog pair: Ez^0 = sin(k(i+1)), Hy^{-1/2} = -A cos(k(i+1/2)) sin(w/2)/(S*sym)*S*sym...
    ez0 = np.sin(k * (i + 1)) * np.ones((n, 12, 12))
    hy0 = -np.sin(w / 2) * np.cos(k * (i + 0.5)) * np.ones((n, 12, 12))
    o.set_field(abi.EZ, ez0)
    o.set_field(abi.HY, hy0)
    o.add_probe(abi.EZ, 31, 6, 6)
    steps = 40
    o.step(steps)
    tr = o.read_probes(100)[0]
    t = np.arange(1, steps + 1)
    expect = math.sin(k * 32) * np.cos(w * t)
    # the y/z walls (zero outside) do not reach the centre within 40 steps for these sizes?
    np.testing.assert_allclose(tr[:4], expect[:4], atol=1e-9)


def _kzero_trace(material, steps):
    """Ex uniform in a mirror-walled box (reference geometry, no absorber):
    y and z mirrors are even for E, so the field stays uniform and only the
    ADE acts.  The ADE state starts at rest (E^{-1} = 0), i.e. a step in E."""
    import pyoracle
    from dtmaxwell4_b200 import abi
    n = 12
    cfg = abi.make_config(n, n, n, courant=0.5, order=2, geometry=abi.GEOM_REFERENCE, absorber=abi.ABS_NONE, pml=0)
    o = pyoracle.OracleSim(cfg)
    o.set_materials([abi.make_material(1.0), material], np.ones((n, n, n), np.uint8))
    o.set_field(abi.EX, np.ones((n, n, n)))
    o.add_probe(abi.EX, n // 2, n // 2, n // 2)
    o.step(steps)
    return o.read_probes(steps + 10)[0]


def _period(tr, dt):
    """Mean spacing of the local maxima (parabolic refinement)."""
    pk = [i for i in range(1, len(tr) - 1) if tr[i] > tr[i - 1] and tr[i] >= tr[i + 1]]
    t = []
    for i in pk:
        a, b, c = tr[i - 1], tr[i], tr[i + 1]
        den = a - 2 * b + c
        t.append((i + (0.5 * (a - c) / den if den != 0 else 0.0)) * dt)
    return float(np.mean(np.diff(t)))


def test_oracle_drude_plasma_oscillation():
    """Drude pole (LorenzDisp::setDrude): the k = 0 mode oscillates at
    sqrt(wp^2/eps_inf - gamma^2/4), the zero of eps(w) = eps_inf - wp^2/(w^2 + i gamma w)."""
    from dtmaxwell4_b200 import abi
    wp, gamma, einf = 0.3, 0.01, 1.0
    drude = abi.make_material(1.0, poles=[(abi.POLE_DRUDE, 1.0, wp, gamma / 2, 0.0)], eps_inf=einf)
    tr = _kzero_trace(drude, 400)
    assert np.ptp(tr) > 0.5
    expect = 2 * math.pi / math.sqrt(wp ** 2 / einf - gamma ** 2 / 4)
    assert abs(_period(tr, 0.5) / expect - 1) < 3e-3, (_period(tr, 0.5), expect)


def test_oracle_lorentz_resonance():
    """Lorentz pole (LorenzDisp::set): k = 0 oscillation at
    w0 sqrt((eps_inf + deps)/eps_inf) (longitudinal resonance)."""
    from dtmaxwell4_b200 import abi
    w0, deps, einf = 0.2, 2.0, 1.5
    lor = abi.make_material(1.0, poles=[(abi.POLE_LORENTZ, deps, w0, 0.0, 0.0)], eps_inf=einf)
    tr = _kzero_trace(lor, 400)
    expect = 2 * math.pi / (w0 * math.sqrt((einf + deps) / einf))
    assert abs(_period(tr, 0.5) / expect - 1) < 3e-3, (_period(tr, 0.5), expect)


def test_oracle_cpml_absorbs():
    """A pulse leaving a CPML-terminated box: energy falls by > 40 dB."""
    import pyoracle
    from dtmaxwell4_b200 import scenarios
    sc = scenarios.point_dipole_sphere(n=40, steps=0, pml=8, radius=0.1, eps=1.0, lambda0=10.0)
    o = pyoracle.OracleSim(sc["cfg"])
    scenarios.apply(o, sc)
    o.step(120)
    e1 = sum(float((o.get_field(c) ** 2).sum()) for c in range(6))
    o.step(380)
    e2 = sum(float((o.get_field(c) ** 2).sum()) for c in range(6))
    assert e2 < 1e-4 * e1, (e1, e2)


def _gyro_uniform_recursion(einf, wp, wc, gamma, dt, steps):
    """The magnetised-Drude scheme on a spatially uniform state (curl H = 0):
    the (Ex, Ey, Jx, Jy) map of one step, started from Ex = 1."""
    a, C, S, b, jc = math.exp(-gamma * dt), math.cos(wc * dt), math.sin(wc * dt), wp * wp * dt, dt / einf
    ex, ey, jx, jy = 1.0, 0.0, 0.0, 0.0
    out = []
    for _ in range(steps):
        jx, jy = a * (C * jx + S * jy) + b * ex, a * (C * jy - S * jx) + b * ey
        ex, ey = ex - jc * jx, ey - jc * jy
        out.append((ex, ey))
    return np.array(out)


def test_oracle_gyrotropic_uniform_mode():
    """Magnetised-Drude current: a uniform Ex in a gyrotropic block follows the
    single-node recursion (until the block edges, where the 4-node averages see
    zero current, reach the probe), and that recursion rotates the polarisation
    at the two magnetoplasma frequencies w = (+-wc + sqrt(wc^2 + 4 wp^2/eps_inf))/2."""
    import pyoracle
    from dtmaxwell4_b200 import abi
    n, steps = 84, 30
    einf, wp, wc, gamma = 1.5, 0.8, 0.6, 0.02
    cfg = abi.make_config(n, n, 6, courant=0.5, order=2, geometry=abi.GEOM_REFERENCE, absorber=abi.ABS_NONE, pml=0)
    o = pyoracle.OracleSim(cfg)
    o.set_materials([abi.make_material(1.0), abi.make_material(eps_inf=einf, gyro=(wp, gamma, wc))],
                    np.ones((n, n, 6), np.uint8))
    o.set_field(abi.EX, np.ones((n, n, 6)))
    o.add_probe(abi.EX, n // 2, n // 2, 3)
    o.add_probe(abi.EY, n // 2, n // 2, 3)
    o.step(steps)
    tr = o.read_probes(steps + 5)
    ref = _gyro_uniform_recursion(einf, wp, wc, gamma, cfg.dt, steps)
    assert np.abs(tr[0] - ref[:, 0]).max() < 1e-12 and np.abs(tr[1] - ref[:, 1]).max() < 1e-12
    assert np.abs(ref[:, 1]).max() > 0.05            # the bias field rotates the polarisation
    # eigenfrequencies of the one-step map (lossless, small dt) vs the continuous modes
    dt = 0.01
    C, S, b, jc = math.cos(wc * dt), math.sin(wc * dt), wp * wp * dt, dt / einf
    T = np.zeros((4, 4))
    # state (Jx, Jy, Ex, Ey): J' = R J + b E ; E' = E - jc J'
    T[:2, :2] = [[C, S], [-S, C]]; T[:2, 2:] = b * np.eye(2)
    T[2:, :] = np.hstack([-jc * T[:2, :2], np.eye(2) - jc * b * np.eye(2)])
    w = sorted(abs(np.angle(np.linalg.eigvals(T))) / dt)
    expect = sorted([(s * wc + math.sqrt(wc * wc + 4 * wp * wp / einf)) / 2 for s in (1, -1)])
    got = sorted(set(round(v, 6) for v in w))
    assert len(got) == 2 and all(abs(g / e - 1) < 2e-3 for g, e in zip(got, expect)), (got, expect)


def test_read_arr_layout(tmp_path):
    """The .arr reader: int32 {12, 0, 0, 0, 3, 4, nz, ny, nx}, z fastest."""
    from dtmaxwell4_b200 import engine
    a = np.arange(2 * 3 * 5, dtype=np.float32).reshape(2, 3, 5)
    p = tmp_path / "f.arr"
    with open(p, "wb") as f:
        np.array([12, 0, 0, 0, 3, 4, 5, 3, 2], np.int32).tofile(f)
        a.tofile(f)
    assert np.array_equal(engine.read_arr(str(p)), a)
