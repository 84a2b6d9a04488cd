"""Flux boxes, DFT windows and Purcell post-processing.

CPU: the reference's Purcell expression against its own data (golden
fixture), the source-spectrum convention, the triangular-lattice geometry,
and known answers of the oracle's flux-box restatement (energy conservation
between nested boxes; W/W0 = sqrt(eps) for a dipole in a homogeneous
dielectric).  GPU: the engine's windows and device flux reduction against the
FP64 oracle on a reduced gyrotropic photonic-crystal configuration.

Tolerances:
  face DFT windows    <= 1e-5 rel L2 per face against the oracle (FP32 fields,
                       FP64 accumulation: the probe-trace bound of the path)
  face / total flux   <= 2e-5 relative to the largest |face flux| (a product of
                       two DFTs: twice the field bound)
  nested boxes        <= 1e-3 (lossless vacuum between the boxes; the O(dx)
                       staggering of E and H on a face is the residual)
  W/W0 homogeneous    |W/W0 - sqrt(eps)| <= 0.06 at 15 cells per wavelength in
                       the medium (grid dispersion of the discrete LDOS)
  far field (dipole)   integral of U over the sphere = flux-box power within
                       0.5 %; U(theta)/U(90 deg) = sin^2(theta) within 0.5 %
                       of U(90 deg); azimuthal ripple < 0.5 % (the lattice's
                       cos 4 phi anisotropy)
  far field vs oracle  U within 2e-5 of max U (products of two DFTs)
"""
import json
import math
import os

import numpy as np
import pytest

from conftest import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))


def test_purcell_reference_matches_gnuplot_fixture():
    from dtmaxwell4_b200 import purcell
    with open(os.path.join(HERE, "golden", "purcell_gp.json")) as f:
        fx = json.load(f)
    rows = np.array(fx["rows"], dtype=np.float64)
    om, aE, pE, aD, pD, want = rows.T
    got = purcell.purcell_reference(aE * np.exp(1j * pE), aD * np.exp(1j * pD), om)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12), np.max(np.abs(got - want))


def test_source_spectrum_is_the_injected_waveform():
    from dtmaxwell4_b200 import abi, purcell, scenarios
    f0, tau, t0 = scenarios.gauss_sine_params(20.0)
    src = abi.PointSource(comp=abi.EZ, i=0, j=0, k=0, waveform=abi.WAVE_GAUSS_SINE, amp=0.7, f0=f0, tau=tau, t0=t0)
    dt, n = 0.5, 400
    om = 2 * math.pi * np.array([0.9, 1.0, 1.1]) * f0
    got = purcell.source_spectrum(src, om, dt, n)
    want = np.zeros(3, np.complex128)
    for s in range(n):                     # point_source_kernel: u = (s + 1/2) dt - t0
        u = (s + 0.5) * dt - t0
        v = 0.7 * math.sin(2 * math.pi * f0 * u) * math.exp(-(u / tau) ** 2)
        want += v * np.exp(-1j * om * (s + 0.5) * dt) * dt
    assert np.allclose(got, want, rtol=1e-12, atol=1e-14)


def test_triangular_lattice_geometry():
    from dtmaxwell4_b200 import scenarios
    period, r = 12, 4
    m = scenarios.triangular_holes(96, 96, (48.5, 48.5), period, r, 2)
    # the defect: no hole within `period - r` of the centre; the six nearest sites are holes
    x = np.arange(96)[:, None] + 0.5 - 48.5
    y = np.arange(96)[None, :] + 0.5 - 48.5
    assert not m[(x ** 2 + y ** 2) < (period - r - 0.5) ** 2].any()
    h = period * math.sqrt(3) / 2
    for (cx, cy) in [(period, 0), (-period, 0), (period / 2, h), (-period / 2, h), (period / 2, -h), (-period / 2, -h)]:
        i, j = int(round(48.5 + cx - 0.5)), int(round(48.5 + cy - 0.5))
        assert m[i, j]
    # fill fraction away from the defect ~ 2 pi r^2 / (sqrt(3) period^2)
    frac = m[24:72, 24:72].mean()
    assert abs(frac - 2 * math.pi * r * r / (math.sqrt(3) * period ** 2)) < 0.03
    with pytest.raises(ValueError):
        scenarios.triangular_holes(16, 16, (8, 8), 10, 5, 0)
    sc = scenarios.gyro_crystal_purcell(n=(64, 64, 64), slab=8, layer=12, period=12, radius=4, box_half=5, nfreq=3,
                                        steps=10, pml=6)
    mats, idx = sc["materials"]
    assert len(mats) == 4 and idx[2][32, 32, 32] == 1           # dipole node in the slab (the defect)
    # the gyrotropic layer (2) inside the absorber-free interior, the plain dielectric (3) in the CPML slabs
    assert (idx[0][6:58, 6:58, 16:28] == 2).all() and (idx[0][:, :, 40:] == 0).all()
    assert (idx[0][:6, :, 16:28] == 3).all() and (idx[0][:, 58:, 16:28] == 3).all()
    assert mats[3].gyro_wp == 0 and mats[3].npoles == 0 and tuple(mats[3].eps) == (4.0, 4.0, 4.0)
    assert sc["flux"][0][0] == [27, 27, 27] and sc["flux"][0][1] == [37, 37, 37]


def _homogeneous(eps, sim_cls, n=56, lam=30.0, halves=(8, 14), steps=900, pml=10):
    """Dipole in a homogeneous medium with two nested flux boxes."""
    from dtmaxwell4_b200 import abi, scenarios
    cfg = abi.make_config(n, n, n, courant=0.5, order=2, pml=pml)
    sim = sim_cls(cfg)
    if eps != 1.0:
        idx = np.ones((n, n, n), np.uint8)
        sim.set_materials([abi.make_material(1.0), abi.make_material(eps)], idx, idx, idx)
    f0, tau, t0 = scenarios.gauss_sine_params(lam)
    sim.add_point_source(abi.PointSource(comp=abi.EZ, i=n // 2, j=n // 2, k=n // 2, waveform=abi.WAVE_GAUSS_SINE,
                                         amp=1.0, f0=f0, tau=tau, t0=t0))
    om = 2 * math.pi * np.array([0.8, 0.9, 1.0, 1.1, 1.2]) * f0
    c = n // 2
    boxes = [([c - h] * 3, [c + h] * 3) for h in halves]
    return sim, boxes, om, steps


def test_oracle_flux_box_known_answers():
    import pyoracle
    from dtmaxwell4_b200 import purcell
    power = {}
    for eps in (1.0, 4.0):
        o, boxes, om, steps = _homogeneous(eps, lambda cfg: pyoracle.OracleSim(cfg, "f64"))
        ids = [pyoracle.add_flux_planes(o, lo, hi, om) for lo, hi in boxes]
        o.step(steps)
        power[eps] = [pyoracle.flux_box_from_planes(o, i, lo, hi)[1] for i, (lo, hi) in zip(ids, boxes)]
        assert (power[eps][0] > 0).all()
        assert np.max(np.abs(power[eps][1] / power[eps][0] - 1)) < 1e-3, power[eps]
    w = purcell.purcell_flux(power[4.0][0], power[1.0][0], 4.0, 1.0)
    print("W/W0 (eps 4):", w)
    assert np.max(np.abs(w - 2.0)) < 0.06, w


@pytest.mark.gpu
def test_flux_box_gyro_crystal_vs_oracle():
    import pyoracle
    from dtmaxwell4_b200 import Simulation, scenarios
    sc = scenarios.gyro_crystal_purcell(n=(48, 48, 64), slab=8, layer=16, period=12, radius=4, box_half=6, nfreq=4,
                                        steps=320, pml=8)
    g = Simulation(sc["cfg"])
    o = pyoracle.OracleSim(sc["cfg"], "f64")
    scenarios.apply(g, sc)
    scenarios.apply(o, sc)
    (lo, hi, om), = sc["flux"]
    fid, = scenarios.apply_flux(g, sc)
    oid = pyoracle.add_flux_planes(o, lo, hi, om)
    g.step(sc["steps"])
    o.step(sc["steps"])
    # probe at the dipole
    tg, to = g.read_probes(), o.read_probes(100000)
    assert rel_l2(tg, to) <= 1e-5
    # every face window against the oracle's plane, cut to the window
    faces = g.flux_faces(fid)
    for q, (a, side) in enumerate([(a, s) for a in range(3) for s in (0, 1)]):
        s1, s2 = (1, 2) if a == 0 else ((0, 2) if a == 1 else (0, 1))
        want = o.read_dft(oid[(a, side)])[:, :, lo[s1]:hi[s1], lo[s2]:hi[s2]]
        got = g.read_dft(faces[q])
        e = rel_l2(np.stack([got.real, got.imag]), np.stack([want.real, want.imag]))
        assert e <= 1e-5, (q, e)
    gf, gt = g.read_flux(fid)
    of, ot = pyoracle.flux_box_from_planes(o, oid, lo, hi)
    scale = np.abs(of).max()
    print("flux faces max err / max|face|: %.2e, total %s vs %s" % (np.abs(gf - of).max() / scale, gt, ot))
    assert np.abs(gf - of).max() <= 2e-5 * scale
    assert np.abs(gt - ot).max() <= 2e-5 * scale
    assert np.array_equal(gt, gf.sum(axis=0))
    # far field of the same box (gyrotropic layer and slab inside the domain)
    th, TH, PH = _sphere_grid(12, 24)
    U, _, _ = g.far_field(fid, TH.ravel(), PH.ravel())
    Uo, _, _ = pyoracle.ntff_from_planes(o, oid, lo, hi, om, TH.ravel(), PH.ravel())
    print("far field max err / max U: %.2e" % (np.abs(U - Uo).max() / Uo.max()))
    assert np.abs(U - Uo).max() <= 2e-5 * Uo.max()


@pytest.mark.gpu
def test_dft_patch_is_the_plane_window():
    """A window and the full plane accumulate the same values in the same
    order: the window equals the cut plane exactly."""
    from dtmaxwell4_b200 import Simulation, scenarios
    sc = scenarios.point_dipole_sphere(n=40, steps=120, pml=6, radius=6, order=2, lambda0=10.0)
    g = Simulation(sc["cfg"])
    scenarios.apply(g, sc)
    om = 2 * math.pi / 10.0 * np.array([0.9, 1.0, 1.1])
    mask = 0b111111
    pid = g.add_dft_plane(1, 17, mask, om)
    wid = g.add_dft_patch(1, 17, 5, 21, 9, 13, mask, om)
    one = g.add_dft_patch(2, 20, 20, 1, 20, 1, 1 << 2, om)      # the dipole's Ez node
    g.step(sc["steps"])
    P, W = g.read_dft(pid), g.read_dft(wid)
    assert np.array_equal(W, P[:, :, 5:26, 9:22])
    assert g.read_dft(one).shape == (1, 3, 1, 1)


@pytest.mark.gpu
def test_engine_purcell_homogeneous_dielectric():
    """Engine flux boxes: W/W0 = sqrt(eps) for a dipole in eps = 4, nested
    boxes agree, and the totals match the oracle."""
    import pyoracle
    from dtmaxwell4_b200 import Simulation, purcell
    power = {}
    for eps in (1.0, 4.0):
        g, boxes, om, steps = _homogeneous(eps, Simulation)
        fids = [g.add_flux_box(lo, hi, om) for lo, hi in boxes]
        g.step(steps)
        power[eps] = [g.read_flux(f)[1] for f in fids]
        assert np.max(np.abs(power[eps][1] / power[eps][0] - 1)) < 1e-3
        if eps == 4.0:
            o, boxes, om, steps = _homogeneous(eps, lambda cfg: pyoracle.OracleSim(cfg, "f64"))
            oid = pyoracle.add_flux_planes(o, boxes[0][0], boxes[0][1], om)
            o.step(steps)
            ot = pyoracle.flux_box_from_planes(o, oid, boxes[0][0], boxes[0][1])[1]
            assert np.max(np.abs(power[eps][0] - ot)) <= 2e-5 * np.abs(ot).max()
    w = purcell.purcell_flux(power[4.0][0], power[1.0][0], 4.0, 1.0)
    assert np.max(np.abs(w - 2.0)) < 0.06, w


def _sphere_grid(nt=36, nph=72):
    th = (np.arange(nt) + 0.5) * np.pi / nt
    ph = (np.arange(nph) + 0.5) * 2 * np.pi / nph
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    return th, TH, PH


def _check_dipole_far_field(U, th, total):
    """U[nt, nph, nf] of a z dipole against the flux-box total[nf]."""
    nt, nph = U.shape[:2]
    P = (U * np.sin(th)[:, None, None]).sum(axis=(0, 1)) * (np.pi / nt) * (2 * np.pi / nph)
    assert np.max(np.abs(P / total - 1)) < 5e-3, (P, total)
    eq = U[nt // 2 - 1: nt // 2 + 1].mean(axis=(0, 1))
    shape = U.mean(axis=1) / eq
    assert np.max(np.abs(shape - np.sin(th)[:, None] ** 2)) < 5e-3
    ripple = np.abs(U - U.mean(axis=1, keepdims=True)).max(axis=(0, 1)) / U.max(axis=(0, 1))
    assert np.max(ripple) < 5e-3, ripple


def test_oracle_far_field_dipole_known_answers():
    import pyoracle
    o, boxes, om, steps = _homogeneous(1.0, lambda cfg: pyoracle.OracleSim(cfg, "f64"), halves=(8,))
    (lo, hi), = boxes
    ids = pyoracle.add_flux_planes(o, lo, hi, om)
    o.step(steps)
    _, total = pyoracle.flux_box_from_planes(o, ids, lo, hi)
    th, TH, PH = _sphere_grid()
    U, _, _ = pyoracle.ntff_from_planes(o, ids, lo, hi, om, TH.ravel(), PH.ravel())
    _check_dipole_far_field(U.reshape(TH.shape + (len(om),)), th, total)


@pytest.mark.gpu
def test_engine_far_field_dipole_and_oracle():
    """Engine near-to-far-field transform: dipole known answers, and the
    same sums as the oracle's restatement on the same run."""
    import pyoracle
    from dtmaxwell4_b200 import Simulation
    g, boxes, om, steps = _homogeneous(1.0, Simulation, halves=(8,))
    (lo, hi), = boxes
    fid = g.add_flux_box(lo, hi, om)
    g.step(steps)
    _, total = g.read_flux(fid)
    th, TH, PH = _sphere_grid()
    U, Et, Ep = g.far_field(fid, TH.ravel(), PH.ravel())
    _check_dipole_far_field(U.reshape(TH.shape + (len(om),)), th, total)
    o, _, _, _ = _homogeneous(1.0, lambda cfg: pyoracle.OracleSim(cfg, "f64"), halves=(8,))
    ids = pyoracle.add_flux_planes(o, lo, hi, om)
    o.step(steps)
    Uo, Eto, Epo = pyoracle.ntff_from_planes(o, ids, lo, hi, om, TH.ravel(), PH.ravel())
    assert np.max(np.abs(U - Uo)) <= 2e-5 * np.max(Uo)
    assert np.allclose(np.abs(U), np.abs(Et) ** 2 + np.abs(Ep) ** 2, rtol=1e-12, atol=0)
