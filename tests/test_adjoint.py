"""Gradient of a Poynting-flux objective with respect to per-node
permittivity by the discrete adjoint.

Oracle (CPU): the FP64 adjoint equals central finite differences of the FP64
forward.  GPU: the FP32 engine's adjoint against the FP64 adjoint and against
its own central differences, identical results from the recorded design
history and from checkpointed recompute at two intervals, the final state, and
the torch.autograd binding.
"""
import math

import numpy as np
import pytest

N_STEPS, PLANE_X, OMEGA = 60, 15, 2 * math.pi / 8.0
LO = (9, 7, 7)


def _eps():
    return np.random.default_rng(1).uniform(1, 4, size=(3, 3, 3, 3))


def _setup(sim, order):
    from dtmaxwell4_b200 import abi, scenarios
    f0, tau, t0 = scenarios.gauss_sine_params(8.0)
    sim.add_point_source(abi.PointSource(comp=abi.EZ, i=6, j=9, k=9, waveform=abi.WAVE_GAUSS_SINE, amp=1.0, f0=f0,
                                         tau=tau, t0=t0))
    return sim


def _cfg(order):
    from dtmaxwell4_b200 import abi
    return abi.make_config(22, 18, 18, dx=1.0, courant=0.5 if order == 2 else 0.4, order=order,
                           absorber=abi.ABS_CPML, pml=4)


def _oracle(order, eps):
    import pyoracle
    o = _setup(pyoracle.OracleSim(_cfg(order)), order)
    o.set_design(LO, eps)
    return o.forward_adjoint(N_STEPS, PLANE_X, OMEGA)


@pytest.mark.parametrize("order", [2, 4])
def test_oracle_adjoint_matches_finite_differences(order):
    eps = _eps()
    J, g = _oracle(order, eps)
    assert J != 0
    for cell in [(2, 1, 1, 1), (0, 0, 2, 1), (2, 0, 0, 2)]:
        h = 1e-4
        ep, em = eps.copy(), eps.copy()
        ep[cell] += h
        em[cell] -= h
        fd = (_oracle(order, ep)[0] - _oracle(order, em)[0]) / (2 * h)
        assert abs(g[cell] - fd) <= 1e-6 * abs(fd), (cell, g[cell], fd)


def _disp_materials(nx=22, ny=18, nz=18, overlap=False):
    """A Drude block across the objective plane and a two-pole (Lorentz +
    Drude) block near the source; overlap: one Drude node inside the design
    region."""
    from dtmaxwell4_b200 import abi
    wp = 2 * math.pi / 8
    mats = [abi.make_material(1.0),
            abi.make_material(1.0, poles=[(abi.POLE_DRUDE, 1.0, wp, wp / 40, 0.0)], eps_inf=1.5),
            abi.make_material(1.0, poles=[(abi.POLE_LORENTZ, 1.5, 0.5, 0.05, 0.0), (abi.POLE_DRUDE, 1.0, 0.8, 0.02, 0.0)],
                              eps_inf=2.0)]
    idx = np.zeros((nx, ny, nz), np.uint8)
    idx[13:18, 4:13, 5:13] = 1
    idx[3:6, 7:12, 6:12] = 2
    if overlap:
        idx[LO[0] + 1, LO[1], LO[2] + 2] = 1
    return mats, idx


def _oracle_disp(eps, overlap=False):
    import pyoracle
    o = _setup(pyoracle.OracleSim(_cfg(2)), 2)
    mats, idx = _disp_materials(overlap=overlap)
    o.set_materials(mats, idx, idx, idx)
    o.set_design(LO, eps)
    return o.forward_adjoint(N_STEPS, PLANE_X, OMEGA)


@pytest.mark.parametrize("overlap", [False, True])
def test_oracle_adjoint_dispersive_matches_finite_differences(overlap):
    """The transposed ADE recursion (Drude and Lorentz poles): the FP64
    adjoint equals central differences of the FP64 forward; a design node
    whose material is dispersive has gradient 0 (its permittivity is the
    material's, not the design's), and so does J's difference quotient."""
    eps = _eps()
    J, g = _oracle_disp(eps, overlap)
    assert J != 0
    cells = [(2, 1, 1, 1), (0, 0, 2, 1), (1, 2, 0, 2)]
    if overlap:
        cells.append((0, 1, 0, 2))
        assert g[0, 1, 0, 2] == 0.0
    for cell in cells:
        h = 1e-4
        ep, em = eps.copy(), eps.copy()
        ep[cell] += h
        em[cell] -= h
        fd = (_oracle_disp(ep, overlap)[0] - _oracle_disp(em, overlap)[0]) / (2 * h)
        assert abs(g[cell] - fd) <= 1e-6 * max(abs(fd), 1e-12 * abs(J)), (cell, g[cell], fd)


def _gyro_materials(nx=22, ny=18, nz=18, overlap=False):
    """A magnetised-Drude block (eps_diag 4, off-diagonal 0.3 at the source
    frequency) across the objective plane, next to the design region;
    overlap: one gyrotropic node inside the design region (refused)."""
    from dtmaxwell4_b200 import abi
    einf, g = abi.gyro_for(4.0, 0.3, OMEGA)
    mats = [abi.make_material(1.0), abi.make_material(1.0, eps_inf=einf, gyro=g)]
    idx = np.zeros((nx, ny, nz), np.uint8)
    idx[13:18, 4:13, 5:13] = 1
    if overlap:
        idx[LO[0] + 1, LO[1], LO[2] + 2] = 1
    return mats, idx


def _oracle_gyro(eps, overlap=False):
    import pyoracle
    o = _setup(pyoracle.OracleSim(_cfg(2)), 2)
    mats, idx = _gyro_materials(overlap=overlap)
    o.set_materials(mats, idx, idx, idx)
    o.set_design(LO, eps)
    return o.forward_adjoint(N_STEPS, PLANE_X, OMEGA)


def test_oracle_adjoint_gyrotropic_matches_finite_differences():
    """The transposed magnetised-Drude current (4-node averages gathered
    back): the FP64 adjoint equals central differences of the FP64 forward;
    a design region holding a gyrotropic node is refused."""
    eps = _eps()
    J, g = _oracle_gyro(eps)
    assert J != 0
    for cell in [(2, 1, 1, 1), (0, 0, 2, 1), (1, 2, 0, 2), (0, 2, 2, 0)]:
        h = 1e-4
        ep, em = eps.copy(), eps.copy()
        ep[cell] += h
        em[cell] -= h
        fd = (_oracle_gyro(ep)[0] - _oracle_gyro(em)[0]) / (2 * h)
        assert abs(g[cell] - fd) <= 1e-6 * abs(fd), (cell, g[cell], fd)
    with pytest.raises(ValueError):
        _oracle_gyro(eps, overlap=True)


def _gpu(order, eps, K=100, budget=-1):
    from dtmaxwell4_b200 import Simulation
    s = _setup(Simulation(_cfg(order)), order)
    s.set_design(LO, eps)
    s.set_adjoint_memory(budget)
    J, g = s.forward_adjoint(N_STEPS, PLANE_X, OMEGA, K)
    return J, g, s


@pytest.mark.gpu
@pytest.mark.parametrize("order", [2, 4])
def test_gpu_adjoint_against_fp64_adjoint(order):
    eps = _eps()
    J, g, s = _gpu(order, eps)
    s.close()
    Jo, go = _oracle(order, eps.astype(np.float32).astype(np.float64))
    assert abs(J - Jo) <= 1e-5 * abs(Jo), (J, Jo)
    cos = float((g * go).sum() / (np.linalg.norm(g) * np.linalg.norm(go)))
    rel = float(np.linalg.norm(g - go) / np.linalg.norm(go))
    assert cos >= 0.9999 and rel <= 1e-3, (cos, rel)


@pytest.mark.gpu
def test_gpu_adjoint_against_central_differences():
    """16 seeded cells, h = 1e-3 (the FP32 forward differenced)."""
    eps = _eps().astype(np.float32)
    J, g, s = _gpu(2, eps)
    s.close()
    rng = np.random.default_rng(5)
    cells = [tuple(int(v) for v in (rng.integers(3), *rng.integers(0, 3, size=3))) for _ in range(16)]
    fd, ad = [], []
    for cell in cells:
        h = 1e-3
        ep, em = eps.copy(), eps.copy()
        ep[cell] += h
        em[cell] -= h
        Jp, _, sp = _gpu(2, ep)
        sp.close()
        Jm, _, sm = _gpu(2, em)
        sm.close()
        fd.append((Jp - Jm) / (2 * h))
        ad.append(float(g[cell]))
    fd, ad = np.array(fd), np.array(ad)
    cos = float(fd @ ad / (np.linalg.norm(fd) * np.linalg.norm(ad)))
    assert cos >= 0.999, (cos, fd, ad)


@pytest.mark.gpu
def test_gpu_adjoint_checkpoint_interval_and_final_state():
    """Recorded design history (default budget) and checkpointed recompute
    (budget 0, two intervals) give bit-identical objectives and gradients and
    leave the state of a plain forward run."""
    from dtmaxwell4_b200 import Simulation
    eps = _eps()
    J0, g0, s0 = _gpu(4, eps)
    J1, g1, s1 = _gpu(4, eps, K=100, budget=0)
    J2, g2, s2 = _gpu(4, eps, K=7, budget=0)
    assert J0 == J1 == J2 and np.array_equal(g0, g1) and np.array_equal(g1, g2)
    ref = _setup(Simulation(_cfg(4)), 4)
    ref.set_design(LO, eps)
    ref.step(N_STEPS)
    for c in range(6):
        assert np.array_equal(s2.get_field(c), ref.get_field(c)), c
        assert np.array_equal(s0.get_field(c), ref.get_field(c)), c
    for q in (s0, s1, s2, ref):
        q.close()


@pytest.mark.gpu
def test_torch_autograd_binding():
    import torch
    from dtmaxwell4_b200 import Simulation
    from dtmaxwell4_b200.autograd import flux_objective
    eps0 = _eps()
    eps = torch.tensor(eps0, dtype=torch.float32, requires_grad=True)
    J = flux_objective(eps, lambda: _setup(Simulation(_cfg(2)), 2), LO, N_STEPS, PLANE_X, OMEGA)
    (2.0 * J).backward()
    Jd, gd, s = _gpu(2, eps0)
    s.close()
    assert float(J.detach()) == pytest.approx(Jd, rel=1e-6)
    np.testing.assert_allclose(eps.grad.numpy(), 2.0 * gd, rtol=1e-6, atol=0)


@pytest.mark.gpu
def test_full_size_gradient_directional_difference():
    """The differentiation configuration at full size (256x256x192, 64x64x32
    design region, 2000 steps): the directional central difference of J along
    d = sign(dJ/deps) with h = 1e-3 on every design node equals sum |dJ/deps|.
    (Per-node differences at this size change J by less than its FP32 rounding;
    they are checked at the small size above.)  Measured agreement 7.2e-6;
    held to 1e-4 (the FP32 rounding of J itself sets the noise of the
    difference quotient)."""
    from dtmaxwell4_b200 import Simulation, scenarios
    sc = scenarios.design_region()
    lo, eps = sc["design"]

    def run(e):
        s = Simulation(sc["cfg"])
        scenarios.apply(s, sc)
        s.set_design(lo, e)
        J, g = s.forward_adjoint(sc["steps"], sc["plane_x"], sc["omega"], 100)
        s.close()
        return J, g
    J, g = run(eps)
    d = np.sign(g).astype(np.float32)
    h = 1e-3
    Jp, _ = run((eps + h * d).astype(np.float32))
    Jm, _ = run((eps - h * d).astype(np.float32))
    # the perturbation actually applied, in FP32
    hp = ((eps + h * d).astype(np.float64) - eps) * d
    hm = (eps.astype(np.float64) - (eps - h * d).astype(np.float32)) * d
    fd = (Jp - Jm) / (2 * h)
    ad = float((np.abs(g).astype(np.float64) * (hp + hm) / (2 * h)).sum())
    print("J %.9g  directional FD %.9g  adjoint %.9g  rel %.2e" % (J, fd, ad, abs(fd - ad) / abs(ad)))
    assert abs(fd - ad) <= 1e-4 * abs(ad)


def _gpu_disp(eps, K=100, budget=-1, overlap=False):
    from dtmaxwell4_b200 import Simulation
    s = _setup(Simulation(_cfg(2)), 2)
    mats, idx = _disp_materials(overlap=overlap)
    s.set_materials(mats, idx, idx, idx)
    s.set_design(LO, eps)
    s.set_adjoint_memory(budget)
    J, g = s.forward_adjoint(N_STEPS, PLANE_X, OMEGA, K)
    return J, g, s


@pytest.mark.gpu
@pytest.mark.parametrize("overlap", [False, True])
def test_gpu_adjoint_dispersive_against_fp64_adjoint(overlap):
    """Drude and two-pole Lorentz+Drude blocks (one Drude node in the design
    region with overlap): the GPU adjoint of the ADE recursion against the
    FP64 adjoint, recorded history and checkpointed recompute bit-identical."""
    eps = _eps()
    J, g, s = _gpu_disp(eps, overlap=overlap)
    s.close()
    J2, g2, s2 = _gpu_disp(eps, K=7, budget=0, overlap=overlap)
    s2.close()
    assert J2 == J and np.array_equal(g2, g)
    Jo, go = _oracle_disp(eps.astype(np.float32).astype(np.float64), overlap)
    assert abs(J - Jo) <= 1e-5 * abs(Jo), (J, Jo)
    cos = float((g * go).sum() / (np.linalg.norm(g) * np.linalg.norm(go)))
    rel = float(np.linalg.norm(g - go) / np.linalg.norm(go))
    print("dispersive adjoint: J %.9g vs %.9g, cos %.8f, rel %.2e" % (J, Jo, cos, rel))
    assert cos >= 0.9999 and rel <= 1e-3, (cos, rel)
    if overlap:
        assert g[0, 1, 0, 2] == 0.0


@pytest.mark.gpu
def test_gpu_adjoint_dispersive_against_central_differences():
    """8 seeded design cells, h = 1e-3, with the dispersive blocks present."""
    eps = _eps().astype(np.float32)
    J, g, s = _gpu_disp(eps)
    s.close()
    rng = np.random.default_rng(9)
    cells = [tuple(int(v) for v in (rng.integers(3), *rng.integers(0, 3, size=3))) for _ in range(8)]
    fd, ad = [], []
    for cell in cells:
        h = 1e-3
        ep, em = eps.copy(), eps.copy()
        ep[cell] += h
        em[cell] -= h
        Jp, _, sp = _gpu_disp(ep)
        sp.close()
        Jm, _, sm = _gpu_disp(em)
        sm.close()
        fd.append((Jp - Jm) / (2 * h))
        ad.append(float(g[cell]))
    fd, ad = np.array(fd), np.array(ad)
    cos = float(fd @ ad / (np.linalg.norm(fd) * np.linalg.norm(ad)))
    assert cos >= 0.999, (cos, fd, ad)


def _gpu_gyro(eps, K=100, budget=-1, overlap=False):
    from dtmaxwell4_b200 import Simulation
    s = _setup(Simulation(_cfg(2)), 2)
    mats, idx = _gyro_materials(overlap=overlap)
    s.set_materials(mats, idx, idx, idx)
    s.set_design(LO, eps)
    s.set_adjoint_memory(budget)
    J, g = s.forward_adjoint(N_STEPS, PLANE_X, OMEGA, K)
    return J, g, s


@pytest.mark.gpu
def test_gpu_adjoint_gyrotropic_against_fp64_adjoint():
    """A magnetised-Drude block: the GPU adjoint of the gyrotropic current
    against the FP64 adjoint; recorded history and checkpointed recompute
    (odd interval: segments start on either current buffer) bit-identical
    with the final state of a plain run; a design region holding a
    gyrotropic node is refused."""
    from dtmaxwell4_b200 import DtmxError, Simulation
    eps = _eps()
    J, g, s = _gpu_gyro(eps)
    fin = [s.get_field(c) for c in range(6)]
    s.close()
    J2, g2, s2 = _gpu_gyro(eps, K=7, budget=0)
    fin2 = [s2.get_field(c) for c in range(6)]
    s2.step(5)
    s2.close()
    assert J2 == J and np.array_equal(g2, g)
    ref = _setup(Simulation(_cfg(2)), 2)
    mats, idx = _gyro_materials()
    ref.set_materials(mats, idx, idx, idx)
    ref.set_design(LO, eps)
    ref.step(N_STEPS)
    for c in range(6):
        assert np.array_equal(fin[c], ref.get_field(c)) and np.array_equal(fin2[c], fin[c])
    ref.close()
    Jo, go = _oracle_gyro(eps.astype(np.float32).astype(np.float64))
    assert abs(J - Jo) <= 1e-5 * abs(Jo), (J, Jo)
    cos = float((g * go).sum() / (np.linalg.norm(g) * np.linalg.norm(go)))
    rel = float(np.linalg.norm(g - go) / np.linalg.norm(go))
    print("gyrotropic adjoint: J %.9g vs %.9g, cos %.8f, rel %.2e" % (J, Jo, cos, rel))
    assert cos >= 0.9999 and rel <= 1e-3, (cos, rel)
    with pytest.raises(DtmxError):
        _gpu_gyro(eps, overlap=True)
