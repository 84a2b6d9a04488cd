"""Wavefront engine (several time steps per launch, working set in L2)
against the one-launch-per-half-step engine.

Both engines evaluate the same expressions in the same order, so from the
same seeded state they must agree bit for bit: dielectric and Drude
materials, CPML slabs, partial tiles along y and z, both stencil orders,
several steps per launch plus a remainder run by the per-step engine.  The
per-step engine itself is checked against the FP64 oracle in
test_gpu_parity.py; one case here also goes to the oracle directly.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case(nx, ny, nz, order, pml=8):
    from dtmaxwell4_b200 import abi
    cfg = abi.make_config(nx, ny, nz, dx=1.0, courant=0.4 if order == 4 else 0.5, order=order,
                          absorber=abi.ABS_CPML, pml=pml)
    wp = 2 * np.pi / 8
    mats = [abi.make_material(1.0), abi.make_material(4.0),
            abi.make_material(1.0, poles=[(abi.POLE_DRUDE, 1.0, wp, wp / 50, 0.0)], eps_inf=1.0)]
    idx = np.zeros((nx, ny, nz), np.uint8)
    idx[nx // 4:nx // 2, ny // 3:2 * ny // 3, 10:30] = 1
    x, y, z = np.ogrid[:nx, :ny, :nz]
    idx[(x - 2 * nx // 3) ** 2 + (y - ny // 2) ** 2 + (z - nz // 2) ** 2 < 8 ** 2] = 2
    rng = np.random.default_rng(7)
    fields = [rng.standard_normal((nx, ny, nz)).astype(np.float32) for _ in range(6)]
    return cfg, mats, idx, fields


def _run(cfg, mats, idx, fields, steps, engine, T=0):
    from dtmaxwell4_b200 import Simulation
    s = Simulation(cfg)
    s.set_materials(mats, idx, idx, idx)
    for c in range(6):
        s.set_field(c, fields[c])
    if engine:
        s.set_engine(engine, T)
    s.step(steps)
    s.sync()
    out = [s.get_field(c) for c in range(6)]
    s.close()
    return out


@pytest.mark.parametrize("order,T", [(2, 1), (2, 2), (2, 4), (4, 1), (4, 2)])
def test_wavefront_bitwise_equal_to_per_step_engine(order, T):
    cfg, mats, idx, fields = _case(56, 64, 80, order)
    steps = 3 * T + 1
    ref = _run(cfg, mats, idx, fields, steps, 1)
    got = _run(cfg, mats, idx, fields, steps, 2, T)
    for c in range(6):
        bad = np.argwhere(got[c] != ref[c])
        assert bad.size == 0, (c, bad[:5], float(np.abs(got[c] - ref[c]).max()))


def test_wavefront_against_oracle():
    import pyoracle
    from dtmaxwell4_b200 import abi
    cfg, mats, idx, fields = _case(40, 32, 48, 4, pml=6)
    got = _run(cfg, mats, idx, fields, 12, 2, 2)
    o = pyoracle.OracleSim(cfg)
    o.set_materials(mats, idx, idx, idx)
    for c in range(6):
        o.set_field(c, fields[c])
    o.step(12)
    for c in range(6):
        assert rel_l2(got[c], o.get_field(c)) < 3e-6, c
