"""Single-sweep engine (engine 3: H and E in one launch per step, two field
buffers) against the one-launch-per-half-step engine and the FP64 oracle.

Without a TF/SF source both engines evaluate the same node expressions in
the same order, so from the same seeded state they agree bit for bit:
dielectric, Drude and gyrotropic materials, a design region, CPML slabs,
partial tiles along y and z, x-chunk boundaries, odd step counts and the
16-step graph replay from either buffer, switching engines mid-run, probes,
DFT planes and a saved/restored state.  With a TF/SF source the single-sweep
engine adds the H correction to the old H (the update is linear in it), so
it is held to the FP64 oracle instead.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(nx=56, ny=61, nz=70, gyro=False, design=False):
    from dtmaxwell4_b200 import abi
    cfg = abi.make_config(nx, ny, nz, dx=1.0, courant=0.5, order=2, absorber=abi.ABS_CPML, pml=7)
    wp = 2 * np.pi / 8
    mats = [abi.make_material(1.0), abi.make_material((4.0, 3.0, 2.5)),
            abi.make_material(1.0, poles=[(abi.POLE_DRUDE, 1.0, wp, wp / 50, 0.0)], eps_inf=1.0)]
    if gyro:
        einf, g = abi.gyro_for(4.0, 0.3, 2 * np.pi / 20)
        mats.append(abi.make_material(1.0, eps_inf=einf, gyro=g))
    idx = np.zeros((nx, ny, nz), np.uint8)
    idx[nx // 4:nx // 2, ny // 3:2 * ny // 3, 10:30] = 1
    x, y, z = np.ogrid[:nx, :ny, :nz]
    idx[(x - 2 * nx // 3) ** 2 + (y - ny // 2) ** 2 + (z - nz // 2) ** 2 < 8 ** 2] = 2
    if gyro:
        idx[8:nx - 8, 8:ny - 8, nz - 22:nz - 12] = 3
    rng = np.random.default_rng(11)
    fields = [rng.standard_normal((nx, ny, nz)).astype(np.float32) for _ in range(6)]
    des = None
    if design:
        des = ((20, 17, 33), 1.0 + 3.0 * rng.random((3, 9, 14, 20)).astype(np.float32))
    return cfg, mats, idx, fields, des


def _sim(case, engine):
    from dtmaxwell4_b200 import Simulation
    cfg, mats, idx, fields, des = case
    s = Simulation(cfg)
    s.set_materials(mats, idx, idx, idx)
    if des is not None:
        s.set_design(*des)
    for c in range(6):
        s.set_field(c, fields[c])
    s.set_engine(engine, 0)
    return s


def _fields(s):
    s.sync()
    return [s.get_field(c) for c in range(6)]


def _same(got, ref):
    for c in range(6):
        bad = np.argwhere(got[c] != ref[c])
        assert bad.size == 0, (c, bad[:5], float(np.abs(got[c] - ref[c]).max()))


@pytest.mark.parametrize("gyro,design", [(False, False), (True, False), (False, True)])
def test_single_sweep_bitwise_equal_to_per_step(gyro, design):
    case = _case(gyro=gyro, design=design)
    a = _sim(case, 1)
    b = _sim(case, 3)
    # 5 (odd: the state ends in the second buffer), 16 (one graph replay from it), 16, 3
    for n in (5, 16, 16, 3):
        a.step(n)
        b.step(n)
        _same(_fields(b), _fields(a))
    a.close()
    b.close()


@pytest.mark.parametrize("xchunk", [1, 5, 13, 64])
def test_single_sweep_x_chunks(xchunk):
    """Chunk boundaries anywhere along x (one plane per CTA up to the longest
    chunk, 64 planes, which here is the whole grid) give the same fields."""
    case = _case()
    a = _sim(case, 1)
    b = _sim(case, 3)
    b.set_xchunk(xchunk)
    a.step(11)
    b.step(11)
    _same(_fields(b), _fields(a))
    a.close()
    b.close()


def test_engines_switch_mid_run_and_state_files(tmp_path):
    case = _case()
    ref = _sim(case, 1)
    ref.step(29)
    want = _fields(ref)
    ref.close()
    s = _sim(case, 3)
    s.step(7)                     # state in the second buffer
    s.set_engine(1, 0)
    s.step(9)                     # per-step engine from the second buffer
    s.set_engine(3, 0)
    s.step(3)
    path = str(tmp_path / "state.bin")
    s.save_state(path)
    s2 = _sim(case, 3)
    s2.load_state(path)
    s2.step(10)
    s.step(10)
    _same(_fields(s), want)
    _same(_fields(s2), want)
    s.close()
    s2.close()


def test_monitors_match_per_step():
    from dtmaxwell4_b200 import abi
    case = _case()
    sims = []
    for eng in (1, 3):
        s = _sim(case, eng)
        s.add_probe(abi.EZ, 30, 30, 35)
        s.add_probe(abi.HY, 12, 50, 9)
        s.add_dft_plane(0, 40, (1 << abi.EY) | (1 << abi.HZ), [0.3, 0.5])
        s.step(37)
        s.sync()
        sims.append((s.read_probes(), s.read_dft(0)))
        s.close()
    assert np.array_equal(sims[0][0], sims[1][0])
    assert np.array_equal(sims[0][1], sims[1][1])


@pytest.mark.parametrize("kind,engine", [("plane", 3), ("dipole", 3), ("dipole", 1)])
def test_single_sweep_tfsf_against_oracle(kind, engine):
    import pyoracle
    from dtmaxwell4_b200 import Simulation, abi, scenarios
    if kind == "plane":
        sc = scenarios.drude_sphere_tfsf(n=(48, 45, 40), steps=150, pml=6, inset=6, radius=6, lambda0=10.0, nfreq=2)
        steps = 150
    else:
        cfg = abi.make_config(48, 45, 40, dx=1.0, courant=0.5, order=2, pml=6)
        t = abi.TFSF()
        t.kind = abi.TFSF_DIPOLE
        t.box_lo[:] = [18.3, 17.4, 15.2]
        t.box_hi[:] = [28.6, 27.9, 24.7]
        t.c, t.w, t.kenv, t.tstop, t.ntime = 1.0, 2 * np.pi / 10, 0.3, 0.0, 1
        slab = np.zeros((48, 45, 40), np.uint8)
        slab[:, :, :10] = 1                     # a dielectric layer below the box
        sc = dict(cfg=cfg, materials=([abi.make_material(1.0), abi.make_material(2.25)], [slab] * 3),
                  tfsf=t, probes=[], dft=[], point_sources=[])
        steps = 120
    g = Simulation(sc["cfg"])
    o = pyoracle.OracleSim(sc["cfg"])
    scenarios.apply(g, sc)
    scenarios.apply(o, sc)
    g.set_engine(engine, 0)
    g.step(steps)
    o.step(steps)
    # each component against the norm of its whole field (E or H): a z dipole
    # has no Hz, whose own norm is round-off
    got = [g.get_field(c).astype(np.float64) for c in range(6)]
    want = [o.get_field(c) for c in range(6)]
    for grp in ((0, 1, 2), (3, 4, 5)):
        ref = np.sqrt(sum(np.linalg.norm(want[c]) ** 2 for c in grp))
        for c in grp:
            err = np.linalg.norm(got[c] - want[c]) / ref
            assert err <= 1e-5, (c, err)
    g.close()


@pytest.mark.parametrize("budget", [-1, 0])
def test_single_sweep_forward_adjoint_matches_per_step(budget):
    """dtmx_forward_adjoint steps its forward pass and recomputed segments with
    the selected engine: the single sweep (Drude sphere, CPML, design region)
    gives the objective, gradient and final state of the per-step engine."""
    case = _case(design=True)
    res = []
    for eng in (1, 3):
        s = _sim(case, eng)
        s.set_adjoint_memory(budget)
        J, g = s.forward_adjoint(25, 40, 2 * np.pi / 10, 7)
        res.append((J, g, _fields(s)))
        s.close()
    assert res[0][0] == res[1][0] and np.array_equal(res[0][1], res[1][1])
    _same(res[1][2], res[0][2])


@pytest.mark.parametrize("gyro,design,xchunk", [(False, False, 0), (True, False, 3), (False, True, 7)])
def test_single_sweep_8_row_tiles(gyro, design, xchunk):
    """8-row tiles (the autotuner's choice for small grids): bit-identical to
    the per-step engine, including partial tiles, CPML slabs, materials,
    design region and gyrotropic layer."""
    case = _case(gyro=gyro, design=design)
    a = _sim(case, 1)
    b = _sim(case, 3)
    b.set_tile_rows(8)
    b.set_xchunk(xchunk)
    assert b.engine_config()[3] == 8
    for n in (5, 16):
        a.step(n)
        b.step(n)
        _same(_fields(b), _fields(a))
    a.close()
    b.close()
