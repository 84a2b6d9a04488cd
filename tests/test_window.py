"""Out-of-core runs (dtmaxwell4_b200.window): a grid stepped as x slabs that
take turns on the device, each slab parked in host memory between its turns.

CPU: the slab walk with the FP32 oracle as the slab engine (its
read_planes / write_planes restate the library's plane-state layout; parking
is a no-op there) against one single-domain FP32 oracle run -- fields, probe
traces and an x-normal DFT plane bit for bit, for 2 and 3 slabs and 1 to 5
time steps per turn (a Drude block crosses a slab face, the dipole sits in a
neighbour's ghost planes).
DFT planes normal to x (one owner) and to y (every slab's own rows).
GPU: dtmx_park / dtmx_unpark keep the state bit for bit and free the device
memory while parked, a parked context refuses its calls, dtmx_read_planes /
dtmx_write_planes round-trip and match the oracle's layout, and a 3-slab
out-of-core run equals the plain in-core run bit for bit on both field
engines.
"""
import numpy as np
import pytest

from test_sharded import NX, NY, NZ, STEPS, _scenario


def _apply(sim, mats, idx, src, probes, fields):
    from dtmaxwell4_b200 import abi
    sim.set_materials(mats, idx, idx, idx)
    sim.add_point_source(src)
    for (c, i, j, k) in probes:
        sim.add_probe(c, i, j, k)
    d0 = sim.add_dft_plane(0, 16, (1 << abi.EY) | (1 << abi.HZ), [0.5, 0.8])
    d1 = sim.add_dft_plane(1, 9, (1 << abi.EX) | (1 << abi.HX), [0.5, 0.8])
    for c in range(6):
        sim.set_field(c, fields[c])
    return d0, d1


@pytest.mark.parametrize("nslabs,K,resident", [(2, 4, 1), (3, 1, 1), (3, 5, 2)])
def test_window_equals_single_domain(nslabs, K, resident):
    import pyoracle
    from dtmaxwell4_b200.window import OutOfCoreSimulation
    cfg, mats, idx, src, probes, fields = _scenario()
    parked = []
    w = OutOfCoreSimulation(cfg, nslabs, steps_per_turn=K, make_local=lambda c: pyoracle.OracleSim(c, "f32"),
                            park=lambda s: parked.append(s), unpark=lambda s: None, resident=resident)
    d0 = _apply(w, mats, idx, src, probes, fields)
    w.step(STEPS)
    turns = -(-STEPS // K)
    assert w.turns == turns
    assert len(parked) == nslabs * (turns + 1)        # every slab parked after set-up and after each turn
    o = pyoracle.OracleSim(cfg, "f32")
    do = _apply(o, mats, idx, src, probes, fields)
    o.step(STEPS)
    for c in range(6):
        want = o.get_field(c)
        assert np.abs(want).max() > 1e-4
        assert np.array_equal(w.get_field(c), want), c
    assert np.array_equal(w.read_probes(), o.read_probes(STEPS + 8))
    for a, b in zip(d0, do):                          # x-normal (owner) and y-normal (every slab's rows)
        assert np.array_equal(w.read_dft(a), o.read_dft(b))
    o.close()
    w.close()


def test_window_single_slab_and_short_turns():
    """One slab (no ghost planes) and a run shorter than one turn are the
    single-domain run."""
    import pyoracle
    from dtmaxwell4_b200.window import OutOfCoreSimulation
    cfg, mats, idx, src, probes, fields = _scenario()
    o = pyoracle.OracleSim(cfg, "f32")
    _apply(o, mats, idx, src, probes, fields)
    o.step(7)
    for nslabs, K in ((1, 4), (2, 8)):
        w = OutOfCoreSimulation(cfg, nslabs, steps_per_turn=K, make_local=lambda c: pyoracle.OracleSim(c, "f32"))
        _apply(w, mats, idx, src, probes, fields)
        w.step(3)
        w.step(4)
        assert w.turns == 2                           # one turn per call: 3 and 4 steps
        for c in range(6):
            assert np.array_equal(w.get_field(c), o.get_field(c)), (nslabs, K, c)
        w.close()
    o.close()


def test_window_refusals():
    from dtmaxwell4_b200 import abi
    from dtmaxwell4_b200.window import OutOfCoreSimulation
    cfg = _scenario()[0]
    w = OutOfCoreSimulation(cfg, 2, make_local=lambda c: None)
    with pytest.raises(ValueError):
        w.set_design((0, 0, 0), None)
    gyro = abi.make_material(1.0, eps_inf=1.0, gyro=(0.3, 0.01, 0.2))
    with pytest.raises(ValueError):
        w.set_materials([gyro], np.zeros((NX, NY, NZ), np.uint8))
    with pytest.raises(ValueError):                   # 6 owned planes, a 9-plane halo
        OutOfCoreSimulation(abi.make_config(12, 8, 8, pml=2), 2, steps_per_turn=8, make_local=lambda c: None)
    with pytest.raises(ValueError):                   # slab 1's ghost planes reach the 6-plane x absorber
        OutOfCoreSimulation(abi.make_config(40, 8, 8, pml=6), 3, steps_per_turn=8, make_local=lambda c: None)
    OutOfCoreSimulation(abi.make_config(40, 8, 8, pml=6), 3, steps_per_turn=4, make_local=lambda c: None)
    with pytest.raises(ValueError):
        OutOfCoreSimulation(abi.make_config(40, 8, 8, order=4, courant=0.4), 2, make_local=lambda c: None)


def test_oracle_plane_state_round_trip():
    """The oracle's plane state: sizes per section, fields as get_field,
    zero ADE sections off the dispersive box, write then read is identity."""
    import pyoracle
    cfg, mats, idx, src, probes, fields = _scenario()
    o = pyoracle.OracleSim(cfg, "f32")
    _apply(o, mats, idx, src, probes, fields)
    o.step(7)
    nyz = NY * NZ
    L = 4                                             # CPML cells per face
    assert o.plane_state_floats() == 6 * nyz + 4 * 2 * L * NZ + 4 * NY * 2 * L + 3 * (1 + 2 * 1) * nyz
    st = o.read_planes(8, 5)
    f = st[:6 * 5 * nyz].reshape(6, 5, NY, NZ)
    for c in range(6):
        assert np.array_equal(f[c], o.get_field(c)[8:13])
    ade = st[-3 * 3 * 5 * nyz:].reshape(3, 3, 5, NY, NZ)
    assert not ade.any()                              # planes 8..12 hold no Drude node
    st2 = o.read_planes(19, 4)
    assert st2[-3 * 3 * 4 * nyz:].any()               # the Drude block 20..23 has current after 7 steps
    p = o.read_planes(4, 3)
    q = p * 1.5
    o.write_planes(4, 3, q)
    assert np.array_equal(o.read_planes(4, 3), q.astype(np.float32).astype(np.float64))
    with pytest.raises(ValueError):
        o.read_planes(2, 3)                           # inside the x absorber slab
    o.close()


@pytest.mark.gpu
def test_park_round_trip_frees_device_memory():
    import torch
    from dtmaxwell4_b200 import Simulation, abi
    from dtmaxwell4_b200.engine import DtmxError
    cfg, mats, idx, src, probes, fields = _scenario()
    pc = abi.make_config(NX, NY, NZ, dx=1.0, courant=0.5, order=2, absorber=abi.ABS_CPML, pml=4,
                         probe_capacity=STEPS + 8, parkable=True)
    a, b = Simulation(pc), Simulation(cfg)
    da, db = _apply(a, mats, idx, src, probes, fields), _apply(b, mats, idx, src, probes, fields)
    a.step(STEPS // 2)
    b.step(STEPS // 2)
    a.park()
    with pytest.raises(DtmxError):
        a.step(1)
    with pytest.raises(DtmxError):
        a.get_field(abi.EX)
    a.park()                                            # parking twice is a no-op
    a.unpark()
    a.unpark()
    a.step(STEPS - STEPS // 2)
    b.step(STEPS - STEPS // 2)
    for c in range(6):
        assert np.array_equal(a.get_field(c), b.get_field(c)), c
    assert np.array_equal(a.read_probes(), b.read_probes())
    for x, y in zip(da, db):
        assert np.array_equal(a.read_dft(x), b.read_dft(y))
    with pytest.raises(DtmxError):
        b.park()                                        # not created parkable
    a.close()
    b.close()
    # a 256^3 context: its arrays leave the device while parked
    big = Simulation(abi.make_config(256, 256, 256, pml=8, parkable=True))
    big.step(2)
    big.sync()
    torch.cuda.synchronize()
    f0 = torch.cuda.mem_get_info()[0]
    big.park()
    f1 = torch.cuda.mem_get_info()[0]
    big.unpark()
    f2 = torch.cuda.mem_get_info()[0]
    assert f1 - f0 >= 6 * 256 ** 3 * 4, (f0, f1)
    assert abs(f2 - f0) < 64 << 20, (f0, f2)
    big.step(1)
    assert big.check_finite()
    big.close()


@pytest.mark.gpu
@pytest.mark.parametrize("engine,resident", [(1, 1), (3, 1), (3, 2)])
def test_window_equals_in_core_run(engine, resident):
    from dtmaxwell4_b200 import Simulation, abi
    from dtmaxwell4_b200.window import OutOfCoreSimulation
    cfg, mats, idx, src, probes, fields = _scenario()

    def make(c):
        from dtmaxwell4_b200.window import parkable_simulation
        s = parkable_simulation(c)
        s.set_engine(engine, 0)
        return s
    w = OutOfCoreSimulation(cfg, 3, steps_per_turn=5, make_local=make, park=lambda s: s.park(),
                            unpark=lambda s: s.unpark(), resident=resident)
    b = Simulation(cfg)
    b.set_engine(engine, 0)
    dw, db = _apply(w, mats, idx, src, probes, fields), _apply(b, mats, idx, src, probes, fields)
    w.step(STEPS)
    b.step(STEPS)
    for c in range(6):
        want = b.get_field(c)
        assert np.abs(want).max() > 1e-4
        assert np.array_equal(w.get_field(c), want), c
    assert np.array_equal(w.read_probes(), b.read_probes().astype(np.float64))
    for x, y in zip(dw, db):
        assert np.array_equal(w.read_dft(x), b.read_dft(y))
    w.close()
    b.close()


@pytest.mark.gpu
def test_gpu_plane_state_layout():
    """dtmx_read_planes: the oracle's section sizes, fields as dtmx_get_field,
    ADE sections zero off the Drude block and nonzero on it; a written state
    reads back unchanged (pinned output buffer too)."""
    import pyoracle
    import torch
    from dtmaxwell4_b200 import Simulation
    cfg, mats, idx, src, probes, fields = _scenario()
    g = Simulation(cfg)
    o = pyoracle.OracleSim(cfg, "f32")
    _apply(g, mats, idx, src, probes, fields)
    _apply(o, mats, idx, src, probes, fields)
    g.step(7)
    nyz = NY * NZ
    assert g.plane_state_floats() == o.plane_state_floats()
    st = g.read_planes(8, 5)
    f = st[:6 * 5 * nyz].reshape(6, 5, NY, NZ)
    for c in range(6):
        assert np.array_equal(f[c], g.get_field(c)[8:13])
    assert not st[-9 * 5 * nyz:].any()
    assert g.read_planes(19, 4)[-9 * 4 * nyz:].any()
    pinned = torch.empty(g.plane_state_floats() * 4, dtype=torch.float32).pin_memory().numpy()
    p = g.read_planes(19, 4, out=pinned).copy()
    q = (p * 1.5).astype(np.float32)
    g.write_planes(19, 4, q)
    assert np.array_equal(g.read_planes(19, 4), q)
    g.write_planes(19, 4, p)
    g.close()
    o.close()


@pytest.mark.gpu
def test_park_pool_keeps_and_releases_memory():
    """dtmx_set_park_pool: parked memory stays with the process up to the
    limit and serves the next unpark; lowering the limit releases it."""
    import torch
    from dtmaxwell4_b200 import Simulation, abi, engine
    dev = torch.cuda.current_device()
    s = Simulation(abi.make_config(256, 256, 256, pml=8, parkable=True))
    s.step(2)
    s.sync()
    a = np.asarray(s.get_field(abi.EZ)).copy()
    engine.set_park_pool(-1, dev)
    try:
        torch.cuda.synchronize()
        f0 = torch.cuda.mem_get_info()[0]
        s.park()
        f1 = torch.cuda.mem_get_info()[0]
        assert abs(f1 - f0) < 64 << 20, (f0, f1)           # kept in the pool
        s.unpark()
        f2 = torch.cuda.mem_get_info()[0]
        assert abs(f2 - f0) < 64 << 20, (f0, f2)           # served from the pool
        assert np.array_equal(s.get_field(abi.EZ), a)
        s.park()
        engine.set_park_pool(0, dev)
        f3 = torch.cuda.mem_get_info()[0]
        assert f3 - f0 >= 6 * 256 ** 3 * 4, (f0, f3)       # released
        s.unpark()
        s.step(1)
        assert s.check_finite()
    finally:
        engine.set_park_pool(0, dev)
        s.close()


def _tfsf_scenario(kind):
    """A plane-wave TF/SF Drude sphere with an x-normal DFT plane, or a
    dipole TF/SF box over a dielectric layer; 40-48 cells along x, 6-cell CPML."""
    from dtmaxwell4_b200 import abi, scenarios
    if kind == "plane":
        sc = scenarios.drude_sphere_tfsf(n=(40, 36, 40), steps=70, pml=6, inset=6, radius=4, lambda0=10.0, nfreq=2)
        sc["probes"] = [(abi.EZ, 20, 18, 16, abi.PROBE_NODE), (abi.HY, 13, 17, 15, abi.PROBE_NODE),
                        (abi.EZ, 29, 18, 16, abi.PROBE_NODE)]
        return sc, 70
    cfg = abi.make_config(48, 45, 40, dx=1.0, courant=0.5, order=2, pml=6, probe_capacity=100)
    t = abi.TFSF()
    t.kind = abi.TFSF_DIPOLE
    t.box_lo[:] = [18.3, 17.4, 15.2]
    t.box_hi[:] = [28.6, 27.9, 24.7]
    t.c, t.w, t.kenv, t.tstop, t.ntime = 1.0, 2 * np.pi / 10, 0.3, 0.0, 1
    layer = np.zeros((48, 45, 40), np.uint8)
    layer[:, :, :10] = 1
    sc = dict(cfg=cfg, materials=([abi.make_material(1.0), abi.make_material(2.25)], [layer] * 3), tfsf=t,
              probes=[(abi.EZ, 23, 22, 20, abi.PROBE_NODE), (abi.HX, 30, 22, 12, abi.PROBE_NODE)],
              dft=[(0, 33, (1 << abi.EZ) | (1 << abi.HY), [0.5])], point_sources=[])
    return sc, 60


@pytest.mark.parametrize("kind,K,resident", [("plane", 3, 1), ("plane", 2, 2), ("dipole", 3, 2)])
def test_window_tfsf_equals_single_domain(kind, K, resident):
    """TF/SF sources across slab faces (the box's x faces fall in owned and
    ghost planes of different slabs): bit for bit with one domain."""
    import pyoracle
    from dtmaxwell4_b200 import scenarios
    from dtmaxwell4_b200.window import OutOfCoreSimulation
    sc, steps = _tfsf_scenario(kind)
    w = OutOfCoreSimulation(sc["cfg"], 3, steps_per_turn=K, make_local=lambda c: pyoracle.OracleSim(c, "f32"),
                            resident=resident)
    dw = scenarios.apply(w, sc)
    w.step(steps)
    o = pyoracle.OracleSim(sc["cfg"], "f32")
    do = scenarios.apply(o, sc)
    o.step(steps)
    for c in range(6):
        want = o.get_field(c)
        assert np.array_equal(w.get_field(c), want), c
    assert np.abs(o.get_field(2)).max() > 1e-4
    assert np.array_equal(w.read_probes(), o.read_probes(100000))
    for a, b in zip(dw, do):
        assert np.array_equal(w.read_dft(a), o.read_dft(b))
    o.close()
    w.close()


def test_tfsf_x_origin_checks():
    """A slab takes the whole grid's TF/SF box; bad origins are refused, and
    the boundary check applies at the grid's uncut x ends only."""
    import pyoracle
    from dtmaxwell4_b200 import abi
    sc, _ = _tfsf_scenario("dipole")
    t = sc["tfsf"]
    lc = abi.make_config(20, 45, 40, dx=1.0, courant=0.5, order=2, pml=((0, 0), (6, 6), (6, 6)))
    o = pyoracle.OracleSim(lc, "f32")
    q = abi.TFSF()
    C = __import__("ctypes")
    C.memmove(C.byref(q), C.byref(t), C.sizeof(abi.TFSF))
    q.x_origin, q.x_cells = 40.0, 48.0                # 40 + 20 > 48
    assert o._f("set_tfsf")(o._h, C.byref(q)) != 0
    q.x_origin = 14.5
    assert o._f("set_tfsf")(o._h, C.byref(q)) != 0
    q.x_origin = 14.0
    assert o._f("set_tfsf")(o._h, C.byref(q)) == 0
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind,engine", [("plane", 3), ("plane", 1), ("dipole", 3)])
def test_window_tfsf_equals_in_core_run(kind, engine):
    from dtmaxwell4_b200 import Simulation, abi, scenarios
    from dtmaxwell4_b200.window import OutOfCoreSimulation, parkable_simulation
    sc, steps = _tfsf_scenario(kind)

    def make(c):
        s = parkable_simulation(c)
        s.set_engine(engine, 0)
        return s
    w = OutOfCoreSimulation(sc["cfg"], 3, steps_per_turn=3, make_local=make, resident=2)
    b = Simulation(sc["cfg"])
    b.set_engine(engine, 0)
    dw, db = scenarios.apply(w, sc), scenarios.apply(b, sc)
    w.step(steps)
    b.step(steps)
    for c in range(6):
        assert np.array_equal(w.get_field(c), b.get_field(c)), c
    assert np.abs(b.get_field(abi.EZ)).max() > 1e-4
    assert np.array_equal(w.read_probes(), b.read_probes().astype(np.float64))
    for x, y in zip(dw, db):
        assert np.array_equal(w.read_dft(x), b.read_dft(y))
    w.close()
    b.close()


@pytest.mark.gpu
def test_copy_planes_between_parked_and_live_contexts():
    """dtmx_copy_planes gives the planes dtmx_read_planes / dtmx_write_planes
    would move, whether the source or the destination is parked."""
    from dtmaxwell4_b200 import Simulation, abi
    cfg, mats, idx, src, probes, fields = _scenario()
    pc = abi.make_config(NX, NY, NZ, dx=1.0, courant=0.5, order=2, absorber=abi.ABS_CPML, pml=4,
                         probe_capacity=STEPS + 8, parkable=True)
    a, b = Simulation(pc), Simulation(pc)
    _apply(a, mats, idx, src, probes, fields)
    _apply(b, mats, idx, src, probes, fields)
    a.step(11)
    b.step(5)
    # the same planes of both grids (the same materials there, as for two slabs' shared planes)
    want = a.read_planes(18, 4)                      # planes 18..21: dielectric, Drude nodes, CPML rows
    assert not np.array_equal(b.read_planes(18, 4), want)
    b.park()
    b.copy_planes(18, a, 18, 4)                      # live source, parked destination
    b.unpark()
    assert np.array_equal(b.read_planes(18, 4), want)
    b.step(2)
    a.park()
    b.copy_planes(18, a, 18, 4)                      # parked source, live destination
    assert np.array_equal(b.read_planes(18, 4), want)
    a.unpark()
    assert np.array_equal(a.read_planes(18, 4), want)
    a.close()
    b.close()
