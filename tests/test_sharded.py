"""Slab sharding along x (dtmaxwell4_b200.sharded) on CPU ranks: world sizes
2 and 3 over gloo, each rank stepping its slab with the FP32 oracle as the
local engine and exchanging E planes with its neighbours every step, against
one single-domain FP32 oracle run of the whole grid: fields, probe traces and
DFT planes (normal to x and to y) bit for bit, with point sources and with a
plane-wave TF/SF source.  The partition rules and the
refused configurations are checked without processes."""
import os
import socket

import numpy as np
import pytest

NX, NY, NZ, STEPS = 31, 18, 20, 45


def _scenario():
    from dtmaxwell4_b200 import abi, scenarios
    cfg = abi.make_config(NX, NY, NZ, dx=1.0, courant=0.5, order=2, absorber=abi.ABS_CPML, pml=4,
                          probe_capacity=STEPS + 8)
    idx = np.zeros((NX, NY, NZ), np.uint8)
    idx[9:19, 5:12, 6:15] = 1
    idx[20:24, 3:9, 4:10] = 2
    wp = 2 * np.pi / 8
    mats = [abi.make_material(1.0), abi.make_material((4.0, 3.0, 2.5)),
            abi.make_material(1.0, poles=[(abi.POLE_DRUDE, 1.0, wp, wp / 50, 0.0)], eps_inf=1.0)]
    f0, tau, t0 = scenarios.gauss_sine_params(8.0)
    src = abi.PointSource(comp=abi.EZ, i=15, j=9, k=10, waveform=abi.WAVE_GAUSS_SINE, amp=1.0, f0=f0, tau=tau, t0=t0)
    probes = [(abi.EZ, 15, 9, 10), (abi.HY, 16, 8, 11), (abi.EX, 6, 9, 9), (abi.HZ, 27, 10, 8)]
    rng = np.random.default_rng(5)
    fields = [(1e-3 * rng.standard_normal((NX, NY, NZ))).astype(np.float32) for _ in range(6)]
    return cfg, mats, idx, src, probes, fields


def _apply(sim, mats, idx, src, probes, fields):
    from dtmaxwell4_b200 import abi
    sim.set_materials(mats, idx, idx, idx)
    sim.add_point_source(src)
    for (c, i, j, k) in probes:
        sim.add_probe(c, i, j, k)
    om = [0.5, 0.8]
    d0 = sim.add_dft_plane(0, 16, (1 << abi.EY) | (1 << abi.HZ), om)
    d1 = sim.add_dft_plane(1, 9, (1 << abi.EX) | (1 << abi.HX), om)
    for c in range(6):
        sim.set_field(c, fields[c])
    return d0, d1


class _OraclePlanes:
    """x planes of an oracle simulation, exchanged through host tensors."""

    def __init__(self, sim):
        self.sim = sim
        self.pending = []

    def send(self, comp, i):
        import torch
        return torch.from_numpy(np.ascontiguousarray(self.sim.get_field(comp)[i]).ravel())

    def recv(self, comp, i):
        import torch
        ny, nz = self.sim.shape[1:]
        buf = torch.empty(ny * nz, dtype=torch.float64)
        self.pending.append((comp, i, buf))
        return buf

    def commit(self):
        ny, nz = self.sim.shape[1:]
        for comp, i, buf in self.pending:
            a = self.sim.get_field(comp)
            a[i] = buf.numpy().reshape(ny, nz)
            self.sim.set_field(comp, a)
        self.pending = []


def _rank_main(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import pyoracle
    from dtmaxwell4_b200.sharded import ShardedSimulation
    os.environ["OMP_NUM_THREADS"] = "1"
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        cfg, mats, idx, src, probes, fields = _scenario()
        s = ShardedSimulation(cfg, make_local=lambda c: pyoracle.OracleSim(c, "f32"), planes=_OraclePlanes)
        d0, d1 = _apply(s, mats, idx, src, probes, fields)
        s.step(STEPS)
        res = dict(fields=np.stack([s.get_field(c) for c in range(6)]), probes=s.read_probes(),
                   dft0=s.read_dft(d0), dft1=s.read_dft(d1))
        if rank == 0:
            np.savez(os.path.join(out_dir, "w%d.npz" % world), **res)
        s.close()
    finally:
        dist.destroy_process_group()


def _rank_main_tfsf(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import pyoracle
    from dtmaxwell4_b200 import scenarios
    from dtmaxwell4_b200.sharded import ShardedSimulation
    os.environ["OMP_NUM_THREADS"] = "1"
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        sc = _tfsf_plane()
        s = ShardedSimulation(sc["cfg"], make_local=lambda c: pyoracle.OracleSim(c, "f32"), planes=_OraclePlanes)
        ids = scenarios.apply(s, sc)
        s.step(TFSF_STEPS)
        res = dict(fields=np.stack([s.get_field(c) for c in range(6)]), dft=s.read_dft(ids[0]))
        if rank == 0:
            np.savez(os.path.join(out_dir, "t%d.npz" % world), **res)
        s.close()
    finally:
        dist.destroy_process_group()


TFSF_STEPS = 60


def _tfsf_plane():
    """Plane-wave TF/SF Drude sphere, 40 cells along x (box faces near x = 12
    and 28), x-normal DFT plane."""
    from dtmaxwell4_b200 import scenarios
    return scenarios.drude_sphere_tfsf(n=(40, 36, 40), steps=TFSF_STEPS, pml=6, inset=6, radius=4, lambda0=10.0,
                                       nfreq=2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_equals_single_domain(world, tmp_path):
    import torch.multiprocessing as mp
    import pyoracle
    pyoracle.lib()
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(os.path.join(str(tmp_path), "w%d.npz" % world))
    cfg, mats, idx, src, probes, fields = _scenario()
    o = pyoracle.OracleSim(cfg, "f32")
    d0, d1 = _apply(o, mats, idx, src, probes, fields)
    o.step(STEPS)
    want = np.stack([o.get_field(c) for c in range(6)])
    assert np.abs(want).max() > 1e-3
    assert np.array_equal(got["fields"], want)
    assert np.array_equal(got["probes"], o.read_probes(STEPS + 8))
    assert np.array_equal(got["dft0"], o.read_dft(d0))
    assert np.array_equal(got["dft1"], o.read_dft(d1))
    o.close()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_tfsf_equals_single_domain(world, tmp_path):
    """A plane-wave TF/SF source across the ranks' slab faces: every rank
    takes the whole grid's box and 1-D line; bit for bit with one domain."""
    import torch.multiprocessing as mp
    import pyoracle
    from dtmaxwell4_b200 import scenarios
    pyoracle.lib()
    mp.start_processes(_rank_main_tfsf, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(os.path.join(str(tmp_path), "t%d.npz" % world))
    sc = _tfsf_plane()
    o = pyoracle.OracleSim(sc["cfg"], "f32")
    ids = scenarios.apply(o, sc)
    o.step(TFSF_STEPS)
    want = np.stack([o.get_field(c) for c in range(6)])
    assert np.abs(want).max() > 1e-4                  # the pulse's leading edge has entered the box
    assert np.array_equal(got["fields"], want)
    assert np.array_equal(got["dft"], o.read_dft(ids[0]))
    o.close()


def test_slab_plan_rules():
    from dtmaxwell4_b200 import abi
    from dtmaxwell4_b200.sharded import SlabPlan, slab_bounds
    assert [slab_bounds(10, 3, r) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    cfg = abi.make_config(40, 8, 8, pml=((5, 6), (2, 2), (2, 2)))
    plans = [SlabPlan(cfg, 3, r) for r in range(3)]
    assert [(p.lx0, p.nxl) for p in plans] == [(0, 15), (13, 15), (26, 14)]
    assert [tuple(p.cfg.pml[0]) for p in plans] == [(5, 0), (0, 0), (0, 6)]
    assert all(tuple(p.cfg.pml[1]) == (2, 2) for p in plans)
    with pytest.raises(ValueError):
        SlabPlan(abi.make_config(12, 8, 8, pml=6), 2, 1)        # 6 owned planes, 6-plane slab
    with pytest.raises(ValueError):
        SlabPlan(abi.make_config(40, 8, 8, order=4, courant=0.4), 2, 0)
    with pytest.raises(ValueError):
        SlabPlan(abi.make_config(40, 8, 8, absorber=abi.ABS_SPLIT_PML), 2, 0)


@pytest.mark.gpu
def test_device_planes_alias_the_fields():
    """The GPU plane accessor: a plane tensor reads the field in place and a
    received plane lands in the field (one GPU, no exchange)."""
    import torch
    from dtmaxwell4_b200 import Simulation, abi
    from dtmaxwell4_b200.sharded import DevicePlanes
    s = Simulation(abi.make_config(12, 10, 37, pml=2))
    a = np.random.default_rng(2).standard_normal((12, 10, 37)).astype(np.float32)
    s.set_field(abi.EY, a)
    s.sync()
    pl = DevicePlanes(s)
    nzp = s.device_ptr(abi.EY)[1][1]
    t = pl.send(abi.EY, 5)
    assert t.numel() == 10 * nzp and t.is_cuda
    assert np.array_equal(t.view(10, nzp)[:, :37].cpu().numpy(), a[5])
    r = pl.recv(abi.EY, 7)
    with torch.cuda.stream(pl.stream):
        r.view(10, nzp)[:, :37].copy_(torch.from_numpy(a[3]).cuda())
    pl.stream.synchronize()
    assert np.array_equal(s.get_field(abi.EY)[7], a[3])
    s.close()


@pytest.mark.gpu
def test_sharded_single_rank_is_the_plain_run():
    from dtmaxwell4_b200 import Simulation
    from dtmaxwell4_b200.sharded import ShardedSimulation
    cfg, mats, idx, src, probes, fields = _scenario()
    a = ShardedSimulation(cfg)
    b = Simulation(cfg)
    da = _apply(a, mats, idx, src, probes, fields)
    db = _apply(b, mats, idx, src, probes, fields)
    a.step(STEPS)
    b.step(STEPS)
    for c in range(6):
        assert np.array_equal(a.get_field(c), b.get_field(c))
    assert np.array_equal(a.read_probes(), b.read_probes())
    assert np.array_equal(a.read_dft(da[1]), b.read_dft(db[1]))
    a.close()
    b.close()
