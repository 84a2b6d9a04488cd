"""Out-of-core runs: a grid larger than the device, stepped as x slabs that
take turns on one GPU, several time steps per turn.

The reference keeps its domain in pinned host memory and streams it through
the device window by window, Ntime time steps per pass (window.hpp:177-267,
params.h:12, params.h:50-52).  Here the grid is cut into x slabs (the split
of sharded.slab_bounds); each slab is a context created parkable (dtmx_park /
dtmx_unpark move its arrays to pinned host memory and back at the same device
addresses) whose local grid carries K + 1 ghost planes on each side that has
a neighbour.  One turn of slab r at time n:

  unpark (its lower ghost planes already hold slab r - 1's last owned planes
  of time n, left in its parked state by r - 1's turn); copy slab r + 1's
  first owned planes into its upper ghost planes and its own last owned
  planes into slab r + 1's lower ghost planes, straight between the device
  and r + 1's parked host copy (the full plane state: fields, y/z CPML
  auxiliaries, ADE currents -- dtmx_copy_planes); step k <= K times; park.
  No edge buffers, one copy of K + 1 planes each way per turn.

Why it is exact: a local order-2 step is wrong only next to the local grid's
faces (one plane at each cut face per step), so after k <= K steps the planes
from the second ghost plane inward still equal the single-domain run's, bit
for bit -- the owned planes and one plane beyond them at every step of the
turn (which probes and DFT planes of the owned planes may read).  Point
sources act in every slab whose local grid holds them, ghost planes
included, and a TF/SF source in every slab (its box and its plane wave's 1-D
line in whole-grid coordinates, dtmx_tfsf.x_origin); probes and x-normal DFT
planes in the slab that owns their plane, y- and z-normal DFT planes in every
slab over its own rows.

Only `resident` slabs' state is on the device at a time (one by default), so
the grid may be as large as host memory allows; a turn moves the slab's state
across the host link twice, once per K time steps (the reference's cadence is
Ntime = NS - 3).
Restrictions: order 2, box geometry with a CPML or no absorber, no
gyrotropic material or design region, and ghost planes outside the x
absorber slabs.
"""
import ctypes as C

import numpy as np

from . import abi
from .sharded import slab_bounds


class WindowSlab:
    """One slab of an out-of-core run: owned planes [x0, x1), local grid
    [lx0, lx0 + nxl) with halo ghost planes toward each neighbour."""

    def __init__(self, cfg, nslabs, rank, halo):
        if cfg.order != 2:
            raise ValueError("out-of-core runs support the order-2 stencil only")
        if cfg.geometry != abi.GEOM_BOX or cfg.absorber == abi.ABS_SPLIT_PML:
            raise ValueError("out-of-core runs support the box geometry with a CPML or no absorber")
        if halo < 1:
            raise ValueError("halo must be >= 1")
        self.rank, self.nslabs, self.halo = rank, nslabs, halo
        self.x0, self.x1 = slab_bounds(cfg.nx, nslabs, rank)
        self.glo = halo if rank > 0 else 0
        self.ghi = halo if rank < nslabs - 1 else 0
        self.lx0 = self.x0 - self.glo
        self.nxl = self.x1 - self.x0 + self.glo + self.ghi
        pml = (0, 0) if cfg.absorber == abi.ABS_NONE else tuple(cfg.pml[0])
        if nslabs > 1 and self.x1 - self.x0 < halo:
            raise ValueError("slab %d owns %d planes: it needs at least the halo (%d)" % (rank, self.x1 - self.x0, halo))
        if (self.glo and self.lx0 < pml[0]) or (self.ghi and self.x1 + self.ghi > cfg.nx - pml[1]):
            raise ValueError("slab %d: ghost planes inside an x absorber slab" % rank)
        lc = abi.Config()
        C.memmove(C.byref(lc), C.byref(cfg), C.sizeof(abi.Config))
        lc.nx = self.nxl
        lc.pml[0][0] = pml[0] if rank == 0 else 0
        lc.pml[0][1] = pml[1] if rank == nslabs - 1 else 0
        self.cfg = lc

    def owns(self, i):
        return self.x0 <= i < self.x1

    def holds(self, i):
        return self.lx0 <= i < self.lx0 + self.nxl

    def local(self, i):
        return i - self.lx0

    def owned_local(self):
        return self.glo, self.glo + self.x1 - self.x0


def parkable_simulation(cfg):
    """A GPU Simulation of cfg created parkable."""
    from .engine import Simulation
    lc = abi.Config()
    C.memmove(C.byref(lc), C.byref(cfg), C.sizeof(abi.Config))
    lc.parkable = 1
    return Simulation(lc)


class OutOfCoreSimulation:
    """One grid stepped as nslabs x slabs that take turns on the device,
    steps_per_turn time steps per turn.

    Set-up calls take the global arrays and coordinates; they are applied to
    the slabs when the slabs are built (at the first step or read-back).
    make_local(cfg) builds a slab's simulation (default: a parkable GPU
    Simulation); it must offer copy_planes or read_planes / write_planes.  park(local) /
    unpark(local) move it off and onto the device (defaults: its park /
    unpark methods where it has them, else nothing).  Slabs without
    copy_planes (a CPU engine) exchange edges by read_planes / write_planes.
    """

    def __init__(self, cfg, nslabs, steps_per_turn=8, make_local=None, park=None, unpark=None, resident=1):
        self.K = int(steps_per_turn)
        if self.K < 1:
            raise ValueError("steps_per_turn must be >= 1")
        self.resident = max(1, int(resident))
        self._pool = None
        self.plans = [WindowSlab(cfg, nslabs, r, self.K + 1) for r in range(nslabs)]
        self.gcfg = cfg
        self._make = make_local or parkable_simulation
        self._park = park or (lambda s: s.park() if hasattr(s, "park") else None)
        self._unpark = unpark or (lambda s: s.unpark() if hasattr(s, "unpark") else None)
        self._pool_dev = None     # device whose park pool this run opened
        self._ops = []            # set-up calls, replayed on each slab when it is built
        self._fields = {}         # initial global fields by component
        self._probes = []         # (slab, global id) in each slab's local order
        self._nprobes = 0
        self._dfts = []           # (slab, local id)
        self.slabs = None
        self.turns = 0

    # ---- set-up (recorded)
    def set_materials(self, table, idx_x, idx_y=None, idx_z=None):
        for m in table:
            if m.gyro_wp > 0:
                raise ValueError("out-of-core slabs do not carry gyrotropic materials")
        self._ops.append(("mat", (table, idx_x, idx_y, idx_z)))

    def add_point_source(self, src):
        self._ops.append(("src", src))

    def set_tfsf(self, t):
        """The TF/SF source of the whole grid (box in whole-grid coordinates):
        every slab takes it with its x origin, so the plane wave's 1-D line
        and the dipole's position are the whole grid's."""
        self._ops.append(("tfsf", t))

    def set_design(self, lo, eps):
        raise ValueError("out-of-core slabs do not carry design regions")

    def add_probe(self, comp, i, j, k, mode=abi.PROBE_NODE):
        gid = self._nprobes
        self._nprobes += 1
        self._ops.append(("probe", (gid, comp, i, j, k, mode)))
        return gid

    def add_dft_plane(self, axis, index, comp_mask, omegas):
        """A DFT plane of the whole grid: normal to x, recorded by the slab
        that owns it; normal to y or z, recorded by every slab over its local
        rows and read back as the owned rows of each."""
        did = len(self._dfts)
        self._dfts.append(None)
        self._ops.append(("dft", (did, axis, index, comp_mask, omegas)))
        return did

    def set_field(self, comp, arr):
        if self.slabs is not None:
            raise ValueError("fields are set before the first step")
        self._fields[comp] = np.asarray(arr, dtype=np.float32)

    # ---- slabs
    # Edge planes move between neighbours directly (dtmx_copy_planes, the
    # parked neighbour's host copy read or written in place): at the start of
    # its turn, slab r takes its upper ghost planes from slab r + 1's first
    # owned planes and leaves its own last owned planes in slab r + 1's lower
    # ghost planes, both at time n, before it steps.  Turn t of slab r runs
    # after turn t of slab r - 1 (which left r's lower ghosts) and after turn
    # t - 1 of slab r + 1, and before turn t of slab r + 1.
    @staticmethod
    def _copy(dst, x0, src, src_x0, n):
        if hasattr(dst, "copy_planes"):
            dst.copy_planes(x0, src, src_x0, n)
        else:
            dst.write_planes(x0, n, src.read_planes(src_x0, n))

    def _open_pool(self, s):
        """The first GPU slab lets parking keep device memory for the slabs
        that follow (released again by close)."""
        from .engine import Simulation, set_park_pool
        if self._pool_dev is None and isinstance(s, Simulation):
            import torch
            self._pool_dev = torch.cuda.current_device()
            set_park_pool(-1, self._pool_dev)

    def _build(self):
        self.slabs = []
        S = len(self.plans)
        for r, pl in enumerate(self.plans):
            s = self._make(pl.cfg)
            a, b = pl.lx0, pl.lx0 + pl.nxl
            for kind, v in self._ops:
                if kind == "mat":
                    table, ix, iy, iz = v
                    s.set_materials(table, *[None if q is None else np.ascontiguousarray(np.asarray(q, np.uint8)[a:b])
                                             for q in (ix, iy, iz)])
                elif kind == "tfsf":
                    q = abi.TFSF()
                    C.memmove(C.byref(q), C.byref(v), C.sizeof(abi.TFSF))
                    q.x_origin, q.x_cells = float(pl.lx0), float(self.gcfg.nx)
                    s.set_tfsf(q)
                elif kind == "src" and pl.holds(v.i):
                    q = abi.PointSource()
                    C.memmove(C.byref(q), C.byref(v), C.sizeof(abi.PointSource))
                    q.i = pl.local(v.i)
                    s.add_point_source(q)
                elif kind == "probe" and pl.owns(v[2]):
                    gid, comp, i, j, k, mode = v
                    s.add_probe(comp, pl.local(i), j, k, mode)
                    self._probes.append((r, gid))
                elif kind == "dft":
                    did, axis, index, mask, om = v
                    if axis == 0 and pl.owns(index):
                        self._dfts[did] = (0, r, s.add_dft_plane(0, pl.local(index), mask, om))
                    elif axis != 0:
                        if self._dfts[did] is None:
                            self._dfts[did] = (axis, [None] * S)
                        self._dfts[did][1][r] = s.add_dft_plane(axis, index, mask, om)
            for comp, arr in self._fields.items():
                s.set_field(comp, np.ascontiguousarray(arr[a:b]))
            self._open_pool(s)
            self._park(s)
            self.slabs.append(s)

    def _turn(self, r, t, k):
        """Turn t of slab r: exchange edge planes with the parked slab r + 1
        (time n), then k steps."""
        s, pl = self.slabs[r], self.plans[r]
        self._unpark(s)
        if r < len(self.slabs) - 1:
            nb, npl = self.slabs[r + 1], self.plans[r + 1]
            lo, hi = pl.owned_local()
            self._copy(s, pl.nxl - pl.halo, nb, npl.owned_local()[0], pl.halo)
            self._copy(nb, 0, s, hi - pl.halo, pl.halo)
        s.step(k)
        self._park(s)

    def _turn_after(self, deps, r, t, k):
        for d in deps:
            d.result()
        self._turn(r, t, k)

    def step(self, n):
        """Advance every slab by n time steps, K per turn.

        Turn t of slab r needs turn t of slab r - 1 and turn t - 1 of slabs r
        and r + 1, so with resident > 1 the turns run as a dataflow on that
        many host threads (a wavefront: slab r at turn t beside slab r + 2 at
        turn t - 1), each slab on its own stream, one slab's copies overlapping
        another's steps."""
        if self.slabs is None:
            self._build()
        ks = []
        n = int(n)
        while n > 0:
            ks.append(min(n, self.K))
            n -= ks[-1]
        S, t0 = len(self.slabs), self.turns
        if self.resident == 1:
            for q, k in enumerate(ks):
                for r in range(S):
                    self._turn(r, t0 + q, k)
                self.turns += 1
            return
        if self._pool is None:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(max_workers=self.resident)
        # Turns are submitted in (turn, slab) order and the pool's threads take
        # them first in, first out, so every turn a thread waits for was taken
        # by a thread before it: the earliest unfinished turn always runs.
        futs = {}
        for q, k in enumerate(ks):
            t = t0 + q
            for r in range(S):
                deps = [futs[x] for x in ((r - 1, t), (r, t - 1), (r + 1, t - 1)) if x in futs]
                futs[(r, t)] = self._pool.submit(self._turn_after, deps, r, t, k)
        try:
            for f in futs.values():
                f.result()
        finally:
            self.turns = t0 + len(ks)

    # ---- results
    def get_field(self, comp):
        if self.slabs is None:
            self._build()
        parts = []
        for s, pl in zip(self.slabs, self.plans):
            self._unpark(s)
            lo, hi = pl.owned_local()
            parts.append(np.asarray(s.get_field(comp))[lo:hi].copy())
            self._park(s)
        return np.concatenate(parts, axis=0)

    def read_probes(self):
        out, ns = {}, 0
        for r, s in enumerate(self.slabs or []):
            ids = [gid for (q, gid) in self._probes if q == r]
            if not ids:
                continue
            self._unpark(s)
            tr = np.asarray(s.read_probes())
            self._park(s)
            for q, gid in enumerate(ids):
                out[gid] = tr[q]
            ns = max(ns, tr.shape[1])
        res = np.zeros((self._nprobes, ns), dtype=np.float64)
        for gid, t in out.items():
            res[gid, :t.shape[0]] = t
        return res

    def read_dft(self, did):
        d = self._dfts[did]
        if d[0] == 0:
            _, r, ld = d
            s = self.slabs[r]
            self._unpark(s)
            out = s.read_dft(ld)
            self._park(s)
            return out
        # normal to y or z: the plane's first in-plane axis is x; keep each slab's owned rows
        parts = []
        for s, pl, ld in zip(self.slabs, self.plans, d[1]):
            self._unpark(s)
            lo, hi = pl.owned_local()
            parts.append(np.asarray(s.read_dft(ld))[:, :, lo:hi].copy())
            self._park(s)
        return np.concatenate(parts, axis=2)

    def close(self):
        if self._pool is not None:
            self._pool.shutdown()
            self._pool = None
        for s in self.slabs or []:
            if hasattr(s, "close"):
                s.close()
        self.slabs = None
        if self._pool_dev is not None:
            from .engine import set_park_pool
            set_park_pool(0, self._pool_dev)
            self._pool_dev = None
