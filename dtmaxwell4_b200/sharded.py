"""Slab-sharded runs: one grid split along x into one slab per rank.

The reference splits its domain into y stripes across the GPUs of a node
(params.h:73-94) and copies half-rag halos between neighbours every time
step (copyrags.cuh:16-82, peer access set up in DTmxw.cu:266-277).  Here the
split is along x, the slowest-varying index of the field layout, so that a
halo is one contiguous x plane per component.

Rank r owns the planes [x0, x1) and keeps one ghost plane on each side that
has a neighbour: its local grid is [x0 - 1, x1 + 1) (without the ghost on
the grid's own faces).  A full leapfrog step (order 2) of the local grid
leaves every owned plane correct as long as, at its start, the ghost planes
hold the neighbours' E and the high ghost plane also holds H and the H
absorber state of plane x1:
  * H'(i) needs E(i-1), E(i): correct for i in [x0, x1] (E(x0-1) and E(x1)
    are the ghosts),
  * E'(i) needs H'(i), H'(i+1): correct for i in [x0, x1 - 1].
H'(x1) and its CPML auxiliaries are the neighbour's own values computed again
from the same inputs (bit for bit), so after the step only E has to move:
each rank sends its first owned E plane to the left neighbour and its last
owned E plane to the right neighbour (3 contiguous planes per direction),
with torch.distributed point-to-point operations (NCCL between GPUs: the
library's device memory is sent and received in place on the context's
stream; gloo on the host).  No collective is issued inside a step.

The CPML slabs of the x faces belong to the first and last ranks (each must
own more planes than its slab, so that no ghost plane lies in one); the y
and z slabs are the same on every rank.
Sources and probes act on the rank that owns their plane; a TF/SF source on
every rank, with its box and plane-wave line in whole-grid coordinates
(dtmx_tfsf.x_origin); DFT planes normal to x are recorded by their owner,
planes normal to y or z by every rank over its owned rows.  Refused
(DTMX_ERR_UNSUPPORTED semantics, raised as ValueError): order 4 (its stencil
needs more ghost planes), gyrotropic materials (their current couples x
neighbours) and design regions.
"""
import ctypes as C

import numpy as np

from . import abi


def slab_bounds(nx, world, rank):
    """Owned planes [x0, x1) of rank: nx split as evenly as possible."""
    base, extra = divmod(nx, world)
    x0 = rank * base + min(rank, extra)
    return x0, x0 + base + (1 if rank < extra else 0)


class SlabPlan:
    """The partition of one grid for one rank and its local configuration."""

    def __init__(self, cfg, world, rank):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad rank / world size")
        if cfg.order != 2:
            raise ValueError("slab sharding supports the order-2 stencil only")
        if cfg.geometry != abi.GEOM_BOX or cfg.absorber == abi.ABS_SPLIT_PML:
            raise ValueError("slab sharding supports the box geometry with a CPML or no absorber")
        self.world, self.rank = world, rank
        self.nx = cfg.nx
        self.x0, self.x1 = slab_bounds(cfg.nx, world, rank)
        self.glo = 1 if rank > 0 else 0
        self.ghi = 1 if rank < world - 1 else 0
        self.lx0 = self.x0 - self.glo                      # global x of local plane 0
        self.nxl = self.x1 - self.x0 + self.glo + self.ghi
        lpml = (cfg.pml[0][0] if rank == 0 else 0, cfg.pml[0][1] if rank == world - 1 else 0)
        if cfg.absorber == abi.ABS_NONE:
            lpml = (0, 0)
        # a ghost plane must not lie in an x slab: the neighbour's copy of it has none
        if self.x1 - self.x0 < 1 or (world > 1 and self.x1 - self.x0 <= max(lpml)):
            raise ValueError("rank %d owns %d planes: it needs more than its x absorber slab (%d)"
                             % (rank, self.x1 - self.x0, max(lpml)))
        lc = abi.Config()
        C.memmove(C.byref(lc), C.byref(cfg), C.sizeof(abi.Config))
        lc.nx = self.nxl
        lc.pml[0][0], lc.pml[0][1] = lpml
        self.cfg = lc

    def owns(self, i):
        return self.x0 <= i < self.x1

    def local(self, i):
        return i - self.lx0

    def owned_local(self):
        """Local plane range of the owned planes."""
        return self.glo, self.glo + self.x1 - self.x0


class _DeviceArray:
    """CUDA array interface of a span of the library's device memory."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


class DevicePlanes:
    """x planes of a GPU Simulation as torch tensors that alias its device
    memory: sent and received in place, ordered on the context's stream."""

    def __init__(self, sim):
        import torch
        self.sim = sim
        self.torch = torch
        self.stream = torch.cuda.ExternalStream(sim.stream_handle())

    def _plane(self, comp, i):
        ptr, st = self.sim.device_ptr(comp)
        return self.torch.as_tensor(_DeviceArray(ptr + 4 * i * st[0], st[0]), device="cuda")

    def send(self, comp, i):
        return self._plane(comp, i)

    def recv(self, comp, i):
        return self._plane(comp, i)

    def commit(self):
        pass


class ShardedSimulation:
    """One grid stepped by all ranks of a process group, one x slab each.

    make_local(cfg) builds the rank's local simulation (default: a GPU
    Simulation on the current device); planes(local) gives its plane accessor
    (default: DevicePlanes).  Arrays passed in (materials, fields) are the
    global ones, the same on every rank; results are gathered to every rank.
    """

    def __init__(self, cfg, make_local=None, planes=None, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.plan = SlabPlan(cfg, world, rank)
        self.gcfg = cfg
        if make_local is None:
            from .engine import Simulation
            make_local = Simulation
        self.local = make_local(self.plan.cfg)
        self.planes = (planes or DevicePlanes)(self.local)
        self._probes = []        # global probe ids owned here, in local order
        self._nprobes = 0
        self._dfts = []          # (axis, local did or None, shape info)

    # ---- set-up
    def set_materials(self, table, idx_x, idx_y=None, idx_z=None):
        for m in table:
            if m.gyro_wp > 0:
                raise ValueError("slab sharding does not carry gyrotropic materials")
        a, b = self.plan.lx0, self.plan.lx0 + self.plan.nxl
        sl = [None if v is None else np.ascontiguousarray(np.asarray(v, np.uint8)[a:b]) for v in (idx_x, idx_y, idx_z)]
        self.local.set_materials(table, *sl)

    def add_point_source(self, src):
        if self.plan.owns(src.i):
            s = abi.PointSource()
            C.memmove(C.byref(s), C.byref(src), C.sizeof(abi.PointSource))
            s.i = self.plan.local(src.i)
            self.local.add_point_source(s)

    def set_tfsf(self, t):
        """The whole grid's TF/SF source (box in whole-grid coordinates), taken
        by every rank with its slab's x origin (dtmx_tfsf.x_origin)."""
        q = abi.TFSF()
        C.memmove(C.byref(q), C.byref(t), C.sizeof(abi.TFSF))
        q.x_origin, q.x_cells = float(self.plan.lx0), float(self.gcfg.nx)
        self.local.set_tfsf(q)

    def set_design(self, lo, eps):
        raise ValueError("slab sharding does not carry design regions")

    def add_probe(self, comp, i, j, k, mode=abi.PROBE_NODE):
        gid = self._nprobes
        self._nprobes += 1
        if self.plan.owns(i):
            self.local.add_probe(comp, self.plan.local(i), j, k, mode)
            self._probes.append(gid)
        return gid

    def add_dft_plane(self, axis, index, comp_mask, omegas):
        did = len(self._dfts)
        if axis == 0:
            ld = self.local.add_dft_plane(0, self.plan.local(index), comp_mask, omegas) if self.plan.owns(index) else None
        else:
            ld = self.local.add_dft_plane(axis, index, comp_mask, omegas)
        self._dfts.append((axis, ld))
        return did

    # ---- fields
    def set_field(self, comp, arr):
        a, b = self.plan.lx0, self.plan.lx0 + self.plan.nxl
        self.local.set_field(comp, np.ascontiguousarray(np.asarray(arr)[a:b]))

    def _gather(self, part):
        if self.plan.world == 1:
            return [part]
        out = [None] * self.plan.world
        self.dist.all_gather_object(out, part, group=self.group)
        return out

    def get_field(self, comp):
        lo, hi = self.plan.owned_local()
        return np.concatenate(self._gather(np.asarray(self.local.get_field(comp))[lo:hi]), axis=0)

    # ---- run
    def _exchange(self):
        """E planes across the slab faces (the ghost planes of the neighbours)."""
        p = self.plan
        if p.world == 1:
            return
        dist = self.dist
        lo, hi = p.owned_local()
        ops = []
        for c in (abi.EX, abi.EY, abi.EZ):
            if p.rank > 0:
                ops.append(dist.P2POp(dist.isend, self.planes.send(c, lo), p.rank - 1, self.group))
                ops.append(dist.P2POp(dist.irecv, self.planes.recv(c, 0), p.rank - 1, self.group))
            if p.rank < p.world - 1:
                ops.append(dist.P2POp(dist.isend, self.planes.send(c, hi - 1), p.rank + 1, self.group))
                ops.append(dist.P2POp(dist.irecv, self.planes.recv(c, p.nxl - 1), p.rank + 1, self.group))
        stream = getattr(self.planes, "stream", None)
        if stream is not None:
            import torch
            with torch.cuda.stream(stream):
                for r in dist.batch_isend_irecv(ops):
                    r.wait()
        else:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        self.planes.commit()

    def step(self, n):
        for _ in range(int(n)):
            self.local.step(1)
            self._exchange()

    def sync(self):
        if hasattr(self.local, "sync"):
            self.local.sync()

    # ---- results
    def read_probes(self):
        tr = self.local.read_probes() if self._probes else None
        parts = self._gather((self._probes, None if tr is None else np.asarray(tr)))
        ns = max((t.shape[1] for _, t in parts if t is not None), default=0)
        out = np.zeros((self._nprobes, ns), dtype=np.float64)
        for ids, t in parts:
            for q, gid in enumerate(ids):
                out[gid] = t[q]
        return out

    def read_dft(self, did):
        axis, ld = self._dfts[did]
        mine = self.local.read_dft(ld) if ld is not None else None
        if axis == 0:
            return next(v for v in self._gather(mine) if v is not None)
        # normal to y or z: the plane's first in-plane axis is x; keep the owned rows
        lo, hi = self.plan.owned_local()
        return np.concatenate(self._gather(mine[:, :, lo:hi]), axis=2)

    def close(self):
        if hasattr(self.local, "close"):
            self.local.close()
