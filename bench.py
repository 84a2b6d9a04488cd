"""Throughput benchmark of the FDTD hot path (Gcell-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: Drude nanoparticle lit by a TF/SF plane wave -- 384^3 FP32 cells,
sphere r = 40 cells (eps_inf = 1, wp = 2 pi c/(8 dx), gamma = wp/50) as a
Drude ADE current, +x Ez-polarised Gaussian-pulse plane wave through a TF/SF
box inset 20 cells from a 12-cell CPML, running FP64 DFT at 16 frequencies on
one x-normal plane.  Synthetic inputs of those shapes (no dataset).  One
bench step = --tsteps leapfrog time steps (default 100).

Multi-GPU: one process per GPU, each running an independent replica
(weak scaling, no data-path collective); time = max over ranks.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=384)
    ap.add_argument("--tsteps", type=int, default=100)
    ap.add_argument("--engine", type=int, default=0)
    ap.add_argument("--tblock", type=int, default=0, help="time steps per wavefront launch (--engine 2)")
    ap.add_argument("--workload", default="drude", choices=["drude", "plain"],
                    help="drude: the headline workload; plain: seeded fields in vacuum with the CPML only "
                         "(no sources or monitors), to time the field kernels of both engines")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-extras", action="store_true", help="skip the adjoint and batched measurements")
    ap.add_argument("--no-point-dipole", action="store_true", help="skip the 128^3 point-dipole measurement")
    ap.add_argument("--extras-only", action="store_true", help="print only the adjoint and batched measurements")
    ap.add_argument("--adj-steps", type=int, default=2000)
    ap.add_argument("--batch-instances", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=1500)
    ap.add_argument("--gyro-steps", type=int, default=100, help="timed steps of the 1024x1024x1536 gyrotropic run")
    ap.add_argument("--gyro-n", type=int, nargs=3, default=[1024, 1024, 1536])
    ap.add_argument("--no-gyro", action="store_true", help="skip the gyrotropic / Purcell measurement")
    ap.add_argument("--gyro-only", action="store_true", help="with --extras-only: only the gyrotropic measurement")
    ap.add_argument("--no-purcell", action="store_true", help="gyrotropic measurement without the Purcell spectrum")
    ap.add_argument("--no-ooc", action="store_true", help="skip the out-of-core (parked slabs) measurement")
    ap.add_argument("--ooc-only", action="store_true", help="with --extras-only: only the out-of-core measurement")
    ap.add_argument("--ooc-n", type=int, nargs=3, default=[1024, 512, 512])
    ap.add_argument("--ooc-slabs", type=int, default=4)
    ap.add_argument("--ooc-k", type=int, default=64, help="time steps per slab turn")
    ap.add_argument("--ooc-resident", type=int, default=3, help="slabs on the device at once")
    ap.add_argument("--ooc-steps", type=int, default=128)
    return ap.parse_args()


METRIC = "Gcell-updates/s (FP32 forward, Drude sphere + TF/SF + 16-freq DFT plane)"
UNIT = "Gcell-updates/s"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(sc):
    """Algorithmic DRAM bytes of one launch of the H and the E field kernel
    (each field value read once and written once; absorber and ADE state only
    where they exist; 1 B material index per E component)."""
    import numpy as np
    cfg = sc["cfg"]
    n = (cfg.nx, cfg.ny, cfg.nz)
    ncell = n[0] * n[1] * n[2]
    slab = 0
    for a in range(3):
        th = cfg.pml[a][0] + cfg.pml[a][1]
        slab += th * ncell // n[a]
    # per slab cell along an axis: 2 E and 2 H components carry a psi (read + write 4 B each)
    hb = 36 * ncell + 2 * 8 * slab
    mats, idx = sc["materials"]
    disp = 0
    if mats is not None:
        for c in range(3):
            for m, mat in enumerate(mats):
                if mat.npoles > 0:
                    disp += int((np.asarray(idx[c]) == m).sum())
    # ADE per dispersive node: Em, Jp, Jm read + write (4 B each) instead of the 1/eps path
    eb = 36 * ncell + 3 * ncell + 2 * 8 * slab + disp * 24
    # the single-sweep kernel reads E and H once and writes them once (the two
    # passes each read the other field again); the ADE nodes are its side pass
    fb = hb + eb - 24 * ncell - disp * 24
    return hb, eb, fb


def dram_bytes_per_cell(kernel, workload):
    """DRAM bytes per cell of one launch of `kernel` on `workload`, from the ncu
    captures summarised in profiles/ (None when there is no capture)."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "dram_bytes_per_cell.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 3 and not line.startswith("#") and f[0] == kernel and f[1] == workload:
            return float(f[2])
    return None


def max_over_ranks(ms, world, device):
    """The timed region's duration on this rank -> the maximum over all ranks
    (every rank takes part; the slowest replica sets the job's time)."""
    import torch
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(cell_updates_per_rank, world, ms_max):
    """Whole-job Gcell-updates/s: the work of all replicas over the slowest rank's time."""
    return cell_updates_per_rank * world / (ms_max * 1e-3) / 1e9


def run_ours(args, rank, world):
    import numpy as np
    import torch
    from dtmaxwell4_b200 import Simulation, scenarios, abi

    dev = rank % max(1, torch.cuda.device_count())
    torch.cuda.set_device(dev)
    if args.workload == "plain":
        sc = scenarios.drude_sphere_tfsf(n=args.n, steps=args.tsteps * (args.steps + args.warmup + 8))
        sc = dict(sc, materials=(None, None), tfsf=None, probes=[], dft=[], point_sources=[],
                  desc="%d^3 vacuum, seeded fields (normal, sigma 1e-3), 12-cell CPML, no sources or monitors" % args.n)
    else:
        sc = scenarios.drude_sphere_tfsf(n=args.n, steps=args.tsteps * (args.steps + args.warmup + 8))
    sim = Simulation(sc["cfg"])
    scenarios.apply(sim, sc)
    if args.workload == "plain":
        rng = np.random.default_rng(0)
        for c in range(6):
            sim.set_field(c, (rng.standard_normal(sim.shape, dtype=np.float32) * 1e-3))
    run_ours.tuned = (max(1, args.engine), args.tblock, 0, 0.0)
    if args.engine:
        sim.set_engine(args.engine, args.tblock)
    else:
        # engine configuration chosen by the library's autotuner (state is restored after the trials)
        tuned = sim.autotune(12)
        run_ours.tuned = tuned
    run_ours.rows = sim.engine_config()[3]
    ncell = sc["cfg"].nx * sc["cfg"].ny * sc["cfg"].nz
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    for _ in range(args.warmup):
        sim.step(args.tsteps)
    sim.sync()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    l0 = sim.launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        sim.step(args.tsteps)
    ev1.record(stream)
    ev1.synchronize()
    launches = sim.launches() - l0
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    torch.cuda.synchronize()
    ms_max = max_over_ranks(ms, world, "cuda")
    value = aggregate_rate(ncell * args.tsteps * args.steps, world, ms_max)
    assert sim.check_finite(), "non-finite fields"

    # roofline of the dominant field kernel: per-launch device time with events
    sim.set_profiling(True)
    sim.step(max(20, args.tsteps // 5))
    h_ms, e_ms, cnt = sim.read_profile()
    sim.set_profiling(False)
    hb, eb, fb = algorithmic_bytes(sc)
    peak, peak_kind = measured_peaks()
    engine_used = args.engine if args.engine else run_ours.tuned[0]
    if engine_used == 3:
        kms = h_ms / cnt
        achieved = fb / (kms * 1e-3) / 1e9
        dpc = dram_bytes_per_cell("fused_kernel", args.workload)
        roof = {"bound": "hbm", "kernel": "fused_kernel", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                "traffic": int(dpc * ncell) if dpc else None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per cell (256^3 capture) x cells",
                "algorithmic_bytes_per_launch": fb, "ms_per_launch": round(kms, 4),
                "step_bytes_per_cell_update": round(fb / ncell, 2)}
    elif args.engine == 2:
        # one wavefront launch reads and writes the state once for tblock steps
        T = max(1, args.tblock)
        kb = (hb + eb) - 36 * ncell - 3 * ncell          # the H and E reads/writes of one step ...
        kb += 48 * ncell + 3 * ncell                        # ... become one read + one write of all fields
        kms = h_ms / cnt * T
        achieved = kb / (kms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": "torre_kernel", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes_per_launch": kb, "ms_per_launch": round(kms, 4), "steps_per_launch": T}
    else:
        if e_ms >= h_ms:
            kname, kms, kbytes = "e_kernel", e_ms / cnt, eb
        else:
            kname, kms, kbytes = "h_kernel", h_ms / cnt, hb
        achieved = kbytes / (kms * 1e-3) / 1e9
        # DRAM bytes per cell of one launch from the ncu capture of the same
        # kernels on the 256^3 case of this workload, scaled by cells
        dpc = dram_bytes_per_cell(kname, args.workload)
        traffic = int(dpc * ncell) if dpc else None
        roof = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": traffic,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per cell (256^3 capture) x cells",
                "algorithmic_bytes_per_launch": kbytes, "ms_per_launch": round(kms, 4),
                "h_ms_per_launch": round(h_ms / cnt, 4), "e_ms_per_launch": round(e_ms / cnt, 4),
                "step_bytes_per_cell_update": round((hb + eb) / ncell, 2)}

    # end to end through the public API with host buffers: the state lives in
    # pinned host memory (as the reference's windowed calcStep keeps it in host
    # RAM); every step uploads the six fields, advances tsteps, downloads them.
    host = [torch.empty(sc["cfg"].nx, sc["cfg"].ny, sc["cfg"].nz, dtype=torch.float32).pin_memory() for _ in range(6)]
    arrs = [h.numpy() for h in host]
    for c in range(6):
        sim.get_field(c, out=arrs[c])
    e_steps = max(2, min(args.steps, 5))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e_steps):
        for c in range(6):
            sim.set_field(c, arrs[c])
        sim.step(args.tsteps)
        for c in range(6):
            sim.get_field(c, out=arrs[c])
    e1.record(stream)
    e1.synchronize()
    e2e_val = aggregate_rate(ncell * args.tsteps * e_steps, world, max_over_ranks(e0.elapsed_time(e1), world, "cuda"))
    nb = 6 * ncell * 4
    e2e = {"value": round(e2e_val, 3), "unit": UNIT, "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb,
           "steps": e_steps,
           "cadence": "the six fields uploaded and downloaded once per bench step (%d time steps) through "
                      "dtmx_set_field / dtmx_get_field; CPML, ADE and DFT state stay on the device" % args.tsteps}
    sim.close()
    return value, ms_max, launches, roof, e2e, clk, sc


def run_adjoint(args):
    """Forward + adjoint of the differentiation workload (256x256x192, 64x64x32
    design region, 2000 steps, checkpoint every 100): gradients/s and the
    forward-only rate of the same run for comparison."""
    import torch
    from dtmaxwell4_b200 import Simulation, scenarios
    sc = scenarios.design_region(steps=args.adj_steps)

    def make():
        # forward and recomputed segments step with the single-sweep engine
        s = Simulation(sc["cfg"])
        scenarios.apply(s, sc)
        s.set_design(*sc["design"])
        s.set_engine(3, 0)
        return s
    w = make()
    w.forward_adjoint(40, sc["plane_x"], sc["omega"], 20)
    w.close()
    s = make()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.step(sc["steps"])
    s.sync()
    t_fwd = time.perf_counter() - t0
    s.close()
    res = {}
    first = {}
    for mode, budget in (("history", -1), ("recompute", 0)):
        # the first call of a mode grows the device memory pool to the run's size
        # (history or checkpoints); the second, timed call is the steady state of
        # an optimisation loop, which takes its buffers from the pool
        for rep in range(2):
            s = make()
            s.set_adjoint_memory(budget)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            J, g = s.forward_adjoint(sc["steps"], sc["plane_x"], sc["omega"], 100)
            dt = time.perf_counter() - t0
            s.close()
            if rep == 0:
                first[mode] = dt
        res[mode] = (dt, J, g)
    t_fa, J, g = res["history"]
    t_rc, J_rc, g_rc = res["recompute"]
    c = sc["cfg"]
    cells = c.nx * c.ny * c.nz
    nd = g.size // 3
    return {"workload": sc["desc"] + ", %d steps" % sc["steps"],
            "mode": "design-region history recorded in the forward pass (%.2f GB), no recompute"
                    % ((sc["steps"] + 1) * 3 * nd * 4 / 1e9),
            "grads_per_s": round(1.0 / t_fa, 4), "seconds": round(t_fa, 3),
            "forward_gcell_per_s": round(cells * sc["steps"] / t_fwd / 1e9, 3),
            "forward_adjoint_gcell_per_s": round(cells * sc["steps"] / t_fa / 1e9, 3),
            "cost_over_forward": round(t_fa / t_fwd, 2), "objective": J,
            "first_call_seconds": round(first["history"], 3),
            "checkpointed": {"mode": "state checkpoint every 100 steps, each segment recomputed",
                             "grads_per_s": round(1.0 / t_rc, 4), "cost_over_forward": round(t_rc / t_fwd, 2),
                             "first_call_seconds": round(first["recompute"], 3),
                             "identical": bool(J_rc == J and (g_rc == g).all())},
            "note": "wall clock around the public-API calls, host-synchronised; second call of each mode "
                    "(the first grows the device memory pool, first_call_seconds)"}


def run_point_dipole(args):
    """The 128^3 point-dipole configuration at full length (1000 steps, 10-cell
    CPML, dielectric sphere, 16 probe traces recorded every step): forward rate
    with the engine configuration chosen by the autotuner, CUDA events on the
    context stream."""
    import torch
    from dtmaxwell4_b200 import Simulation, scenarios
    sc = scenarios.point_dipole_sphere()
    s = Simulation(sc["cfg"])
    scenarios.apply(s, sc)
    tuned = s.autotune(20)
    s_rows = s.engine_config()[3]
    stream = torch.cuda.ExternalStream(s.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.sync()
    e0.record(stream)
    s.step(sc["steps"])
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    tr = s.read_probes()
    s.close()
    c = sc["cfg"]
    return {"workload": sc["desc"] + ", %d steps, %d probe traces" % (sc["steps"], tr.shape[0]),
            "engine": "engine %d, x chunk %d, %d-row tiles, chosen by dtmx_autotune" % (tuned[0], tuned[2], s_rows),
            "gcell_per_s": round(c.nx * c.ny * c.nz * sc["steps"] / (ms * 1e-3) / 1e9, 3),
            "ms_per_step": round(ms / sc["steps"], 4),
            "note": "50 MB of fields: L2-resident, issue/latency-bound (ncu capture of the field kernels on this grid)"}


def run_out_of_core(args):
    """A grid stepped as x slabs that take turns on the device (parked in
    pinned host memory between turns, K steps per turn): rate against the
    same grid in core, and whether the fields after the same steps are
    identical.  Wall clock around the public-API calls, host-synchronised."""
    import numpy as np
    import torch
    from dtmaxwell4_b200 import Simulation, scenarios
    from dtmaxwell4_b200.window import OutOfCoreSimulation, parkable_simulation
    nx, ny, nz = args.ooc_n
    K, steps = args.ooc_k, args.ooc_steps
    sc = scenarios.point_dipole_sphere(n=(nx, ny, nz), steps=K + steps, pml=10, nprobes=4)
    cells = nx * ny * nz

    def make(c):
        s = parkable_simulation(c)
        s.set_engine(3, 0)
        return s
    w = OutOfCoreSimulation(sc["cfg"], args.ooc_slabs, steps_per_turn=K, make_local=make, resident=args.ooc_resident)
    scenarios.apply(w, sc)
    w.step(K)                                   # builds the slabs, one warm-up turn
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    w.step(steps)
    t_ooc = time.perf_counter() - t0
    free_ooc = torch.cuda.mem_get_info()[0]
    ez_ooc = w.get_field(2)
    tr_ooc = w.read_probes()
    w.close()
    g = Simulation(sc["cfg"])
    scenarios.apply(g, sc)
    g.set_engine(3, 0)
    g.step(K)
    g.sync()
    free_in = torch.cuda.mem_get_info()[0]
    stream = torch.cuda.ExternalStream(g.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.step(steps)
    e1.record(stream)
    e1.synchronize()
    t_in = e0.elapsed_time(e1) * 1e-3
    same = bool(np.array_equal(ez_ooc, g.get_field(2)) and np.array_equal(tr_ooc, g.read_probes().astype(np.float64)))
    g.close()
    pl = w.plans
    ghost = sum(p.nxl for p in pl) / nx - 1.0
    return {"workload": sc["desc"] + ", %d timed steps" % steps,
            "slabs": args.ooc_slabs, "steps_per_turn": K, "resident_slabs": args.ooc_resident,
            "ghost_overhead": round(ghost, 3),
            "gcell_per_s": round(cells * steps / t_ooc / 1e9, 3),
            "in_core_gcell_per_s": round(cells * steps / t_in / 1e9, 3),
            "device_bytes_free_out_of_core": int(free_ooc), "device_bytes_free_in_core": int(free_in),
            "identical_to_in_core": same,
            "note": "engine 3 in both; each turn unparks a slab (H2D of its state), exchanges K+1 edge planes "
                    "with the parked next slab's host copy, steps K times and parks it (D2H)"}


def run_out_of_core_headline(args):
    """The headline workload (384^3 Drude sphere, plane-wave TF/SF, 16-frequency
    DFT plane) stepped out of core: 2 x slabs parked in host memory, 64 steps
    per turn, one resident (at this size more slabs and concurrent turns
    measured slower), against the same run in core; fields and DFT compared
    bit for bit.  Wall clock around the public-API calls."""
    import numpy as np
    import torch
    from dtmaxwell4_b200 import Simulation, scenarios
    from dtmaxwell4_b200.window import OutOfCoreSimulation, parkable_simulation
    K, steps, nsl = 64, 128, 2
    sc = scenarios.drude_sphere_tfsf(n=args.n, steps=K + steps)
    cells = args.n ** 3

    def make(c):
        s = parkable_simulation(c)
        s.set_engine(3, 0)
        return s
    w = OutOfCoreSimulation(sc["cfg"], nsl, steps_per_turn=K, make_local=make, resident=1)
    dw = scenarios.apply(w, sc)
    w.step(K)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    w.step(steps)
    t_ooc = time.perf_counter() - t0
    got = ([w.get_field(c) for c in range(6)], w.read_dft(dw[0]))
    w.close()
    g = Simulation(sc["cfg"])
    dg = scenarios.apply(g, sc)
    g.set_engine(3, 0)
    g.step(K)
    g.sync()
    t0 = time.perf_counter()
    g.step(steps)
    g.sync()
    t_in = time.perf_counter() - t0
    same = all(np.array_equal(got[0][c], g.get_field(c)) for c in range(6)) and np.array_equal(got[1], g.read_dft(dg[0]))
    g.close()
    return {"workload": sc["desc"] + ", %d timed steps" % steps, "slabs": nsl, "steps_per_turn": K,
            "resident_slabs": 1, "gcell_per_s": round(cells * steps / t_ooc / 1e9, 3),
            "in_core_gcell_per_s": round(cells * steps / t_in / 1e9, 3), "identical_to_in_core": bool(same),
            "note": "single sweep in both; host-synchronised wall clock (in core: the public step call)"}


def run_batched(args):
    """Independent design-block instances (edges from {64..256}, 8 blocks,
    one dipole, 10-cell CPML): one-at-a-time forward+adjoint loop against the
    interleaved batch, gradients/s of each and whether results are identical."""
    import numpy as np
    import torch
    from dtmaxwell4_b200 import Simulation, engine, scenarios
    n, steps = args.batch_instances, args.batch_steps
    scs = [scenarios.design_block_instance(seed, steps=steps) for seed in range(n)]

    def make(sc):
        # both arms step with the single-sweep engine (its automatic x chunk)
        s = Simulation(sc["cfg"])
        scenarios.apply(s, sc)
        s.set_design(*sc["design"])
        s.set_engine(3, 0)
        return s
    w = make(scs[0])
    w.forward_adjoint(20, scs[0]["plane_x"], scs[0]["omega"], 10)
    w.close()
    sims = [make(sc) for sc in scs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loop = [s.forward_adjoint(steps, sc["plane_x"], sc["omega"], 100) for s, sc in zip(sims, scs)]
    t_loop = time.perf_counter() - t0
    for s in sims:
        s.close()
    sims = [make(sc) for sc in scs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J, G = engine.batch_forward_adjoint(sims, steps, [sc["plane_x"] for sc in scs], [sc["omega"] for sc in scs], 100)
    t_batch = time.perf_counter() - t0
    for s in sims:
        s.close()
    same = all(J[b] == loop[b][0] and np.array_equal(G[b], loop[b][1]) for b in range(n))
    cells = sum(sc["cfg"].nx * sc["cfg"].ny * sc["cfg"].nz for sc in scs)
    return {"workload": "%d design-block instances (edges 64..256, 8 blocks, dipole, 10-cell CPML, 16^3 design), "
                        "%d steps each, checkpoint every 100" % (n, steps),
            "cells": cells, "loop_grads_per_s": round(n / t_loop, 3), "batch_grads_per_s": round(n / t_batch, 3),
            "batch_over_loop": round(t_loop / t_batch, 3), "identical_to_loop": bool(same),
            "note": "wall clock around the public-API calls, host-synchronised"}


def run_gyro_purcell(args):
    """Gyrotropic photonic-crystal workload with its FP64 flux box: the
    forward rate at the full 1024 x 1024 x 1536 size over a bounded number of
    steps, and the Purcell spectrum W/W0 of the same lattice, slab, layer and
    dipole on a 256 x 256 x 512 cut of it run for the full 8000 steps against
    a vacuum run with the same source and box."""
    import numpy as np
    from dtmaxwell4_b200 import Simulation, purcell, scenarios
    out = {}
    # full size: forward rate
    n = tuple(args.gyro_n)
    sc = scenarios.gyro_crystal_purcell(n=n, steps=args.gyro_steps)
    s = Simulation(sc["cfg"])
    scenarios.apply(s, sc)
    scenarios.apply_flux(s, sc)
    tuned = s.autotune(4)
    s_rows = s.engine_config()[3]
    s.step(3)
    s.sync()
    t0 = time.perf_counter()
    s.step(args.gyro_steps)
    s.sync()
    dt = time.perf_counter() - t0
    s.close()
    hb, eb, fb = algorithmic_bytes(sc)
    gyro = sum(int((sc["materials"][1][c] == 2).sum()) for c in range(3))
    ncell = n[0] * n[1] * n[2]
    # the field bytes of the engine the autotuner chose (one sweep or two passes), plus the
    # gyrotropic current (read and written by its pass)
    b_cell = ((fb if tuned[0] == 3 else hb + eb) + 8 * gyro) / ncell
    rate = ncell * args.gyro_steps / dt / 1e9
    hbm, kind = measured_peaks()
    out.update({"workload": sc["desc"] + ", %d timed steps (of 8000) after 3 warm-up steps" % args.gyro_steps,
                "engine": "engine %d, x chunk %d, %d-row tiles, chosen by dtmx_autotune" % (tuned[0], tuned[2], s_rows),
                "gcell_per_s": round(rate, 3), "ms_per_step": round(1e3 * dt / args.gyro_steps, 3),
                "bytes_per_cell_update": round(b_cell, 2),
                "hbm_frac": round(rate * 1e9 * b_cell / (hbm * 1e9), 4), "hbm_peak_gbs": hbm, "peak_kind": kind})
    del sc
    if args.no_purcell:
        return out
    # Purcell spectrum on a cut of the structure, full step count
    cut = scenarios.gyro_crystal_purcell(n=(256, 256, 512), steps=8000)
    vac = scenarios.gyro_crystal_purcell(n=(128, 128, 128), steps=8000, structure=False)
    power = []
    t0 = time.perf_counter()
    for sc in (cut, vac):
        s = Simulation(sc["cfg"])
        scenarios.apply(s, sc)
        fid, = scenarios.apply_flux(s, sc)
        s.step(sc["steps"])
        power.append(s.read_flux(fid)[1])
        s.close()
    t_p = time.perf_counter() - t0
    om = cut["flux"][0][2]
    w = purcell.purcell_flux(power[0], power[1], cut["eps_src"], vac["eps_src"])
    lam = 2 * np.pi / om
    out["purcell"] = {"workload": cut["desc"] + "; W0: " + vac["desc"] + "; 8000 steps each",
                      "wavelength_cells": [round(float(v), 3) for v in lam],
                      "w_over_w0": [round(float(v), 5) for v in w], "seconds": round(t_p, 2),
                      "note": "flux-box powers normalised to equal source currents (eps_src^2)"}
    return out


def cpu_sample(args, n, tsteps):
    """Time the oracle (FP32 port, all host threads) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from dtmaxwell4_b200 import scenarios
    sc = scenarios.drude_sphere_tfsf(n=n, steps=tsteps + 8)
    o = pyoracle.OracleSim(sc["cfg"], "f32")
    scenarios.apply(o, sc)
    o.step(1)                       # first step pays for lazy allocations
    t0 = time.perf_counter()
    o.step(tsteps)
    dt = time.perf_counter() - t0
    ncell = sc["cfg"].nx * sc["cfg"].ny * sc["cfg"].nz
    o.close()
    return ncell * tsteps / dt / 1e9, pyoracle.threads(), dt


def cpu_check_fp64(args, n=64, steps=4000):
    """Part of the CPU leg: the headline workload at its full length (4000
    steps, 16 DFT frequencies, 12-cell CPML) on an n^3 grid, run through the
    library with the engine configuration the timed run used and by the FP64
    oracle on the host (the oracle only checks: it is not what is measured).
    Returns the relative L2 errors against FP64 of the DFT plane, of each
    probe trace (against the strongest trace: E and H share units) and of the
    final fields (against the largest field norm of the run: after the ring-
    down the fields are six orders of magnitude below it)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from dtmaxwell4_b200 import Simulation, scenarios
    sc = scenarios.drude_sphere_tfsf(n=n, steps=steps, pml=12, inset=4, nfreq=16)
    eng, tb, xc = run_ours.tuned[:3]
    g = Simulation(sc["cfg"])
    gid = scenarios.apply(g, sc)
    if eng in (1, 3):
        g.set_engine(eng, tb)
        g.set_tile_rows(getattr(run_ours, "rows", 16))
    g.step(steps)
    g.sync()
    o = pyoracle.OracleSim(sc["cfg"], "f64")
    oid = scenarios.apply(o, sc)
    t0 = time.perf_counter()
    peak = 0.0
    for _ in range(steps // 250):
        o.step(250)
        peak = max(peak, max(float(np.sqrt(sum(np.linalg.norm(o.get_field(c)) ** 2 for c in grp)))
                             for grp in ((0, 1, 2), (3, 4, 5))))
    dt = time.perf_counter() - t0
    tg, to = g.read_probes(), o.read_probes(100000)
    norms = np.linalg.norm(to, axis=1)
    pe = float((np.linalg.norm(np.asarray(tg, np.float64) - to, axis=1) / norms.max()).max())
    dg, do = g.read_dft(gid[0]).view(np.float64), o.read_dft(oid[0]).view(np.float64)
    de = float(np.linalg.norm(dg - do) / np.linalg.norm(do))
    fe = float(np.sqrt(sum(np.linalg.norm(g.get_field(c).astype(np.float64) - o.get_field(c)) ** 2
                           for c in range(6)))) / peak
    g.close()
    o.close()
    return {"workload": sc["desc"] + ", %d steps" % steps, "engine": eng,
            "dft_rel_l2": float("%.3g" % de), "probe_rel_l2_of_strongest": float("%.3g" % pe),
            "final_fields_rel_l2_of_peak": float("%.3g" % fe), "oracle_seconds": round(dt, 1),
            "note": "relative L2 against the FP64 oracle of the same update equations"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        # the reference has no CPU implementation of the path; its CPU arm is
        # the oracle port (FP32, all host threads), one time step per bench step
        vals = []
        for it in range(args.warmup + args.steps):
            v, cores, dt = cpu_sample(args, args.n, 1)
            if it >= args.warmup:
                vals.append(v)
        value = sum(vals) / len(vals)
        line = {"metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(1e3 * (args.n ** 3) / (value * 1e9), 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": "drude_sphere_tfsf %d^3" % args.n, "time_steps_per_step": 1},
                "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "port",
                                 "sample": "1 time step of the %d^3 workload per bench step" % args.n},
                "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    if args.extras_only:
        if rank == 0:
            if args.ooc_only:
                print(json.dumps({"out_of_core": run_out_of_core(args),
                                  "out_of_core_headline": run_out_of_core_headline(args)}))
                return 0
            ex = {} if args.gyro_only else {"point_dipole": None if args.no_point_dipole else run_point_dipole(args),
                                            "adjoint": run_adjoint(args),
                                            "batched": run_batched(args)}
            if not args.no_ooc and not args.gyro_only:
                ex["out_of_core"] = run_out_of_core(args)
            if not args.no_gyro:
                ex["gyro_purcell"] = run_gyro_purcell(args)
            print(json.dumps(ex))
        return 0
    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    value, ms, launches, roof, e2e, clk, sc = run_ours(args, rank, world)
    cpu = None
    err_fp64 = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, dt = cpu_sample(args, args.n, args.cpu_steps)
        cpu = {"value": round(v, 5), "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "%d time steps of the %d^3 workload (oracle FP32, %.1f s)" % (args.cpu_steps, args.n, dt)}
        if args.workload == "drude":
            err_fp64 = cpu_check_fp64(args)
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        if not args.no_point_dipole:
            extras["point_dipole"] = run_point_dipole(args)
        extras["adjoint"] = run_adjoint(args)
        extras["batched"] = run_batched(args)
        if not args.no_ooc:
            for key, fn in (("out_of_core", run_out_of_core), ("out_of_core_headline", run_out_of_core_headline)):
                try:
                    extras[key] = fn(args)
                except Exception as e:             # e.g. pinned host memory refused on this host
                    extras[key] = {"error": "%s: %s" % (type(e).__name__, e)}
        if not args.no_gyro:
            extras["gyro_purcell"] = run_gyro_purcell(args)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "%s %d^3, %d time steps per step" % (
                               "drude_sphere_tfsf" if args.workload == "drude" else "plain_cpml", args.n, args.tsteps),
                           "engine": ("wavefront T=%d" % max(1, args.tblock)) if args.engine == 2 else
                                     "engine %d, T %d, x chunk %d (0: automatic), %d-row tiles%s" % (tuple(run_ours.tuned[:3]) + (
                                         run_ours.rows, ", chosen by dtmx_autotune" if not args.engine else "",)),
                           "desc": sc["desc"], "time_steps_per_step": args.tsteps,
                           "l2": "inputs larger than L2 (%.2f GB of fields)" % (6 * args.n ** 3 * 4 / 1e9),
                           "parallelism": "replicas%d" % world},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
                "err_vs_fp64": err_fp64}
        line.update(extras)
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
