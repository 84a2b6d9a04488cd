"""Parity with the reference's own CUDA implementation.

oracle/refbuild/build_ref.py builds DTmaxwell4 from its sources for sm_100a
into oracle/_ref/ (its generated torre kernels, window scheduler, sensors and
DROP_DATA field drops, one GPU, a 60 x 60 rag grid of 180 x 180 x 128 cells,
window Ns = 20, big step Ntime = 17), in FP32 and in FP64, and a driver that
does what run.py does.  With DROP_DATA the reference writes, after every big
step, Ez of one node per rag over the whole domain (ragEz_NNNNN.arr,
drop.cu:83-107); dtmx_ref_main writes the same file with --drop_data.

GPU:
  * the FP32 build against this engine on run.py's own configuration: every
    field drop and the sensor traces;
  * the FP64 build against the FP64 CPU oracle (which the other tests check
    the engine against) with the TF/SF box moved a quarter cell: run.py's box
    faces lie on node planes, where the reference's inSF test decides by its
    rounding and its FP32 and FP64 builds disagree with each other.
CPU: the reference's run.py itself, run against the DTmxw module, gives the
shotpoint that run_py() below restates (when the reference tree is present).
"""
import math
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle", "refbuild"))

NP, NA, NV, NS, NTIME = 60, 60, 128, 20, 17
NBIG = 20


def _exe(double):
    import build_ref
    exe = build_ref.binary_path(NP, NA, NV, NS, double)
    if not os.path.exists(exe):
        pytest.skip("reference build missing (python oracle/refbuild/build_ref.py%s)" % (" --double" if double else ""))
    return exe


def run_py(cv, box_shift=0.0):
    """run.py:17-35 on the DTmxw module globals (GridNx/2 is an integer
    division in the Python 2 the script was written for); box_shift moves the
    TF/SF box by that many cells along every axis."""
    dx, dy, dz, dt = cv.ds, cv.da, cv.dv, cv.dt
    center = [cv.GridNx // 2 * dx, cv.GridNy // 2 * dy, 0.150 + 0.08 + 0 * (cv.GridNz // 2) * dz]
    SS = cv.shotpoint
    SS.srcXs, SS.srcXa, SS.srcXv = center
    SS.BoxMs, SS.BoxPs = SS.srcXs - 5 * dx, SS.srcXs + 5 * dx
    SS.BoxMa, SS.BoxPa = SS.srcXa - 5 * dy, SS.srcXa + 5 * dy
    SS.BoxMv, SS.BoxPv = SS.srcXv - 5 * dz, SS.srcXv + 5 * dz
    if box_shift:
        SS.BoxMs, SS.BoxPs = SS.BoxMs + box_shift * dx, SS.BoxPs + box_shift * dx
        SS.BoxMa, SS.BoxPa = SS.BoxMa + box_shift * dy, SS.BoxPa + box_shift * dy
        SS.BoxMv, SS.BoxPv = SS.BoxMv + box_shift * dz, SS.BoxPv + box_shift * dz
    diag = math.sqrt((SS.BoxPs - SS.BoxMs) ** 2 + (SS.BoxPa - SS.BoxMa) ** 2 + (SS.BoxMv - SS.BoxPv) ** 2)
    cL = 1.0 / 1.75
    SS.set(cL, cL, 0.5 * cL)
    SS.tStop = diag / cL + 20 * 2 * math.pi / SS.w + SS.t0 + 10 * dt
    return SS


def _cvar():
    from dtmaxwell4_b200 import DTmxw
    cv = DTmxw.cvar
    cv.Np, cv.Na, cv.Nv, cv.Ns, cv.Ntime = NP, NA, NV, NS, NTIME
    cv.Npmlx, cv.Npmly, cv.Npmlz = 10, 10, 32
    cv.ds = cv.da = cv.dv = DTmxw._ftype(0.005)
    cv.dt = DTmxw._ftype(0.002)
    cv.shotpoint = DTmxw.TFSFsrc()
    return DTmxw, cv


def read_drop(path):
    head = np.fromfile(path, np.int32, 9)
    assert list(head[:5]) == [12, 0, 0, 0, 3] and head[5] in (4, 8)
    data = np.fromfile(path, np.float32 if head[5] == 4 else np.float64, offset=36)
    return data.reshape(head[8], head[7], head[6]).astype(np.float64)


def rag_sample(ez):
    """Ez of cell (3x-1, 3y-1, z) per rag (x, y): what SeismoDrops::drop writes."""
    out = np.zeros((NP, NA, NV))
    out[1:, 1:] = ez[2::3, 2::3][:NP - 1, :NA - 1]
    return out


def _run_reference(exe, steps, out, box_shift=0.0):
    # the reference keeps the drop directory in a 64-byte buffer (im3D.hpp:21): run it there, as "."
    os.makedirs(out, exist_ok=True)
    cmd = [exe, "--steps", str(steps), "--drop_dir", "."] + (["--box_shift", repr(box_shift)] if box_shift else [])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=out)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rates = [float(m) for m in re.findall(r"rate\s+([0-9.eE+-]+) GYee_cells/sec", r.stdout)]
    assert len(rates) == steps // NTIME
    return rates


@pytest.mark.gpu
def test_fp32_build_matches_engine_on_run_py(tmp_path):
    exe = _exe(False)
    steps = NTIME * NBIG
    rates = _run_reference(exe, steps, str(tmp_path / "ref"))
    DTmxw, cv = _cvar()
    run_py(cv)
    cv.Tsteps = steps
    assert DTmxw._main(["run.py", "--test", "--drop_dir", str(tmp_path / "ours"), "--drop_data"]) == 0
    ref = np.array([read_drop(tmp_path / "ref" / ("ragEz_%05d.arr" % s)) for s in range(NBIG)])
    got = np.array([read_drop(tmp_path / "ours" / ("ragEz_%05d.arr" % s)) for s in range(NBIG)])
    norms = np.linalg.norm(ref.reshape(NBIG, -1), axis=1)
    errs = np.linalg.norm((got - ref).reshape(NBIG, -1), axis=1)
    whole = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    print("reference FP32 build: %.3f GYee_cells/s (median big step); drops rel L2 %s; all drops %.3g" % (
        float(np.median(rates)), np.array2string(errs / norms, precision=2), whole))
    # The reference evaluates the dipole's incident field in float (DipoleTFSF,
    # signal.hpp:51-97), this engine in double: while the pulse is still in its
    # far Gaussian tail (the first big step, |Ez| ~ 1e-6 of its later size)
    # that float evaluation is the larger error, so the per-drop check starts
    # where the drop holds at least 1% of the largest one.
    assert whole <= 1e-5
    big = norms >= 1e-2 * norms.max()
    assert big.sum() >= NBIG - 3
    assert np.all(errs[big] <= 1e-5 * norms[big]), errs / norms
    # sensor traces (%g text): on the dipole axis only Ez is non-zero by symmetry
    X0, Y0, Z0 = NP * 3 // 2, NA * 3 // 2, 30
    tr = {}
    for side in ("ref", "ours"):
        tr[side] = np.array([np.loadtxt(tmp_path / side / ("%s-x%05dy%05dz%05d.dat" % (n, X0, Y0, Z0)))
                             for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")])
    assert tr["ref"].shape == tr["ours"].shape == (6, NBIG)
    ez = np.linalg.norm(tr["ref"][2])
    assert np.linalg.norm(tr["ours"][2] - tr["ref"][2]) <= 1e-5 * ez
    assert np.abs(tr["ours"] - tr["ref"]).max() <= 1e-5 * ez


@pytest.mark.gpu
def test_fp64_build_matches_fp64_oracle(tmp_path):
    """The oracle against the reference's FP64 build, run.py's source with the
    box a quarter cell off the node planes."""
    import pyoracle
    import ref_geometry
    from dtmaxwell4_b200 import abi
    exe = _exe(True)
    # Big steps 1-5: the pulse crosses the organic layer and reaches the top
    # of the Drude (Ag) film.  From big step 6 on, the FP64 build departs from
    # the reference's own FP32 build inside the film (3e-4 by step 7, 1e-3 by
    # step 9, almost all of it on Ag nodes), while the FP32 build, this
    # engine and the FP64 oracle keep agreeing to FP32 rounding (5e-6) there:
    # the FP64 configuration of the reference's dispersive path is the odd
    # one, so the FP64 pin stops at step 5 and the FP32 test above carries
    # the film.
    nbig = 6
    _run_reference(exe, NTIME * nbig, str(tmp_path / "ref64"), box_shift=0.25)
    # run.py in double (the FP64 build's ftype is double, so nothing is rounded to float)
    d = 0.005
    nx, ny, nz = 3 * NP, 3 * NA, NV
    c = [nx // 2 * d, ny // 2 * d, 0.150 + 0.08]
    lo = [v - 5 * d + 0.25 * d for v in c]
    hi = [v + 5 * d + 0.25 * d for v in c]
    cL = 1.0 / 1.75
    st = ref_geometry.tfsfsrc_set(cL, cL, 0.5 * cL, ftype=np.float64)
    diag = math.sqrt(sum((h - l) ** 2 for l, h in zip(lo, hi)))
    tstop = diag / cL + 20 * 2 * math.pi / st["w"] + st["t0"] + 10 * 0.002
    cfg = abi.make_config(nx, ny, nz, dx=d, dy=d, dz=d, dt=0.002, order=4, geometry=abi.GEOM_REFERENCE,
                          absorber=abi.ABS_SPLIT_PML, pml=((15, 15), (15, 15), (0, 16)), spml_vmax=st["V_max"])
    o = pyoracle.OracleSim(cfg)
    mats = [abi.make_material(1.75 ** 2),
            abi.make_material(1.0, poles=[(abi.POLE_DRUDE, 1.0, 136.66 / 3.0, 2.69e13 / 2 / 3e14, 0.0)], eps_inf=1.0),
            abi.make_material(1.8 ** 2), abi.make_material(1.5 ** 2)]
    o.set_materials(mats, *ref_geometry.material_indices(NP, NA, NV, d, d, d))
    t = abi.TFSF()
    t.kind = abi.TFSF_DIPOLE
    t.box_lo[:] = lo
    t.box_hi[:] = hi
    t.c, t.w, t.kenv, t.tstop, t.ntime = st["cSrc"], st["w"], st["kEnv"], tstop, NTIME
    o.set_tfsf(t)
    errs = []
    for s in range(nbig):
        o.step(NTIME)
        want = rag_sample(o.get_field(abi.EZ))
        got = read_drop(tmp_path / "ref64" / ("ragEz_%05d.arr" % s))
        if s == 0:
            # the first drop holds no field yet in either run
            assert np.abs(want).max() == 0 and np.abs(got).max() == 0
            continue
        errs.append(np.linalg.norm(got - want) / np.linalg.norm(want))
    o.close()
    print("reference FP64 build vs FP64 oracle, drops 1-%d rel L2:" % (nbig - 1), np.array2string(np.array(errs), precision=2))
    assert max(errs) <= 1e-7


def test_run_py_restatement_matches_run_py(monkeypatch):
    """Executes the reference's run.py with DTmxw = this package's module and
    a _main that records instead of running; the shotpoint must equal what
    run_py() computes."""
    import build_ref
    run_py_path = os.path.join(build_ref.DEFAULT_REF, "run.py")
    if not os.path.exists(run_py_path):
        pytest.skip("reference tree not present")
    from dtmaxwell4_b200 import engine
    try:
        engine.load()
    except OSError as e:
        pytest.skip(str(e))
    DTmxw, cv = _cvar()
    seen = {}
    monkeypatch.setattr(DTmxw, "_main", lambda argv: seen.setdefault("argv", list(argv)) and 0)
    monkeypatch.setitem(sys.modules, "DTmxw", DTmxw)
    monkeypatch.setattr(sys, "argv", ["run.py", "--test"])
    src = open(run_py_path).read()
    exec(compile(src, run_py_path, "exec"), {"__name__": "__main__"})
    assert seen["argv"] == ["run.py", "--test"]
    got = {n: getattr(cv.shotpoint, n) for n, _ in DTmxw.TFSFsrc._fields_}
    assert cv.Tsteps == 1000000
    _, cv2 = _cvar()
    run_py(cv2)
    want = {n: getattr(cv2.shotpoint, n) for n, _ in DTmxw.TFSFsrc._fields_}
    # run.py divides GridNx/2 with Python 3's true division here; both grids are even
    assert got == want
