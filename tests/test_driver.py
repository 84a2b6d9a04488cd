"""The reference's driver surface (SWIG module DTmxw, mxw.i:1-36) on the C ABI.

CPU: TFSFsrc::set and the analytic geometry get_mat_indev against the numpy
oracle, argument checks of _main.  GPU: a run.py-style run of _main on a
small grid whose sensor files (the reference's ``%g`` text format) match the
FP64 oracle run of the same scenario.
"""
import glob
import math
import os

import numpy as np
import pytest


def test_tfsfsrc_set_matches_reference():
    import ref_geometry
    from dtmaxwell4_b200 import DTmxw
    cL = 1.0 / 1.75
    sp = DTmxw.TFSFsrc()
    sp.set(cL, cL, 0.5 * cL)
    for k, v in ref_geometry.tfsfsrc_set(cL, cL, 0.5 * cL).items():
        assert getattr(sp, k) == pytest.approx(v, rel=1e-15, abs=0), k


def test_reference_geometry_matches_oracle():
    """Ag film with the hole lattice, organic, ITO and glass layers, per E component."""
    import ref_geometry
    from dtmaxwell4_b200 import DTmxw
    g = DTmxw.RefGlobals(60, 60, 100, 20, 18, 0.005, 0.005, 0.005, 0.002, 0)
    mats, idx = DTmxw.reference_materials(g)
    ref = ref_geometry.material_indices(60, 60, 100, 0.005, 0.005, 0.005)
    for c in range(3):
        assert idx[c].shape == ref[c].shape
        assert np.array_equal(idx[c], ref[c]), (c, int((idx[c] != ref[c]).sum()))
    counts = np.bincount(idx[2].ravel(), minlength=4)
    assert all(counts > 0), counts          # every layer and the holes are present
    assert len(mats) == 4 and mats[1].npoles == 1 and mats[0].eps[0] == pytest.approx(1.75 ** 2)


def test_main_rejects_bad_globals(capfd):
    from dtmaxwell4_b200 import DTmxw
    saved = (DTmxw.cvar.Np, DTmxw.cvar.Ns)
    try:
        DTmxw.cvar.Np, DTmxw.cvar.Ns = 10, 3
        assert DTmxw._main(["run.py", "--test"]) == -1
        assert "Np must be dividable by Ns" in capfd.readouterr().out
    finally:
        DTmxw.cvar.Np, DTmxw.cvar.Ns = saved


def _small_run(tmp):
    """run.py (the reference driver script) on a 48x48x64 grid."""
    from dtmaxwell4_b200 import DTmxw
    cv = DTmxw.cvar
    cv.Np, cv.Na, cv.Nv, cv.Ns, cv.Ntime = 16, 16, 64, 4, 2
    dx, dy, dz, dt = cv.ds, cv.da, cv.dv, cv.dt
    center = [cv.GridNx / 2 * dx, cv.GridNy / 2 * dy, 0.150 + 0.03]
    SS = cv.shotpoint
    SS.srcXs, SS.srcXa, SS.srcXv = center
    SS.BoxMs, SS.BoxPs = SS.srcXs - 5 * dx, SS.srcXs + 5 * dx
    SS.BoxMa, SS.BoxPa = SS.srcXa - 5 * dy, SS.srcXa + 5 * dy
    SS.BoxMv, SS.BoxPv = SS.srcXv - 5 * dz, SS.srcXv + 5 * dz
    cL = 1.0 / 1.75
    SS.set(cL, cL, 0.1 * cL)
    SS.kEnv = 0.3                      # a short pulse, so that the small run sees it
    SS.tStop = 0.3                     # the TF/SF box switches off mid-run
    cv.Tsteps = 240
    rc = DTmxw._main(["run.py", "--test", "--drop_dir", tmp])
    return rc, cv


@pytest.mark.gpu
def test_main_sensor_files_match_oracle(tmp_path):
    import pyoracle
    import ref_geometry
    from dtmaxwell4_b200 import abi
    rc, cv = _small_run(str(tmp_path))
    assert rc == 0
    files = sorted(glob.glob(str(tmp_path / "*.dat")))
    assert len(files) == 6, files
    nx, ny, nz = cv.GridNx, cv.GridNy, cv.GridNz
    sp = cv.shotpoint
    cfg = abi.make_config(nx, ny, nz, dx=cv.ds, dy=cv.da, dz=cv.dv, dt=cv.dt, order=4, geometry=abi.GEOM_REFERENCE,
                          absorber=abi.ABS_SPLIT_PML, pml=((15, 15), (15, 15), (0, 16)), spml_vmax=sp.V_max,
                          probe_every=cv.Ntime, probe_capacity=cv.Tsteps // cv.Ntime + 2)
    o = pyoracle.OracleSim(cfg)
    mats = [abi.make_material(1.75 ** 2),
            abi.make_material(1.0, poles=[(abi.POLE_DRUDE, 1.0, 136.66 / 3.0, 2.69e13 / 2 / 3e14, 0.0)], eps_inf=1.0),
            abi.make_material(1.8 ** 2), abi.make_material(1.5 ** 2)]
    o.set_materials(mats, *ref_geometry.material_indices(cv.Np, cv.Na, cv.Nv, cv.ds, cv.da, cv.dv))
    t = abi.TFSF()
    t.kind = abi.TFSF_DIPOLE
    t.box_lo[:] = [sp.BoxMs, sp.BoxMa, sp.BoxMv]
    t.box_hi[:] = [sp.BoxPs, sp.BoxPa, sp.BoxPv]
    t.c, t.w, t.kenv, t.tstop, t.ntime = sp.cSrc, sp.w, sp.kEnv, sp.tStop, cv.Ntime
    o.set_tfsf(t)
    X0, Y0, Z0 = round((sp.BoxMs + sp.BoxPs) / 2 / cv.ds), round((sp.BoxMa + sp.BoxPa) / 2 / cv.da), round(0.150 / cv.dv)
    for c in range(6):
        o.add_probe(c, X0, Y0, Z0, abi.PROBE_REFERENCE)
    o.step(cv.Tsteps)
    ref = o.read_probes(1000)
    got = []
    for c, name in enumerate(abi.COMP_NAMES):
        fn = tmp_path / ("%s-x%05dy%05dz%05d.dat" % (name, X0, Y0, Z0))
        got.append(np.loadtxt(fn))
    got = np.array(got)
    assert got.shape == ref.shape == (6, cv.Tsteps // cv.Ntime)
    # %g keeps 6 significant digits (<= 5e-6 relative per value).  The sensor
    # line starts on the dipole axis, where Ex, Ey and the whole H field vanish
    # by symmetry up to the boundary asymmetry (|H| ~ 1e-5 |Ez| here), so each
    # trace is measured against max(its norm, 1% of the strongest trace).
    # Ez, the field of the dipole on its axis, is held to 1e-5; the other five
    # are symmetry-zero there and carry only FP32 round-off of the asymmetric
    # boundaries (a few 1e-7 of |Ez|, i.e. up to a few 1e-5 of the 1% floor).
    norms = np.linalg.norm(ref, axis=1)
    assert norms[2] > 0
    floor = 1e-2 * norms.max()
    for c in range(6):
        err = np.linalg.norm(got[c] - ref[c]) / max(norms[c], floor)
        assert err <= (1e-5 if c == abi.EZ else 5e-5), (abi.COMP_NAMES[c], err)
