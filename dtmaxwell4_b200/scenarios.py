"""Scenario builders: a scenario is a plain dict (config, materials, sources,
probes, DFT planes) applied to any object with the Simulation call surface.

Workloads (all in c = 1 units with dx = 1 cell unless stated):

* point_dipole_sphere -- vacuum box, centred dielectric sphere, soft Ez point
  source with a Gaussian-modulated sine, CPML on all faces, Ez/Hx traces at
  seeded random probe points (128^3, lambda0 = 20 cells, Courant 0.5, 10-cell
  CPML, sphere r = 20 cells eps = 4, 1000 steps at full size).
* gyro_crystal_purcell -- photonic-crystal slab (eps 12, triangular lattice of
  air holes) on a magnetised-Drude gyrotropic layer (eps_diag 4, off-diagonal
  0.3 at the source frequency), soft Ez dipole in a missing-hole defect at the
  slab's mid-plane, running FP64 DFTs on the six faces of a flux box around
  the dipole (1024 x 1024 x 1536, slab 40 cells, layer 200 cells, period 32,
  hole radius 10, box half-width 20, 32 frequencies, 8000 steps at full size).
* drude_sphere_tfsf -- Drude sphere (eps_inf = 1, wp = 2 pi c/(8 dx),
  gamma = wp/50) lit by a +x, Ez-polarised Gaussian-pulse plane wave through a
  TF/SF box inset 20 cells from a 12-cell CPML; running DFT at 16 frequencies
  over the pulse's -20 dB band on one x-normal plane (384^3, 4000 steps at
  full size).
"""
import math

import numpy as np

from . import abi


def gauss_sine_params(lambda0_cells, dx=1.0, periods=3.0):
    """f0 = c/lambda0; amplitude-envelope FWHM = periods*T0, so
    tau = periods*T0/(2 sqrt(ln 2)); t0 = 4 tau."""
    f0 = 1.0 / (lambda0_cells * dx)
    T0 = 1.0 / f0
    tau = periods * T0 / (2.0 * math.sqrt(math.log(2.0)))
    return f0, tau, 4.0 * tau


def sphere_mask(n, center, radius, comp):
    """Boolean mask of the nodes of E component comp inside a sphere (cells)."""
    nx, ny, nz = n
    off = [(0, 1, 1), (1, 0, 1), (1, 1, 0)][comp]
    x = (np.arange(nx) + 0.5 * off[0])[:, None, None]
    y = (np.arange(ny) + 0.5 * off[1])[None, :, None]
    z = (np.arange(nz) + 0.5 * off[2])[None, None, :]
    return (x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2 <= radius ** 2


def point_dipole_sphere(n=128, steps=1000, pml=10, radius=None, eps=4.0, order=2, courant=0.5, nprobes=8,
                        lambda0=20.0, seed=0):
    nx = ny = nz = n if isinstance(n, int) else None
    if not isinstance(n, int):
        nx, ny, nz = n
    radius = radius if radius is not None else 20.0 * min(nx, ny, nz) / 128.0
    cfg = abi.make_config(nx, ny, nz, dx=1.0, courant=courant, order=order, pml=pml, probe_capacity=steps + 8)
    ctr = (nx / 2.0, ny / 2.0, nz / 2.0)
    idx = [sphere_mask((nx, ny, nz), ctr, radius, c).astype(np.uint8) for c in range(3)]
    mats = [abi.make_material(1.0), abi.make_material(eps)]
    f0, tau, t0 = gauss_sine_params(lambda0)
    src = abi.PointSource(comp=abi.EZ, i=nx // 2, j=ny // 2, k=nz // 2, waveform=abi.WAVE_GAUSS_SINE,
                          amp=1.0, f0=f0, tau=tau, t0=t0)
    rng = np.random.default_rng(seed)
    lo, hi = pml + 1, np.array([nx, ny, nz]) - pml - 2
    pts = rng.integers(lo, hi + 1, size=(nprobes, 3))
    probes = []
    for p in pts:
        probes.append((abi.EZ, int(p[0]), int(p[1]), int(p[2]), abi.PROBE_NODE))
        probes.append((abi.HX, int(p[0]), int(p[1]), int(p[2]), abi.PROBE_NODE))
    return dict(name="point_dipole_sphere", cfg=cfg, materials=(mats, idx), point_sources=[src], tfsf=None,
                probes=probes, dft=[], steps=steps,
                desc="%dx%dx%d, dx=lambda0/%g, Courant %g, order %d, %d-cell CPML, sphere r=%g eps=%g, soft Ez dipole"
                     % (nx, ny, nz, lambda0, courant, order, pml, radius, eps))


def drude_sphere_tfsf(n=384, steps=4000, pml=12, inset=20, radius=None, order=2, courant=0.5, lambda0=20.0,
                      nfreq=16, dft_plane=None):
    nx = ny = nz = n if isinstance(n, int) else None
    if not isinstance(n, int):
        nx, ny, nz = n
    radius = radius if radius is not None else 40.0 * min(nx, ny, nz) / 384.0
    cfg = abi.make_config(nx, ny, nz, dx=1.0, courant=courant, order=order, pml=pml, probe_capacity=steps + 8)
    ctr = (nx / 2.0, ny / 2.0, nz / 2.0)
    wp = 2.0 * math.pi / 8.0          # 2 pi c / (8 dx)
    gamma = wp / 50.0
    # reference LorenzDisp::setDrude(Deps, wp, gp, gp_): b1 = 2 gp = gamma
    drude = abi.make_material(1.0, poles=[(abi.POLE_DRUDE, 1.0, wp, gamma / 2.0, 0.0)], eps_inf=1.0)
    mats = [abi.make_material(1.0), drude]
    idx = [sphere_mask((nx, ny, nz), ctr, radius, c).astype(np.uint8) for c in range(3)]
    f0, tau, t0 = gauss_sine_params(lambda0)
    t = abi.TFSF()
    t.kind = abi.TFSF_PLANE_X
    for a, m in enumerate((nx, ny, nz)):
        t.box_lo[a] = float(pml + inset)
        t.box_hi[a] = float(m - pml - inset)
    t.amp, t.f0, t.tau, t.t0 = 1.0, f0, tau, t0
    t.tstop = 0.0
    t.ntime = 1
    # -20 dB band of the Gaussian envelope exp(-(t/tau)^2): |f-f0| <= sqrt(ln 10)/(pi tau)
    df = math.sqrt(math.log(10.0)) / (math.pi * tau)
    freqs = np.linspace(f0 - df, f0 + df, nfreq)
    omegas = 2.0 * math.pi * freqs
    xplane = dft_plane if dft_plane is not None else nx - pml - inset // 2
    dft = [(0, xplane, (1 << abi.EY) | (1 << abi.EZ) | (1 << abi.HY) | (1 << abi.HZ), omegas)]
    c = (nx // 2, ny // 2, nz // 2)
    probes = [(abi.EZ, c[0] + int(radius) + 4, c[1], c[2], abi.PROBE_NODE),
              (abi.EZ, pml + inset // 2, c[1], c[2], abi.PROBE_NODE),
              (abi.HY, c[0], c[1], c[2], abi.PROBE_NODE)]
    return dict(name="drude_sphere_tfsf", cfg=cfg, materials=(mats, idx), point_sources=[], tfsf=t, probes=probes,
                dft=dft, steps=steps,
                desc="%dx%dx%d Drude sphere r=%g (wp=2pi/8, gamma=wp/50), TF/SF +x Ez plane wave lambda0=%g, "
                     "%d-cell CPML, box inset %d, %d-freq DFT plane x=%d" % (nx, ny, nz, radius, lambda0, pml,
                                                                             inset, nfreq, xplane))


def triangular_holes(nx, ny, center, period, radius, comp):
    """2-D mask (nx, ny) of the E component comp's nodes inside the air holes of
    a triangular lattice (a1 = (period, 0), a2 = (period/2, period sqrt(3)/2))
    through `center`, leaving the hole at `center` out (the defect).  Needs
    radius < period/2: a node then lies within `radius` of at most one site,
    and the nearest site of each of the two lattice rows around it is tested."""
    if not radius < 0.5 * period:
        raise ValueError("hole radius must be below half the period")
    off = [(0, 1), (1, 0), (1, 1)][comp]
    x = (np.arange(nx) + 0.5 * off[0])[:, None] - center[0]
    y = (np.arange(ny) + 0.5 * off[1])[None, :] - center[1]
    h = period * math.sqrt(3.0) / 2.0
    mask = np.zeros((nx, ny), bool)
    l0 = np.floor(y / h)
    for dl in (0.0, 1.0):
        l = l0 + dl
        m = np.round((x - 0.5 * l * period) / period)
        cx, cy = m * period + 0.5 * l * period, l * h
        hit = (x - cx) ** 2 + (y - cy) ** 2 <= radius ** 2
        mask |= hit & ~((m == 0) & (l == 0))
    return mask


def gyro_crystal_purcell(n=(1024, 1024, 1536), slab=40, layer=200, period=32, radius=10, eps_slab=12.0,
                         eps_diag=4.0, g=0.3, pml=10, a_over_lambda=0.3, box_half=20, nfreq=32, steps=8000, order=2,
                         courant=0.5, structure=True):
    """Gyrotropic + Purcell workload (z is the slab normal).  The slab fills
    z in [zs, zs + slab) with zs = nz/2 - slab/2, the gyrotropic layer the
    `layer` cells below it; the lattice of air holes (period, radius) runs
    through the slab with the centre hole left out; the soft Ez dipole sits
    at the centre of that defect.  Source centre wavelength lambda0 =
    period / a_over_lambda; the gyrotropic tensor is fitted at its angular
    frequency; the flux box is the dipole +- box_half cells on every axis with
    nfreq frequencies over the pulse's -20 dB band.  structure=False gives the
    same grid, source and box in vacuum (the W0 run of a Purcell ratio).
    Inside the CPML slabs the layer is the plain dielectric eps_diag: a
    magnetised-Drude current inside the CPML grows without bound late in long
    runs (measured with the FP64 oracle: the field norm of a 64 x 64 x 96 cut
    rises 25-fold between steps 5500 and 8000 with the layer running through
    the absorber, and keeps decaying with the dielectric there)."""
    nx, ny, nz = n
    lambda0 = period / a_over_lambda
    w0 = 2.0 * math.pi / lambda0
    cfg = abi.make_config(nx, ny, nz, dx=1.0, courant=courant, order=order, pml=pml, probe_capacity=steps + 8)
    d = (nx // 2, ny // 2, nz // 2)
    zs = nz // 2 - slab // 2
    einf, gyro = abi.gyro_for(eps_diag, g, w0)
    mats = [abi.make_material(1.0), abi.make_material(eps_slab), abi.make_material(eps_inf=einf, gyro=gyro),
            abi.make_material(eps_diag)]
    idx = None
    if structure:
        idx = []
        for c in range(3):
            a = np.zeros((nx, ny, nz), np.uint8)
            zo = 0.5 if c < 2 else 0.0                       # Ex, Ey sit at k + 1/2, Ez at k
            z = np.arange(nz) + zo
            in_slab = (z >= zs) & (z < zs + slab)
            in_layer = (z >= zs - layer) & (z < zs)
            holes = triangular_holes(nx, ny, (d[0] + 0.5, d[1] + 0.5), period, radius, c)
            k0, k1 = int(np.argmax(in_slab)), int(nz - np.argmax(in_slab[::-1]))
            a[:, :, k0:k1] = np.where(holes, 0, 1).astype(np.uint8)[:, :, None]
            if in_layer.any():
                l0, l1 = int(np.argmax(in_layer)), int(nz - np.argmax(in_layer[::-1]))
                a[:, :, l0:l1] = 3
                a[pml:nx - pml, pml:ny - pml, max(l0, pml):min(l1, nz - pml)] = 2
            idx.append(a)
    f0, tau, t0 = gauss_sine_params(lambda0)
    src = abi.PointSource(comp=abi.EZ, i=d[0], j=d[1], k=d[2], waveform=abi.WAVE_GAUSS_SINE, amp=1.0, f0=f0,
                          tau=tau, t0=t0)
    df = math.sqrt(math.log(10.0)) / (math.pi * tau)
    omegas = 2.0 * math.pi * np.linspace(f0 - df, f0 + df, nfreq)
    lo = [v - box_half for v in d]
    hi = [v + box_half for v in d]
    if structure:
        desc = ("%dx%dx%d: slab %d cells eps=%g, triangular air holes period %d r=%d, %d-cell gyrotropic layer "
                "(eps_diag=%g, g=%g, magnetised Drude), Ez dipole in a missing-hole defect, %d-cell CPML, "
                "%d-freq FP64 flux box +-%d" % (nx, ny, nz, slab, eps_slab, period, radius, layer, eps_diag, g, pml,
                                               nfreq, box_half))
    else:
        desc = ("%dx%dx%d vacuum, the same Ez dipole (lambda0=%g), %d-cell CPML, %d-freq FP64 flux box +-%d"
                % (nx, ny, nz, lambda0, pml, nfreq, box_half))
    return dict(name="gyro_crystal_purcell", cfg=cfg, materials=(mats if structure else None, idx),
                point_sources=[src], tfsf=None, probes=[(abi.EZ, d[0], d[1], d[2], abi.PROBE_NODE)], dft=[],
                flux=[(lo, hi, omegas)], steps=steps, eps_src=eps_slab if structure else 1.0, desc=desc)


def apply_flux(sim, sc):
    """Add the scenario's flux boxes to a Simulation; returns their ids."""
    return [sim.add_flux_box(lo, hi, om) for (lo, hi, om) in sc.get("flux", [])]


def apply(sim, sc):
    """Apply a scenario dict to a Simulation (or any object with its surface)."""
    mats, idx = sc["materials"]
    if mats is not None:
        sim.set_materials(mats, idx[0], idx[1], idx[2])
    for s in sc["point_sources"]:
        sim.add_point_source(s)
    if sc["tfsf"] is not None:
        sim.set_tfsf(sc["tfsf"])
    for (c, i, j, k, m) in sc["probes"]:
        sim.add_probe(c, i, j, k, m)
    ids = []
    for (axis, index, mask, om) in sc["dft"]:
        ids.append(sim.add_dft_plane(axis, index, mask, om))
    return ids


def design_block_instance(seed, edges=(64, 96, 128, 160, 192, 224, 256), pml=10, steps=1500, nblocks=8,
                          design=16, lambda0=24.0, order=2, courant=0.5):
    """One instance of the batched workload: each axis edge drawn from
    `edges`, `nblocks` random dielectric blocks with eps ~ U[1, 12], one Ez
    dipole at a random interior position, a CPML of `pml` cells and a
    `design`^3 per-node permittivity region at the centre (initialised to
    U[1, 12]); the objective is the flux through the plane x = nx - pml - 4
    at lambda0.  The gradient is taken with respect to the design region."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(v) for v in rng.choice(edges, size=3))
    cfg = abi.make_config(nx, ny, nz, dx=1.0, courant=courant, order=order, pml=pml)
    idx = np.zeros((nx, ny, nz), np.uint8)
    mats = [abi.make_material(1.0)]
    lo_d = [n // 2 - design // 2 for n in (nx, ny, nz)]
    for b in range(nblocks):
        size = rng.integers(4, 17, size=3)
        lo = [int(rng.integers(pml + 1, n - pml - s - 1)) for n, s in zip((nx, ny, nz), size)]
        mats.append(abi.make_material(float(rng.uniform(1.0, 12.0))))
        idx[lo[0]:lo[0] + size[0], lo[1]:lo[1] + size[1], lo[2]:lo[2] + size[2]] = len(mats) - 1
    # the source stays outside the design region and away from the absorber
    while True:
        p = [int(rng.integers(pml + 4, n - pml - 4)) for n in (nx, ny, nz)]
        if not all(lo_d[a] - 2 <= p[a] < lo_d[a] + design + 2 for a in range(3)):
            break
    f0, tau, t0 = gauss_sine_params(lambda0)
    src = abi.PointSource(comp=abi.EZ, i=p[0], j=p[1], k=p[2], waveform=abi.WAVE_GAUSS_SINE, amp=1.0, f0=f0, tau=tau,
                          t0=t0)
    eps = rng.uniform(1.0, 12.0, size=(3, design, design, design)).astype(np.float32)
    return dict(name="design_block_instance", cfg=cfg, materials=(mats, [idx, idx, idx]), point_sources=[src],
                tfsf=None, probes=[], dft=[], steps=steps, design=(tuple(lo_d), eps), plane_x=nx - pml - 4,
                omega=2 * math.pi / lambda0,
                desc="%dx%dx%d, %d blocks eps~U[1,12], Ez dipole, %d-cell CPML, %d^3 design region" %
                     (nx, ny, nz, nblocks, pml, design))


def design_region(n=(256, 256, 192), design=(64, 64, 32), pml=10, lambda0=24.0, steps=2000, seed=0, order=2,
                  courant=0.5):
    """Differentiation workload: a centred design region of per-node
    permittivity eps ~ U[1, 12] (seed), an Ez dipole between the design
    region and the low-x absorber, and the Poynting flux at lambda0 through
    the plane x = nx - pml - 4 as the objective."""
    nx, ny, nz = n
    cfg = abi.make_config(nx, ny, nz, dx=1.0, courant=courant, order=order, pml=pml)
    lo = tuple((m - d) // 2 for m, d in zip(n, design))
    eps = np.random.default_rng(seed).uniform(1.0, 12.0, size=(3,) + tuple(design)).astype(np.float32)
    f0, tau, t0 = gauss_sine_params(lambda0)
    src = abi.PointSource(comp=abi.EZ, i=(pml + lo[0]) // 2, j=ny // 2, k=nz // 2, waveform=abi.WAVE_GAUSS_SINE,
                          amp=1.0, f0=f0, tau=tau, t0=t0)
    return dict(name="design_region", cfg=cfg, materials=(None, None), point_sources=[src], tfsf=None, probes=[],
                dft=[], steps=steps, design=(lo, eps), plane_x=nx - pml - 4, omega=2 * math.pi / lambda0,
                desc="%dx%dx%d, %dx%dx%d design region eps~U[1,12] (seed %d), Ez dipole, %d-cell CPML, "
                     "flux at lambda0=%g through x=%d" % (nx, ny, nz, design[0], design[1], design[2], seed, pml,
                                                            lambda0, nx - pml - 4))
