/*
 * dtmx.h -- C ABI of the B200-native DiamondTorre-style FDTD engine.
 *
 * Plain C, plain pointers and sizes; no exceptions cross this boundary and
 * every entry point returns a status code (DTMX_OK or DTMX_ERR_*), where the
 * reference printed a message and called exit() (params.h:130-136,
 * DTmxw.cu:281-336).
 *
 * Units follow the reference: c = 1 (eps0 = mu0 = 1); E is advanced by
 * curl(H)*dt/eps and H by -curl(E)*dt (defs.h:11-13, genAlg.py:182-301).
 *
 * Lattice.  Cell (i,j,k) of an nx*ny*nz grid carries six nodes whose
 * coordinates in half-cell units (X,Y,Z) are
 *     Ex (2i, 2j+1, 2k+1)   Ey (2i+1, 2j, 2k+1)   Ez (2i+1, 2j+1, 2k)
 *     Hx (2i+1, 2j, 2k)     Hy (2i, 2j+1, 2k)     Hz (2i, 2j, 2k+1)
 * which is the reference's V (=E, two odd coordinates) / T (=H, one odd
 * coordinate) lattice (genAlg.py:24, DTmxw.cu:77-83).  Host arrays exchanged
 * through this ABI are dense nx*ny*nz float arrays, z fastest (index
 * (i*ny + j)*nz + k).
 *
 * Threading: one context per host thread; calls on one context must be
 * serialised by the caller.  Kernels run asynchronously on the context's
 * own CUDA stream; read-back calls synchronise that stream.
 */
#ifndef DTMX_H
#define DTMX_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DTMX_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
enum {
  DTMX_OK = 0,
  DTMX_ERR_INVALID = 1,      /* bad argument / configuration (Courant, sizes, ...) */
  DTMX_ERR_CUDA = 2,         /* CUDA runtime error (message in dtmx_last_error) */
  DTMX_ERR_OOM = 3,          /* device allocation failed */
  DTMX_ERR_NONFINITE = 4,    /* NaN/Inf found by dtmx_check_finite */
  DTMX_ERR_TIMEOUT = 5,      /* a bounded device wait gave up (flag set by a kernel) */
  DTMX_ERR_STATE = 6,        /* call not valid in the current state */
  DTMX_ERR_UNSUPPORTED = 7,  /* combination not implemented */
  DTMX_ERR_NODEVICE = 8,     /* no CUDA device visible */
  DTMX_ERR_TOO_LARGE = 9     /* input larger than a fixed-size scratch allows */
};

/* ---- field components -------------------------------------------------- */
enum { DTMX_EX = 0, DTMX_EY = 1, DTMX_EZ = 2, DTMX_HX = 3, DTMX_HY = 4, DTMX_HZ = 5 };

/* ---- geometry / boundary modes ----------------------------------------- */
enum {
  /* Plain box: every node of the nx*ny*nz array is updated, the field is
   * zero outside the array (PEC-like outer wall behind the absorber). */
  DTMX_GEOM_BOX = 0,
  /* The reference's domain (window.hpp:126-145, defs.h:39-81, genAlg.py:8-10,
   * 166-168,199-201): nx = 3*Np, ny = 3*Na, nz = Nv cells; nodes with
   * X <= 3 or X >= 2*nx-3 are held at zero (isOutS); Y < 0 mirrors Y -> -Y
   * with H odd and E even (I-kernel free reflection); Y > 2*ny-3 mirrors
   * evenly about Y = 2*ny-3 (X-kernel); Z mirrors evenly about Z = 0 and
   * Z = 2*nz-1 (Vrefl). */
  DTMX_GEOM_REFERENCE = 1
};

enum {
  DTMX_ABS_NONE = 0,
  DTMX_ABS_CPML = 1,       /* convolutional PML (Roden-Gedney), DTMX_GEOM_BOX only */
  DTMX_ABS_SPLIT_PML = 2   /* Berenger split-field PML with the reference grading
                              (DTmxw.cu:220-265, genAlg.py:117-148), GEOM_REFERENCE only */
};

typedef struct dtmx_config {
  int nx, ny, nz;            /* cells */
  double dx, dy, dz, dt;     /* grid steps and time step (c = 1) */
  int order;                 /* 2 (Yee) or 4 (reference (27,-1)/24 stencil, defs.h:3-13) */
  int geometry;              /* DTMX_GEOM_* */
  int absorber;              /* DTMX_ABS_* */
  int pml[3][2];             /* absorber thickness in cells, [axis][lo,hi]; 0 = none on that face */
  /* CPML grading: sigma = sigma_max*(d/L)^m, kappa = 1+(kappa_max-1)(d/L)^m,
   * alpha = alpha_max*(1-d/L); sigma_max = cpml_sigma_factor*0.8*(m+1)/d_axis.
   * Zero values select m=3, factor=1, kappa_max=1, alpha_max=0. */
  double cpml_m, cpml_sigma_factor, cpml_kappa_max, cpml_alpha_max;
  /* Split-PML grading: reference TFSFsrc.V_max (signal.hpp:191-199 sets it to c). */
  double spml_vmax;
  /* Probe samples are recorded after every probe_every-th step (reference:
   * once per calcStep of Ntime steps, diamond.cu:473-475).  0 = every step. */
  int probe_every;
  /* Capacity of the probe trace buffer in samples per probe (0 = 4096). */
  int probe_capacity;
  /* 1: the context's device arrays can be parked (dtmx_park) -- each is a
   * CUDA virtual-memory reservation with its own physical allocation, rounded
   * up to the allocation granularity.  0: plain device allocations. */
  int parkable;
  int reserved[7];
} dtmx_config;

/* ---- materials ----------------------------------------------------------- */
enum { DTMX_POLE_LORENTZ = 0, DTMX_POLE_DRUDE = 1 };
#define DTMX_MAX_POLES 2
#define DTMX_MAX_MATERIALS 64

typedef struct dtmx_material {
  /* Non-dispersive part: E update coefficient 1/eps per axis (CoffStruct
   * depsXX/YY/ZZ, defs.h:88-118). */
  double eps[3];
  /* Dispersive part (DispStruct::set, dispersion.cpp:41-82): active when
   * npoles > 0; then eps_inf and sigma are used and eps[] is ignored in the
   * cell, as the reference's ISDISP branch bypasses coffV (genAlg.py:258,319). */
  int npoles;
  int pole_kind[DTMX_MAX_POLES];        /* DTMX_POLE_LORENTZ / DTMX_POLE_DRUDE */
  double pole[DTMX_MAX_POLES][4];       /* Deps, wp, gp, gp_ (LorenzDisp::set/setDrude) */
  double eps_inf;
  double sigma;
  /* Gyrotropic magnetised-Drude current (no reference counterpart: the
   * reference's Gyration() is disabled, genAlg.py:303-304): plasma frequency
   * wp, collision rate gamma and cyclotron frequency wc (bias along +z).
   * Active when gyro_wp > 0; then eps_inf is the background permittivity,
   * eps[] is ignored and npoles must be 0.  With J on the E nodes:
   *   eps_inf dE/dt = curl H - J,   dJ/dt = -gamma J + wp^2 E + wc J x z,
   * stepped as J_x <- a (cos th J_x + sin th <J_y>) + b E_x,
   *            J_y <- a (cos th J_y - sin th <J_x>) + b E_y,  J_z <- a J_z + b E_z,
   * a = exp(-gamma dt), th = wc dt, b = wp^2 dt, <.> the 4-node average of
   * the other component around the node; then E += dt/eps_inf (curl H - J).
   * Keep these nodes out of the CPML slabs: the CPML recursion does not
   * account for the current, and a gyrotropic layer running through the
   * absorber was measured to grow without bound after some thousands of
   * steps (use a plain dielectric of the same diagonal permittivity there). */
  double gyro_wp, gyro_gamma, gyro_wc;
  double reserved[4];
} dtmx_material;

/* ---- sources --------------------------------------------------------------- */
enum {
  DTMX_WAVE_GAUSS_SINE = 0   /* amp*sin(2*pi*f0*(t-t0))*exp(-((t-t0)/tau)^2) */
};

typedef struct dtmx_point_source {
  int comp;                  /* DTMX_EX..DTMX_EZ: soft source added to that E node */
  int i, j, k;
  int waveform;
  double amp, f0, tau, t0;
} dtmx_point_source;

enum {
  DTMX_TFSF_DIPOLE = 0,      /* analytic z-dipole field, reference DipoleTFSF (signal.hpp:51-97) */
  DTMX_TFSF_PLANE_X = 1      /* +x propagating, Ez-polarised plane wave from a 1-D auxiliary grid */
};

typedef struct dtmx_tfsf {
  int kind;
  /* Total-field box in physical units (reference TFSFsrc Box{M,P}{s,a,v});
   * a node is inside when strictly between both faces on every axis, with
   * the reference's single-precision position arithmetic (inSF, signal.hpp:153-160). */
  double box_lo[3], box_hi[3];
  /* Dipole parameters (TFSFsrc::set, signal.hpp:99-115): */
  double c, w, kenv;
  /* Corrections are applied while (floor(n/ntime)+1)*ntime*dt < tstop
   * (window.hpp:125-132); tstop <= 0 means always. ntime 0 means 1. */
  double tstop;
  int ntime;
  /* Plane wave (kind DTMX_TFSF_PLANE_X): Ez_inc(x,t) from a 1-D line driven by
   * amp*sin(2*pi*f0*(t-t0))*exp(-((t-t0)/tau)^2) at the line's left end. */
  double amp, f0, tau, t0;
  /* Slab of a larger grid (x slabs of dtmaxwell4_b200.window): x_origin is
   * the whole grid's cell index of this grid's plane 0 and x_cells the whole
   * grid's cells along x (both 0 for a whole grid).  box_lo/box_hi stay in
   * the whole grid's coordinates: the dipole sits at its global position and
   * the plane wave's 1-D line spans the whole grid, so every slab integrates
   * the same line.  Box faces outside this grid are left to the slabs that
   * hold them; the boundary checks apply to the grid's uncut x ends only. */
  double x_origin, x_cells;
  double reserved[2];
} dtmx_tfsf;

/* ---- probes ---------------------------------------------------------------- */
enum {
  DTMX_PROBE_NODE = 0,       /* the single node of the component at cell (i,j,k) */
  DTMX_PROBE_REFERENCE = 1   /* reference Sensor averaging: 4 E nodes / 2 H nodes
                                around cell point (x,y,z) (sensor.h:51-83) */
};

/* ---- context --------------------------------------------------------------- */
typedef struct dtmx_ctx dtmx_ctx;

int  dtmx_version(void);
const char* dtmx_error_string(int code);

/* Validate cfg and allocate device state on the current CUDA device.
 * Replaces GeoParamsHost::set + init_index (DTmxw.cu:278-487, 502-561). */
int  dtmx_create(const dtmx_config* cfg, dtmx_ctx** out);
void dtmx_destroy(dtmx_ctx* ctx);
const char* dtmx_last_error(const dtmx_ctx* ctx);

/* Material table and per-component material index arrays (nx*ny*nz uint8,
 * z fastest); idx_y/idx_z may be NULL to reuse idx_x.  Replaces
 * init_material + the coffs/DispCoffs __constant__ tables (DTmxw.cu:604-706). */
int  dtmx_set_materials(dtmx_ctx* ctx, const dtmx_material* table, int nmat,
                        const uint8_t* idx_x, const uint8_t* idx_y, const uint8_t* idx_z);

int  dtmx_add_point_source(dtmx_ctx* ctx, const dtmx_point_source* src);
/* One TF/SF source per context (reference __constant__ TFSFsrc src, signal.hpp:11). */
int  dtmx_set_tfsf(dtmx_ctx* ctx, const dtmx_tfsf* src);

/* Probes (reference Sensor, sensor.h:6-84).  Coordinates are cell indices. */
int  dtmx_add_probe(dtmx_ctx* ctx, int comp, int i, int j, int k, int mode, int* id_out);
/* Copies traces into out[probe*max_samples + s]; *nsamples gets the count. */
int  dtmx_read_probes(dtmx_ctx* ctx, float* out, int max_samples, int* nsamples);

/* Running DFT on the plane {axis = index}; comp_mask bit c selects component c.
 * FP64 complex accumulators sum f(t_n) * exp(-i*omega*t_n) * dt, with t_n the
 * component's own time level (E at n*dt, H at (n-1/2)*dt after step n). */
int  dtmx_add_dft_plane(dtmx_ctx* ctx, int axis, int index, int comp_mask,
                        int nfreq, const double* omegas, int* id_out);
/* out: [ncomp_selected][nfreq][plane points][2] doubles, plane points in
 * (slow, fast) order of the two remaining axes. */
int  dtmx_read_dft(dtmx_ctx* ctx, int id, double* out, size_t out_len);
/* Running DFT on the n1 x n2 window starting at (lo1, lo2) of the plane
 * {axis = index}, the two in-plane axes in (slow, fast) order; read back with
 * dtmx_read_dft like a plane (window points in place of plane points).
 * dtmx_add_dft_plane is the full-plane window. */
int  dtmx_add_dft_patch(dtmx_ctx* ctx, int axis, int index, int lo1, int n1, int lo2, int n2,
                        int comp_mask, int nfreq, const double* omegas, int* id_out);

/* Power flux box (no reference counterpart: the reference estimates the
 * Purcell factor from the field at the dipole, purcell.gp:3, after an offline
 * Fourier transform, calc_purcell.sh).  Six DFT windows of the tangential E
 * and H components on the faces {axis a = lo[a]} and {axis a = hi[a]}, each
 * covering [lo_b, hi_b) x [lo_c, hi_c) of the other two axes (nodes of those
 * cell indices).  The outward flux of a face normal to axis a is
 *   sign * d_b * d_c * sum Re(E_b conj(H_c) - E_c conj(H_b)),
 * (a, b, c) cyclic, sign -1 on the lo face and +1 on the hi face, accumulated
 * in FP64 on the device from the running DFTs (dtmx_add_dft_plane's
 * convention).  The box also records the tangential H one plane beyond each
 * face, for dtmx_ntff.  Requires 0 <= lo[a] < hi[a] < n[a] - 1. */
int  dtmx_add_flux_box(dtmx_ctx* ctx, const int lo[3], const int hi[3], int nfreq,
                       const double* omegas, int* id_out);
/* out[7*nfreq]: the outward flux of the faces (x lo, x hi, y lo, y hi, z lo,
 * z hi), nfreq values each, then their sum. */
int  dtmx_read_flux(dtmx_ctx* ctx, int id, double* out, size_t out_len);
/* DFT ids of the six face windows (same order), for dtmx_read_dft. */
int  dtmx_flux_faces(dtmx_ctx* ctx, int id, int faces[6]);
/* Near-to-far-field transform of flux box id (surface equivalence, FP64 on
 * the device; no reference counterpart).  For every direction (theta[d],
 * phi[d]) (polar angle from +z, azimuth from +x) and frequency f:
 *   out[(d*nfreq + f)*5 + 0]   radiation intensity U, normalised so that its
 *                              integral over the sphere equals the box's
 *                              dtmx_read_flux total in free space (the
 *                              transform uses the free-space Green's function:
 *                              the box surface must lie in vacuum),
 *   out[...+1 .. +4]           r E_theta and r E_phi (re, im) without the
 *                              exp(-i k r) factor, phase referred to origin
 *                              (physical units; NULL = the box centre).
 * The currents lie on the surface of the tangential E (half a cell outside
 * each face plane along its normal), with H averaged onto it from the face
 * plane and the next one; in the plane every component enters at its own
 * Yee position; k = omega. */
int  dtmx_ntff(dtmx_ctx* ctx, int id, int ndir, const double* theta, const double* phi,
               const double* origin, double* out, size_t out_len);

/* Advance nsteps leapfrog steps (H half step then E half step each,
 * genAlg.py:420-501).  Asynchronous on the context stream.  Replaces
 * calcStep (diamond.cu:335-506), which advanced Ntime steps per call. */
int  dtmx_step(dtmx_ctx* ctx, int nsteps);
int  dtmx_sync(dtmx_ctx* ctx);
int  dtmx_get_step(const dtmx_ctx* ctx, int64_t* n);

/* Field access (host buffers, nx*ny*nz floats, z fastest). */
int  dtmx_get_field(dtmx_ctx* ctx, int comp, float* host_out);
int  dtmx_set_field(dtmx_ctx* ctx, int comp, const float* host_in);
/* Device pointer of a component and its element strides (x, y, z). */
int  dtmx_field_device_ptr(dtmx_ctx* ctx, int comp, void** dptr, int64_t strides[3]);

/* Host-side NaN/Inf check of the probe traces and a device reduction over E;
 * returns DTMX_ERR_NONFINITE if any is found. */
int  dtmx_check_finite(dtmx_ctx* ctx);

/* Number of kernels this context has launched so far. */
int  dtmx_kernel_launches(const dtmx_ctx* ctx, int64_t* n);

/* Bound of every device-side wait of this context's kernels (staged copies,
 * wavefront neighbours), in polls; polls <= 0 restores the default 2^26.
 * A wait that runs out sets an error word, the CTA stops issuing copies,
 * waits for those in flight and returns, and the next dtmx_sync reports
 * DTMX_ERR_TIMEOUT (the results of that step are not valid).  Lowering it
 * exists to exercise that path in tests without a hang. */
int  dtmx_set_wait_limit(dtmx_ctx* ctx, int64_t polls);

/* The context's CUDA stream (cudaStream_t), for event timing by the caller. */
int  dtmx_get_stream(dtmx_ctx* ctx, void** stream);

/* Per-kernel device timing: when enabled, CUDA events bracket the H and E
 * field kernels; dtmx_read_profile returns their summed milliseconds and the
 * number of timed launches of each since profiling was enabled. */
int  dtmx_set_profiling(dtmx_ctx* ctx, int enable);
int  dtmx_read_profile(dtmx_ctx* ctx, double* ms_h, double* ms_e, int64_t* count);

/* sizeof of the ABI structs, in the order config, material, point_source,
 * tfsf, tfsfsrc, ref_globals (for binding checks). */
int  dtmx_abi_sizes(int64_t out[6]);

/* ---- the reference's driver surface (SWIG module DTmxw, mxw.i:1-36) ------ */

/* TFSFsrc (py_consts.h:73-91): the shotpoint the Python driver fills in. */
typedef struct dtmx_tfsfsrc {
  double tStop;
  double srcXs, srcXa, srcXv, sphR;
  double BoxMs, BoxPs, BoxMa, BoxPa, BoxMv, BoxPv;
  double V_max;
  int start;
  double wavelength, w, k, Omega, kEnv, theta, phi;
  double cSrc, Imp;
  double t0, tw, T;
} dtmx_tfsfsrc;

/* Compile-time constants of the reference (py_consts.h, params.h:44-62) as
 * run-time values: grid in rags (x = 3*Np, y = 3*Na cells, z = Nv cells),
 * window Ns and big-step length Ntime, steps, the run length Tsteps, and the
 * split-PML sizes Npmlx, Npmly (in half rags: Npmlx/2 rags of NDT = 3 cells
 * on each x face) and Npmlz (Npmlz/2 layers at the top z face),
 * py_consts.h:67-69; values <= 0 select the reference's 10, 10, 32. */
typedef struct dtmx_ref_globals {
  int Np, Na, Nv, Ns, Ntime;
  double ds, da, dv, dt;
  int Tsteps;
  int Npmlx, Npmly, Npmlz;
} dtmx_ref_globals;

/* TFSFsrc::set (signal.hpp:99-115). */
void dtmx_tfsfsrc_set(dtmx_tfsfsrc* s, double c, double impedance, double lmb);

/* Material index arrays (nx*ny*nz each, z fastest) of the reference's analytic
 * geometry, get_mat_indev (defs.h:128-148): Ag film with a hole lattice,
 * organic, ITO and glass layers; indices into dtmx_ref_material_table. */
int  dtmx_ref_materials(const dtmx_ref_globals* g, uint8_t* idx_x, uint8_t* idx_y, uint8_t* idx_z);
/* Their material table (init_material, DTmxw.cu:604-635); returns the count. */
int  dtmx_ref_material_table(dtmx_material* out, int n);

/* The reference's _main with --test (DTmxw.cu:731-834): reference geometry
 * (get_mat_indev, defs.h:128-148) and materials (init_material), split PML,
 * TF/SF dipole from the shotpoint, the default sensor line of init_index
 * written to <drop_dir>/<fld>-xXXXXXyYYYYYzZZZZZ.dat once per Ntime steps, and
 * Tsteps/Ntime calls of dtmx_step(Ntime) (calcStep).  With --drop_data (the
 * reference's compile-time DROP_DATA switch, py_consts.h:18) every big step
 * also writes <drop_dir>/ragEz_NNNNN.arr like SeismoDrops::drop
 * (drop.cu:83-107): int32 header {12,0,0,0,3,4,Nv,Na,Np}, then per rag
 * (x < Np, y < Na) and z < Nv the Ez node of the rag's first V domain, the
 * node of cell (3x-1, 3y-1, z) (0 where that cell lies outside the grid).
 * Returns 0 on success. */
int  dtmx_ref_main(const dtmx_ref_globals* g, const dtmx_tfsfsrc* shotpoint, int argc, char** argv);

/* ---- differentiation (no reference counterpart: the reference has no
 * gradient path) -------------------------------------------------------------- */

/* Per-node permittivity of the three E components over the cell box
 * [lo, lo+n): eps holds 3*n0*n1*n2 values (component-major, z fastest).  Inside
 * the box it replaces the permittivity of non-dispersive materials; a node
 * whose material is dispersive keeps its ADE update (and its gradient in
 * dtmx_forward_adjoint is 0).  Set before the first step. */
int  dtmx_set_design(dtmx_ctx* ctx, const int lo[3], const int n[3], const float* eps);

/* Advance nsteps from the current state and return the objective
 *   J = sum over the plane x = plane_x of Re(Ey^ conj(Hz^) - Ez^ conj(Hy^)),
 * the Poynting flux of the running DFTs at omega (E^ = sum_s E^s e^{-i w s dt} dt,
 * H^ with t = (s - 1/2) dt), and dJ/d eps at every design node (3*nd floats,
 * the layout of dtmx_set_design).  The gradient is the discrete adjoint of the
 * update (transposed stencils, CPML recursions and Drude/Lorentz ADE
 * recursions of countDisp, dispersion.cpp:85-99), run backward over the
 * steps; the accumulation is in double precision.  The adjoint needs, of the
 * forward run, only E in the design region at every step: when that history
 * ((nsteps+1) * 3 * nd floats) fits the budget of dtmx_set_adjoint_memory the
 * forward pass records it and nothing is recomputed; otherwise the state is
 * checkpointed every checkpoint_every steps in device memory and each segment
 * is recomputed before its adjoint.  Both modes give bit-identical results.
 * Box geometry, CPML or no absorber, no gyrotropic node in the design region, no point source
 * inside the design region.  On return the context holds the state after
 * nsteps, as after dtmx_step(nsteps).  The run's device buffers (adjoint
 * fields, history or checkpoints) come from the device's stream-ordered memory
 * pool and return to it afterwards; the pool keeps them for later runs. */
int  dtmx_forward_adjoint(dtmx_ctx* ctx, int nsteps, int checkpoint_every, int plane_x, double omega,
                          double* objective, float* grad_eps);

/* Device memory the adjoint may use for the recorded design-region history:
 * bytes >= 0 sets the budget (0 always checkpoints and recomputes), a negative
 * value restores the default, a quarter of the free device memory. */
int  dtmx_set_adjoint_memory(dtmx_ctx* ctx, int64_t bytes);

/* A batch of independent dtmx_forward_adjoint runs (contexts of any sizes,
 * same nsteps and checkpoint_every): every phase is issued step by step for
 * all contexts, each on its own stream, so their kernels run concurrently.
 * plane_x, omega and objectives have n entries, grads n pointers of 3*nd_b
 * floats.  Results equal those of n separate dtmx_forward_adjoint calls. */
int  dtmx_batch_forward_adjoint(dtmx_ctx* const* ctxs, int n, int nsteps, int checkpoint_every, const int* plane_x,
                                const double* omega, double* objectives, float* const* grads);

/* ---- files (reference field drops, drop.cu:45-107; restart) ------------------ */

/* Write component comp as an .arr file: int32 header {12, 0, 0, 0, 3, 4, nz,
 * ny, nx} followed by nx*ny*nz floats, z fastest (the reference's drop layout
 * with dense cells instead of one value per rag). */
int  dtmx_write_arr(dtmx_ctx* ctx, int comp, const char* path);
/* Save / restore the complete time-stepping state (fields, absorber and
 * dispersive state, step counter, plane-wave line) of a context; a context set
 * up the same way that loads the file continues the saved run bit for bit.
 * Probe traces and DFT accumulators are not included. */
int  dtmx_save_state(dtmx_ctx* ctx, const char* path);
int  dtmx_load_state(dtmx_ctx* ctx, const char* path);

/* Count NaN/Inf values in nfields caller-owned device arrays of nelem floats
 * each, without allocating any device memory (no cudaMalloc/cudaFree and no
 * allocating library routine).  For callers that cannot allocate: processes
 * whose device memory is reserved by another allocator, or health-check
 * threads that must stay out of the allocator.  No counterpart in the
 * reference.  The reduction's scratch is a fixed file-scope device array of
 * one count per block of DTMX_NOALLOC_BLOCK_ELEMS elements, so:
 *   - each field is cut into ceil(nelem / DTMX_NOALLOC_BLOCK_ELEMS) blocks
 *     and nfields times that must not exceed DTMX_NOALLOC_MAX_BLOCKS, else
 *     DTMX_ERR_TOO_LARGE (nothing is launched).  That allows
 *     DTMX_NOALLOC_MAX_ELEMS (2^24) floats in all when nelem is a multiple of
 *     the block size, fewer otherwise;
 *   - the first call on a device looks up that array's device address with the
 *     device current; make that first call before any stream capture;
 *   - calls whose work overlaps on the GPU race on the shared array.
 * Kernels run on the legacy default stream and the count is copied back
 * synchronously into *count_out.  The legacy default stream does not wait for
 * a context's own stream (created non-blocking): finish the work that writes
 * the arrays first (dtmx_sync, or cudaStreamSynchronize of the writer's
 * stream), else fields still being updated are counted. */
#define DTMX_NOALLOC_BLOCK_ELEMS 4096LL
#define DTMX_NOALLOC_MAX_BLOCKS 4096
#define DTMX_NOALLOC_MAX_ELEMS (DTMX_NOALLOC_BLOCK_ELEMS * DTMX_NOALLOC_MAX_BLOCKS)
int  dtmx_count_nonfinite_noalloc(const float* const* d_fields, int nfields, int64_t nelem, int64_t* count_out);

/* Engine choice for dtmx_step: 0 = auto, 1 = one launch per half step,
 * 2 = L2-resident wavefront (several time steps per launch), 3 = single sweep
 * (one launch per time step updating H and then E over two field buffers; box
 * geometry, order 2, CPML or no absorber).  The reference compiles its kernel
 * families per build (chooseV.h:3-38); here the choice is made at run time. */
int  dtmx_set_engine(dtmx_ctx* ctx, int engine, int time_block);

/* Planes of the x walk per CTA for engines 1 and 3 (0: automatic; engine 3
 * uses at most 64).  The reference fixes its block shape per build
 * (params.h:50-52); dtmx_autotune searches this value. */
int  dtmx_set_xchunk(dtmx_ctx* ctx, int planes);

/* Parking (contexts created with cfg.parkable = 1; no reference counterpart,
 * the reference's out-of-core window streams its domain through the device,
 * window.hpp:177-267): dtmx_park waits for the context's stream, copies every
 * device array to pinned host memory and releases the device memory, keeping
 * the addresses reserved; dtmx_unpark maps device memory at the same
 * addresses again and copies the arrays back.  While parked, every call that
 * touches the context's device state returns DTMX_ERR_STATE.  Several parked
 * contexts then share one GPU's memory, one resident at a time
 * (dtmaxwell4_b200.window steps a grid larger than the device that way). */
int  dtmx_park(dtmx_ctx* ctx);
int  dtmx_unpark(dtmx_ctx* ctx);
/* Device memory that dtmx_park releases on CUDA device `device` is kept, up to
 * `bytes` (< 0: no limit; 0, the default: none), for the next dtmx_unpark of a
 * block of the same size, instead of being returned to the driver; lowering
 * the limit releases what it no longer holds.  For contexts that take turns
 * on one device. */
int  dtmx_set_park_pool(int device, int64_t bytes);

/* The time-stepping state of a run of x planes, handed between contexts of
 * the same y/z configuration (the reference's window hands x slices of its
 * domain between host and device, window.hpp:203-241; here a slab context
 * receives its neighbours' planes).  dtmx_plane_state_floats gives the floats
 * per plane: the six fields (ny*nz each), the four CPML auxiliaries of the y
 * and z absorber slabs (4*(Ly0+Ly1)*nz and 4*ny*(Lz0+Lz1)), and, when the
 * material table has poles (P = most poles of one material), Em, Jp[P] and
 * Jm[P] of the three E components as dense ny*nz planes (zero off the
 * dispersive nodes).  The host buffer is section-major: section s of plane p
 * starts at (section offset)*nplanes + p*(section plane size).
 * dtmx_read_planes fills it for planes [x0, x0+nplanes), dtmx_write_planes
 * stores it back.  Refused (DTMX_ERR_UNSUPPORTED): planes inside an x
 * absorber slab, gyrotropic materials, TF/SF sources and design regions
 * (their state is not per plane); DTMX_ERR_INVALID for planes outside the
 * grid.  Both wait for the context's stream. */
int  dtmx_plane_state_floats(dtmx_ctx* ctx, size_t* floats_per_plane);
int  dtmx_read_planes(dtmx_ctx* ctx, int x0, int nplanes, float* host);
int  dtmx_write_planes(dtmx_ctx* ctx, int x0, int nplanes, const float* host);
/* The same state of planes [src_x0, src_x0 + nplanes) of src copied straight
 * into planes [dst_x0, ...) of dst (same y/z configuration and material
 * table), either context parked or not: a parked context's pinned host copy
 * is read or written, so a slab can take its neighbour's edge planes from,
 * or leave its own in, the neighbour's parked state without a staging
 * buffer.  Same refusals as dtmx_read_planes; waits for both streams. */
int  dtmx_copy_planes(dtmx_ctx* dst, int dst_x0, dtmx_ctx* src, int src_x0, int nplanes);

/* Tile height (y rows) of the single-sweep engine: 16 (default) or 8 (more
 * CTAs for grids of a few million cells; 0 restores 16).  The reference's
 * block shape is a per-build parameter (params.h:50-52); dtmx_autotune
 * searches this value. */
int  dtmx_set_tile_rows(dtmx_ctx* ctx, int rows);

/* The engine configuration dtmx_step uses (as set or as chosen by
 * dtmx_autotune); any pointer may be NULL.  No reference counterpart. */
int  dtmx_get_engine(dtmx_ctx* ctx, int* engine, int* time_block, int* xchunk, int* tile_rows);

/* Time every applicable engine configuration for trial_steps steps from the
 * current state (probes and DFT planes paused; the state is restored after
 * each trial) and keep the fastest: the per-step engine with x chunks of 4 to 64
 * planes per CTA, the single-sweep engine with x chunks of 2 to 64 planes and
 * tiles of 16 or 8 rows, and the wavefront engine with 1, 2 and 4 steps per
 * launch (the reference's block shape and torre height, chosen at run time
 * instead of compiled in, params.h:50-52).  Results are cached per grid shape
 * and feature set. */
int  dtmx_autotune(dtmx_ctx* ctx, int trial_steps, int* engine_out, int* time_block_out, int* xchunk_out,
                   double* ms_per_step_out);

#ifdef __cplusplus
}
#endif
#endif /* DTMX_H */
