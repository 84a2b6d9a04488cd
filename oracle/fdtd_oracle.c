/*
 * fdtd_oracle.c -- CPU restatement of the DTmaxwell4 leapfrog update, used
 * ONLY as test infrastructure (parity checker and the timed CPU baseline).
 * Nothing in the product links or calls this file.
 *
 * Parity status: the reference ships no tests, golden vectors or CPU path.
 * This oracle is pinned (1) by analytic known answers (dispersion relation of
 * the stencils, Drude/Lorentz resonances of the ADE recursion, CPML
 * absorption; tests/test_cpu.py) and (2) against the reference itself: its
 * own CUDA implementation, generated and compiled from its sources for
 * sm_100a by oracle/refbuild/build_ref.py (oracle/_ref), whose FP64 build's
 * field drops over the whole domain (Drude film, split PML, dipole TF/SF,
 * mirror and zero boundaries) match this oracle's FP64 run
 * (tests/test_reference_build.py).
 *
 * Built twice from this one source: REAL=double (prefix orc64_) and
 * REAL=float (prefix orc32_).  Dense SoA fields, z fastest, generic
 * per-node loops, OpenMP over x.
 *
 * What each part restates:
 *   stencil and signs ........ genAlg.py:182-301 (dif = (-f[-3]+f[+3]+27f[-1]-27f[+1])*dt/d/24,
 *                              signs genAlg.py:246-247), defs.h:3-13
 *   lattice / components ..... genAlg.py:24 (T = one odd coord = H, V = two odd = E), DTmxw.cu:77-83
 *   z mirror (Vrefl) ......... defs.h:76-81, defs.h:212-213
 *   y boundaries ............. genAlg.py:8-10,35-38 (isOutA/Ashift), 166-168,199-201 (free reflection)
 *   x zero region ............ defs.h:40 (isOutS), genAlg.py:93-95
 *   split PML ................ genAlg.py:117-148, DTmxw.cu:220-265 (PMLgamma_func, setPMLcoeffs),
 *                              defs.h:45,59-68 (inPMLsync, get_pml_iy/ix), defs.h:206-208 (z)
 *   ADE (Drude/Lorentz) ...... dispersion.cpp:5-99 (LorenzDisp, DispStruct::set, countDisp)
 *   TF/SF tap rule ........... genAlg.py:209-234, signal.hpp:153-160 (inSF)
 *   dipole field ............. signal.hpp:51-97 (DipoleTFSF)
 *   sensors .................. sensor.h:51-83
 *   CPML (new, no reference counterpart) ...... Roden & Gedney, Microw. Opt. Tech. Lett. 27 (2000)
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "dtmx.h"

#ifndef REAL
#define REAL double
#endif
#ifndef PFX
#define PFX(name) orc64_##name
#endif

typedef REAL real;

/* half-cell offsets of each component on the lattice, [comp][axis] */
static const int OFF[6][3] = {
  {0, 1, 1}, {1, 0, 1}, {1, 1, 0},   /* Ex Ey Ez */
  {1, 0, 0}, {0, 1, 0}, {0, 0, 1}    /* Hx Hy Hz */
};

typedef struct { int comp, i, j, k, mode; } probe_t;
typedef struct {
  int axis, index, comp_mask, nfreq, ncomp, n1, n2;
  double* omega;
  double* acc;   /* [ncomp][nfreq][n1*n2][2] */
} dft_t;

typedef struct {
  dtmx_config cfg;
  int nx, ny, nz;
  size_t ncell;
  real* f[6];
  /* boundary per axis & side: type, plane, sign E, sign H */
  int btype[3][2], bplane[3][2], bsE[3][2], bsH[3][2];
  int live_lo[6][3], live_hi[6][3];
  /* absorber slabs: thickness in cells per [axis][side]; storage [axis][slot] */
  int L[3][2];
  real* aux[3][4];
  /* per-axis per-half-coordinate absorber coefficients, length 2*n+2 */
  double* cb[3]; double* ca[3]; double* cik[3];    /* CPML b, a, 1/kappa */
  real*   k1[3]; real* k2[3];                        /* split PML K1, K2 */
  /* materials */
  dtmx_material mat[DTMX_MAX_MATERIALS];
  int nmat;
  uint8_t* midx[3];
  real inv_eps[DTMX_MAX_MATERIALS][3];
  /* ADE coefficients (DispStruct) */
  real kEJ[DTMX_MAX_MATERIALS][3][DTMX_MAX_POLES][2];
  real kE[DTMX_MAX_MATERIALS][3][3];
  real kJ[DTMX_MAX_MATERIALS][3][DTMX_MAX_POLES][5];
  int ade_box[3][2];   /* cell box holding ADE state, [lo, hi) */
  size_t ade_n;
  real* Em[3]; real* Jp[3][DTMX_MAX_POLES]; real* Jm[3][DTMX_MAX_POLES];
  /* gyrotropic current: coefficients per material, double-buffered J over the ADE box */
  int gyro[DTMX_MAX_MATERIALS];
  real gA[DTMX_MAX_MATERIALS], gC[DTMX_MAX_MATERIALS], gS[DTMX_MAX_MATERIALS], gB[DTMX_MAX_MATERIALS];
  real gjc[DTMX_MAX_MATERIALS];
  int has_gyro, gcur;
  real* Jg[2][3];
  /* adjoint runs: the adjoint of the intermediate E' of the dispersive nodes */
  real* amu[3];
  /* design region: per-node 1/eps of each E component over a cell box */
  int des_on, des_lo[3], des_n[3];
  real* des_ie[3];
  /* sources */
  dtmx_point_source psrc[64]; int npsrc;
  int has_tfsf; dtmx_tfsf tfsf;
  int sf_lo[3], sf_hi[3];       /* inclusive half-coordinate range inside the box */
  int sf_xo;                    /* whole-grid cell index of plane 0 (x slabs) */
  int line_M, line_n; double* line_e; double* line_h; int line_src;
  /* monitors */
  probe_t probes[4096]; int nprobes;
  int probe_cap; int nsamples; real* traces;
  dft_t dft[64]; int ndft;
  int64_t step;
} osim;

/* ------------------------------------------------------------------ setup */

static int half_max(const osim* s, int a) { return a == 0 ? 2 * s->nx : a == 1 ? 2 * s->ny : 2 * s->nz; }
static int ncells_axis(const osim* s, int a) { return a == 0 ? s->nx : a == 1 ? s->ny : s->nz; }

/* PMLgamma_func (DTmxw.cu:220-229), identical for the X/Y/Z variants. */
static double ref_pml_gamma(int i, int N, double dstep, double vmax) {
  if (i >= N - 3) return 0.0;
  if (i < 0) i = 0;
  N -= 3;
  double att = 4.0;
  double sigma_max = vmax * log(10000.0) * ((att + 1.0) / (2.0 * (N * dstep * 0.5)));
  double x_max = pow(sigma_max, 1.0 / att);
  double x = x_max - i * (x_max / N);
  return pow(x, att);
}

static void setup_boundaries(osim* s) {
  int n[3] = {s->nx, s->ny, s->nz};
  for (int a = 0; a < 3; a++) {
    if (s->cfg.geometry == DTMX_GEOM_BOX) {
      s->btype[a][0] = 0; s->bplane[a][0] = -1;
      s->btype[a][1] = 0; s->bplane[a][1] = 2 * n[a];
      s->bsE[a][0] = s->bsE[a][1] = s->bsH[a][0] = s->bsH[a][1] = 1;
    }
  }
  if (s->cfg.geometry == DTMX_GEOM_REFERENCE) {
    /* x: isOutS(x) = x<=NDT || x>=Ns*2*NDT-NDT  (defs.h:40) -> zero planes 3 and 2nx-3 */
    s->btype[0][0] = 0; s->bplane[0][0] = 3;
    s->btype[0][1] = 0; s->bplane[0][1] = 2 * s->nx - 3;
    /* y low: I-kernel, nodes y<0 not updated, mirror Y->-Y, H neighbours of E
     * taken with a minus sign (genAlg.py:166-168,199-201) */
    s->btype[1][0] = 1; s->bplane[1][0] = 0; s->bsE[1][0] = 1; s->bsH[1][0] = -1;
    /* y high: X-kernel, nodes with y > YbndX=NDT in the last rag row are not
     * updated, even mirror about it (genAlg.py:9,36): plane 6*Na-3 = 2ny-3 */
    s->btype[1][1] = 1; s->bplane[1][1] = 2 * s->ny - 3; s->bsE[1][1] = 1; s->bsH[1][1] = 1;
    /* z: Vrefl mirrors about Z=0 and Z=2Nv-1 for all fields (defs.h:76-81) */
    s->btype[2][0] = 1; s->bplane[2][0] = 0; s->bsE[2][0] = 1; s->bsH[2][0] = 1;
    s->btype[2][1] = 1; s->bplane[2][1] = 2 * s->nz - 1; s->bsE[2][1] = 1; s->bsH[2][1] = 1;
  }
  for (int c = 0; c < 6; c++)
    for (int a = 0; a < 3; a++) {
      int lo = 0, hi = n[a] - 1;
      /* live: zero side -> H > plane; mirror side -> H >= plane (lo), <= (hi) */
      while (lo <= hi) {
        int H = 2 * lo + OFF[c][a];
        int ok = s->btype[a][0] == 0 ? (H > s->bplane[a][0]) : (H >= s->bplane[a][0]);
        if (ok) break;
        lo++;
      }
      while (hi >= lo) {
        int H = 2 * hi + OFF[c][a];
        int ok = s->btype[a][1] == 0 ? (H < s->bplane[a][1]) : (H <= s->bplane[a][1]);
        if (ok) break;
        hi--;
      }
      s->live_lo[c][a] = lo; s->live_hi[c][a] = hi;
    }
}

static void setup_absorber(osim* s) {
  const dtmx_config* cf = &s->cfg;
  double d[3] = {cf->dx, cf->dy, cf->dz};
  int n[3] = {s->nx, s->ny, s->nz};
  for (int a = 0; a < 3; a++) {
    int H = 2 * n[a] + 2;
    s->cb[a] = calloc(H, sizeof(double)); s->ca[a] = calloc(H, sizeof(double)); s->cik[a] = calloc(H, sizeof(double));
    s->k1[a] = calloc(H, sizeof(real)); s->k2[a] = calloc(H, sizeof(real));
    for (int h = 0; h < H; h++) { s->cik[a][h] = 1.0; s->k1[a][h] = 1; s->k2[a][h] = 1; }
    s->L[a][0] = s->L[a][1] = 0;
  }
  if (cf->absorber == DTMX_ABS_CPML) {
    double m = cf->cpml_m > 0 ? cf->cpml_m : 3.0;
    double fac = cf->cpml_sigma_factor > 0 ? cf->cpml_sigma_factor : 1.0;
    double kmax = cf->cpml_kappa_max >= 1 ? cf->cpml_kappa_max : 1.0;
    double amax = cf->cpml_alpha_max;
    for (int a = 0; a < 3; a++) {
      for (int side = 0; side < 2; side++) {
        int Lc = cf->pml[a][side];
        s->L[a][side] = Lc;
        if (Lc <= 0) continue;
        double smax = fac * 0.8 * (m + 1.0) / d[a];
        for (int h = 0; h < 2 * n[a]; h++) {
          /* depth in cells from the inner interface (lo: X=2L-1, hi: X=2n-2L) */
          double dep = side == 0 ? (2.0 * Lc - 1.0 - h) * 0.5 : (h - (2.0 * n[a] - 2.0 * Lc)) * 0.5;
          if (dep <= 0) continue;
          if (dep > Lc) dep = Lc;
          double r = dep / Lc;
          double sg = smax * pow(r, m);
          double kp = 1.0 + (kmax - 1.0) * pow(r, m);
          double al = amax * (1.0 - r);
          double b = exp(-(sg / kp + al) * cf->dt);
          double aa = (sg > 0) ? sg / (sg * kp + kp * kp * al) * (b - 1.0) : 0.0;
          s->cb[a][h] = b; s->ca[a][h] = aa; s->cik[a][h] = 1.0 / kp;
        }
      }
    }
  } else if (cf->absorber == DTMX_ABS_SPLIT_PML) {
    /* Reference grading (DTmxw.cu:250-265).  K2 = 1/(1+0.5*dt*gamma), K1 = 2*K2-1,
     * computed in double and stored in the field precision (ftype __constant__). */
    double V = cf->spml_vmax;
    /* x: KNpmlx = 2*Npmlx*NDT (params.h:106-108), the slab Npmlx/2 rags of
     * NDT cells = pml[0] cells; index i = X (left) or X - 2nx + KNpmlx
     * (right); gamma(KNpmlx/2-|i-KNpmlx/2|-3, KNpmlx/2-3).  KNpmly, KNpmlz
     * likewise from the y slab and the Npmlz/2 top layers. */
    int KX = 4 * cf->pml[0][0], KY = 4 * cf->pml[1][0], KZ = 4 * cf->pml[2][1];
    int XS = 2 * cf->pml[0][0] - 3;                        /* inPMLsync: Npmlx/2*2*NDT - NDT (defs.h:45) */
    s->L[0][0] = cf->pml[0][0]; s->L[0][1] = cf->pml[0][1];
    s->L[1][0] = cf->pml[1][0]; s->L[1][1] = cf->pml[1][1];
    s->L[2][0] = 0;             s->L[2][1] = cf->pml[2][1];
    for (int h = 0; h < 2 * s->nx + 2; h++) {
      int i = -1;
      if (h < XS) i = h;                                   /* inPMLsync left */
      else if (h >= 2 * s->nx - XS) i = h - 2 * s->nx + KX; /* inPMLsync right */
      if (i < 0 || i >= KX) continue;
      double g = ref_pml_gamma(KX / 2 - abs(i - KX / 2) - 3, KX / 2 - 3, cf->dx, V);
      double k2 = 1.0 / (1.0 + 0.5 * cf->dt * g);
      s->k2[0][h] = (real)k2; s->k1[0][h] = (real)(2.0 * k2 - 1.0);
    }
    for (int h = 0; h < 2 * s->ny + 2; h++) {
      int i = -1;
      if (h < KY / 2) i = h;
      else if (h >= 2 * s->ny - KY / 2) i = h - 2 * s->ny + KY;
      if (i < 0 || i >= KY) continue;
      double g = ref_pml_gamma((i < KY / 2) ? i : (KY - i - 3), KY / 2, cf->dy, V);
      double k2 = 1.0 / (1.0 + 0.5 * cf->dt * g);
      s->k2[1][h] = (real)k2; s->k1[1][h] = (real)(2.0 * k2 - 1.0);
    }
    for (int h = 0; h < 2 * s->nz + 2; h++) {
      /* only the top face absorbs: k2z = 1 for i < KNpmlz/2 (DTmxw.cu:262) */
      int i = h - 2 * s->nz + KZ;
      if (i < KZ / 2 || i >= KZ) continue;
      double g = ref_pml_gamma(KZ - i - 1, KZ / 2, cf->dz, V);
      double k2 = 1.0 / (1.0 + 0.5 * cf->dt * g);
      s->k2[2][h] = (real)k2; s->k1[2][h] = (real)(2.0 * k2 - 1.0);
    }
  }
  for (int a = 0; a < 3; a++) {
    size_t th = (size_t)(s->L[a][0] + s->L[a][1]);
    if (!th) continue;
    size_t cnt = th * (s->ncell / ncells_axis(s, a));
    for (int q = 0; q < 4; q++) s->aux[a][q] = calloc(cnt, sizeof(real));
  }
}

/* slab index of cell (i,j,k) in the axis-a absorber storage, -1 if outside */
static long slab_index(const osim* s, int a, int i, int j, int k) {
  int n = ncells_axis(s, a);
  int c = a == 0 ? i : a == 1 ? j : k;
  int lo = s->L[a][0], hi = s->L[a][1];
  int cs;
  if (c < lo) cs = c;
  else if (c >= n - hi) cs = lo + (c - (n - hi));
  else return -1;
  int th = lo + hi;
  if (a == 0) return ((long)cs * s->ny + j) * s->nz + k;
  if (a == 1) return ((long)i * th + cs) * s->nz + k;
  return ((long)i * s->ny + j) * th + cs;
}

/* absorber storage slot of component c for derivative axis a */
static int slot_of(int c, int a) {
  static const int S[6][3] = {
    {-1, 0, 0}, {0, -1, 1}, {1, 1, -1},
    {-1, 2, 2}, {2, -1, 3}, {3, 3, -1}
  };
  return S[c][a];
}

/* ------------------------------------------------------------ field access */

static inline size_t IDX(const osim* s, int i, int j, int k) { return ((size_t)i * s->ny + j) * s->nz + k; }

/* Value of component c at cell index (i,j,k), applying the boundary rules
 * for indices outside the live range (mirror: reflect with sign; zero: 0). */
static real fetch(const osim* s, int c, int i, int j, int k) {
  int idx[3] = {i, j, k};
  int n[3] = {s->nx, s->ny, s->nz};
  real sign = 1;
  for (int a = 0; a < 3; a++) {
    int v = idx[a];
    int H = 2 * v + OFF[c][a];
    if (v < s->live_lo[c][a]) {
      if (s->btype[a][0] == 0) { if (v < 0) return 0; continue; }
      int H2 = 2 * s->bplane[a][0] - H;
      idx[a] = (H2 - OFF[c][a]) / 2;
      sign *= (c < 3) ? s->bsE[a][0] : s->bsH[a][0];
    } else if (v > s->live_hi[c][a]) {
      if (s->btype[a][1] == 0) { if (v >= n[a]) return 0; continue; }
      int H2 = 2 * s->bplane[a][1] - H;
      idx[a] = (H2 - OFF[c][a]) / 2;
      sign *= (c < 3) ? s->bsE[a][1] : s->bsH[a][1];
    }
  }
  for (int a = 0; a < 3; a++) if (idx[a] < 0 || idx[a] >= n[a]) return 0;
  return sign * s->f[c][IDX(s, idx[0], idx[1], idx[2])];
}

/* ------------------------------------------------------------- TF/SF */

static int in_sf(const osim* s, int X, int Y, int Z) {
  return X >= s->sf_lo[0] && X <= s->sf_hi[0] && Y >= s->sf_lo[1] && Y <= s->sf_hi[1] &&
         Z >= s->sf_lo[2] && Z <= s->sf_hi[2];
}

/* reference DipoleTFSF (signal.hpp:51-97), evaluated in double */
static double dipole_inc(const osim* s, int comp, int X, int Y, int Z, double tt) {
  const dtmx_tfsf* p = &s->tfsf;
  double x = (X + 2 * s->sf_xo) * 0.5 * s->cfg.dx, y = Y * 0.5 * s->cfg.dy, z = Z * 0.5 * s->cfg.dz;
  double t = tt * s->cfg.dt;
  double xd = (p->box_lo[0] + p->box_hi[0]) * 0.5, yd = (p->box_lo[1] + p->box_hi[1]) * 0.5,
         zd = (p->box_lo[2] + p->box_hi[2]) * 0.5;
  double nx_ = x - xd, ny_ = y - yd, nz_ = z - zd;
  double R = sqrt(nx_ * nx_ + ny_ * ny_ + nz_ * nz_);
  double c = p->c, w = p->w, ke = p->kenv;
  double ph = w * t - w / c * R;
  double d = sin(ph) * 0.5 * (1 - cos(ph * ke));
  double ds = w * cos(ph) * 0.5 - 0.5 * w * cos(ph) * cos(ph * ke) + 0.5 * sin(ph) * w * ke * sin(ph * ke);
  double dss = -w * w * sin(ph) * 0.5 + 0.5 * w * w * sin(ph) * cos(ph * ke) +
               0.5 * w * cos(ph) * w * ke * sin(ph * ke) + 0.5 * w * cos(ph) * w * ke * sin(ph * ke) +
               0.5 * sin(ph) * w * ke * w * ke * cos(ph * ke);
  if (ph * ke < 0 || ph * ke > 2 * M_PI) { d = 0; ds = 0; dss = 0; }
  double n0 = nx_ / R, n1 = ny_ / R, n2 = nz_ / R;
  /* vectors d, ds, dss are along z */
  if (comp < 3) {
    /* (dss x n) x n with dss = (0,0,D): dss x n = (-D n1, D n0, 0);
       ((a) x n) = (a1 n2 - a2 n1, a2 n0 - a0 n2, a0 n1 - a1 n0) */
    double a0 = -dss * n1, a1 = dss * n0, a2 = 0;
    double cc[3] = {a1 * n2 - a2 * n1, a2 * n0 - a0 * n2, a0 * n1 - a1 * n0};
    double nn[3] = {n0, n1, n2};
    double e3 = c * (cc[comp] / (c * c * R) +
                     (3 * ds * n2 * nn[comp] - (comp == 2 ? ds : 0)) / (c * R * R) +
                     (3 * d * n2 * nn[comp] - (comp == 2 ? d : 0)) / (R * R * R));
    return e3;
  } else {
    double b1[3] = {-dss * n1, dss * n0, 0};
    double b2[3] = {-ds * n1, ds * n0, 0};
    int q = comp - 3;
    return b1[q] / (c * c * R) + b2[q] / (c * R * R);
  }
}

/* incident value of component g at node (X,Y,Z), time index tt (steps) */
static double inc_value(const osim* s, int g, int X, int Y, int Z, double tt) {
  if (s->tfsf.kind == DTMX_TFSF_DIPOLE) return dipole_inc(s, g, X, Y, Z, tt);
  /* plane wave along +x: only Ez (odd X) and Hy (even X) are non-zero */
  if (g == DTMX_EZ) { int m = (X - 1) / 2 + s->line_M; return (m >= 0 && m < s->line_n) ? s->line_e[m] : 0; }
  if (g == DTMX_HY) { int m = X / 2 + s->line_M; return (m >= 0 && m < s->line_n) ? s->line_h[m] : 0; }
  return 0;
}

static int tfsf_active(const osim* s, int64_t n) {
  if (!s->has_tfsf) return 0;
  if (s->tfsf.tstop <= 0) return 1;
  int nt = s->tfsf.ntime > 0 ? s->tfsf.ntime : 1;
  int64_t istep = n / nt;
  return (double)(istep + 1) * nt * s->cfg.dt < s->tfsf.tstop;
}

/* float semantics of inSF along one axis (signal.hpp:153-160) */
static void sf_range(double dstep, double bm, double bp, int hmax, int* lo, int* hi) {
  float bmf = (float)bm, bpf = (float)bp, df = (float)dstep;
  *lo = 1; *hi = 0;
  int first = 1;
  for (int h = -8; h <= hmax + 8; h++) {
    float sv = (float)((double)h * 0.5 * (double)df);
    if (sv > bmf && sv < bpf) { if (first) { *lo = h; first = 0; } *hi = h; }
  }
}

/* 1-D auxiliary line for the plane wave (same stencil and time step) */
static double line_wave(const dtmx_tfsf* p, double t) {
  double u = t - p->t0;
  return p->amp * sin(2 * M_PI * p->f0 * u) * exp(-(u / p->tau) * (u / p->tau));
}
static void line_update_h(osim* s) {
  int n = s->line_n; double r = s->cfg.dt / s->cfg.dx;
  double* e = s->line_e; double* h = s->line_h;
  int o4 = s->cfg.order == 4;
  for (int m = 0; m < n; m++) {
    double e0 = e[m], em1 = m >= 1 ? e[m - 1] : 0;
    double d;
    if (o4) { double ep1 = m + 1 < n ? e[m + 1] : 0, em2 = m >= 2 ? e[m - 2] : 0; d = (27 * (e0 - em1) - (ep1 - em2)) / 24; }
    else d = e0 - em1;
    h[m] += r * d;
  }
}
static void line_update_e(osim* s) {
  int n = s->line_n; double r = s->cfg.dt / s->cfg.dx;
  double* e = s->line_e; double* h = s->line_h;
  int o4 = s->cfg.order == 4;
  for (int m = 0; m < n; m++) {
    double h0 = h[m], hp1 = m + 1 < n ? h[m + 1] : 0;
    double d;
    if (o4) { double hp2 = m + 2 < n ? h[m + 2] : 0, hm1 = m >= 1 ? h[m - 1] : 0; d = (27 * (hp1 - h0) - (hp2 - hm1)) / 24; }
    else d = hp1 - h0;
    e[m] += r * d;
  }
}

/* ------------------------------------------------------------- update */

/* derivative of component g along axis a at the node of component c in
 * cell (i,j,k).  H nodes take backward taps (-2..+1), E nodes forward
 * (-1..+2); TF/SF corrections are added to each tap per the reference rule. */
static real deriv(const osim* s, int c, int g, int a, int i, int j, int k, int sfact, double tt) {
  int isH = c >= 3;
  int t0 = isH ? -2 : -1;    /* first tap index offset */
  real v[4];
  int nn[3] = {i, j, k};
  int n[3] = {s->nx, s->ny, s->nz};
  /* fast path: every tap inside the live range of g -> direct reads */
  int fast = 1;
  for (int b = 0; b < 3; b++) {
    int lo = nn[b], hi = nn[b];
    if (b == a) { lo += t0; hi += t0 + 3; }
    if (lo < s->live_lo[g][b] || hi > s->live_hi[g][b]) { fast = 0; break; }
  }
  if (fast && !sfact) {
    long st = a == 0 ? (long)n[1] * n[2] : a == 1 ? n[2] : 1;
    const real* base = s->f[g] + IDX(s, i, j, k) + (long)t0 * st;
    v[0] = base[0]; v[1] = base[st]; v[2] = base[2 * st]; v[3] = base[3 * st];
  } else {
    int X = 2 * i + OFF[c][0], Y = 2 * j + OFF[c][1], Z = 2 * k + OFF[c][2];
    int self_in = sfact ? in_sf(s, X, Y, Z) : 0;
    for (int q = 0; q < 4; q++) {
      int m[3] = {nn[0], nn[1], nn[2]};
      m[a] += t0 + q;
      v[q] = fetch(s, g, m[0], m[1], m[2]);
      if (sfact) {
        int TX = 2 * m[0] + OFF[g][0], TY = 2 * m[1] + OFF[g][1], TZ = 2 * m[2] + OFF[g][2];
        int tin = in_sf(s, TX, TY, TZ);
        if (!self_in && tin) v[q] += (real)inc_value(s, g, TX, TY, TZ, tt);
        else if (self_in && !tin) v[q] -= (real)inc_value(s, g, TX, TY, TZ, tt);
      }
    }
  }
  /* v[0..3] = taps at offsets (t0, t0+1, t0+2, t0+3); centre lies between v[1], v[2] */
  if (s->cfg.order == 2) return v[2] - v[1];
  return ((real)27 * (v[2] - v[1]) - (v[3] - v[0])) / (real)24;
}

static const int CURL[6][2][2] = {
  /* comp: {axis, source comp} for the + term and the - term of curl */
  {{1, DTMX_HZ}, {2, DTMX_HY}},   /* Ex: dy Hz - dz Hy */
  {{2, DTMX_HX}, {0, DTMX_HZ}},   /* Ey: dz Hx - dx Hz */
  {{0, DTMX_HY}, {1, DTMX_HX}},   /* Ez: dx Hy - dy Hx */
  {{1, DTMX_EZ}, {2, DTMX_EY}},   /* Hx: -(dy Ez - dz Ey) */
  {{2, DTMX_EX}, {0, DTMX_EZ}},   /* Hy */
  {{0, DTMX_EY}, {1, DTMX_EX}},   /* Hz */
};

static double src_wave(const dtmx_point_source* p, double t) {
  double u = t - p->t0;
  return p->amp * sin(2 * M_PI * p->f0 * u) * exp(-(u / p->tau) * (u / p->tau));
}

/* node within 4 half cells of the TF/SF box surface (taps reach 3) */
static int near_box(const osim* s, int X, int Y, int Z) {
  int H[3] = {X, Y, Z};
  int close = 0;
  for (int a = 0; a < 3; a++) {
    if (H[a] < s->sf_lo[a] - 4 || H[a] > s->sf_hi[a] + 4) return 0;
    if (H[a] <= s->sf_lo[a] + 4 || H[a] >= s->sf_hi[a] - 4) close = 1;
  }
  return close;
}

/* design-region index of cell (i,j,k), -1 outside */
static long des_index(const osim* s, int i, int j, int k) {
  if (!s->des_on) return -1;
  int v[3] = {i - s->des_lo[0], j - s->des_lo[1], k - s->des_lo[2]};
  for (int a = 0; a < 3; a++) if (v[a] < 0 || v[a] >= s->des_n[a]) return -1;
  return ((long)v[0] * s->des_n[1] + v[1]) * s->des_n[2] + v[2];
}

/* 1/eps of E component c at a non-dispersive node: the design value inside the
 * design region, else the material's */
static real node_ie(const osim* s, int c, int mi, int i, int j, int k) {
  long di = des_index(s, i, j, k);
  return di >= 0 ? s->des_ie[c][di] : s->inv_eps[mi][c];
}

/* ADE-box index of cell (i,j,k), -1 outside the box */
static long ade_index(const osim* s, int i, int j, int k) {
  if (i < s->ade_box[0][0] || i >= s->ade_box[0][1] || j < s->ade_box[1][0] || j >= s->ade_box[1][1] ||
      k < s->ade_box[2][0] || k >= s->ade_box[2][1])
    return -1;
  return ((long)(i - s->ade_box[0][0]) * (s->ade_box[1][1] - s->ade_box[1][0]) + (j - s->ade_box[1][0])) *
             (s->ade_box[2][1] - s->ade_box[2][0]) + (k - s->ade_box[2][0]);
}

static real gyro_old(const osim* s, int c, int i, int j, int k) {
  long ai = ade_index(s, i, j, k);
  return ai < 0 ? 0 : s->Jg[s->gcur][c][ai];
}

/* Magnetised-Drude current J^{n+1/2} from J^{n-1/2} and E^n (dtmx.h,
 * dtmx_material), written to the other buffer; the E half step then
 * subtracts dt/eps_inf J^{n+1/2}. */
static void gyro_pass(osim* s) {
  if (!s->has_gyro || s->ade_n == 0) return;
  const int cur = s->gcur, nxt = 1 - cur;
  #pragma omp parallel for schedule(static)
  for (int i = s->ade_box[0][0]; i < s->ade_box[0][1]; i++)
    for (int j = s->ade_box[1][0]; j < s->ade_box[1][1]; j++)
      for (int k = s->ade_box[2][0]; k < s->ade_box[2][1]; k++) {
        size_t id = IDX(s, i, j, k);
        long ai = ade_index(s, i, j, k);
        for (int c = 0; c < 3; c++) {
          int mi = s->midx[c] ? s->midx[c][id] : 0;
          if (!s->gyro[mi]) continue;
          real E = s->f[c][id], Jo = s->Jg[cur][c][ai], t;
          if (c == 0) {
            real avg = (real)0.25 * (((gyro_old(s, 1, i - 1, j, k) + gyro_old(s, 1, i, j, k)) + gyro_old(s, 1, i - 1, j + 1, k)) +
                                     gyro_old(s, 1, i, j + 1, k));
            t = s->gC[mi] * Jo + s->gS[mi] * avg;
          } else if (c == 1) {
            real avg = (real)0.25 * (((gyro_old(s, 0, i, j - 1, k) + gyro_old(s, 0, i + 1, j - 1, k)) + gyro_old(s, 0, i, j, k)) +
                                     gyro_old(s, 0, i + 1, j, k));
            t = s->gC[mi] * Jo - s->gS[mi] * avg;
          } else {
            t = Jo;
          }
          s->Jg[nxt][c][ai] = s->gA[mi] * t + s->gB[mi] * E;
        }
      }
}

/* E -= dt/eps_inf J^{n+1/2} on gyrotropic nodes; J^{n+1/2} becomes current */
static void gyro_finish(osim* s) {
  if (!s->has_gyro || s->ade_n == 0) return;
  const int nxt = 1 - s->gcur;
  #pragma omp parallel for schedule(static)
  for (int i = s->ade_box[0][0]; i < s->ade_box[0][1]; i++)
    for (int j = s->ade_box[1][0]; j < s->ade_box[1][1]; j++)
      for (int k = s->ade_box[2][0]; k < s->ade_box[2][1]; k++) {
        size_t id = IDX(s, i, j, k);
        long ai = ade_index(s, i, j, k);
        for (int c = 0; c < 3; c++) {
          int mi = s->midx[c] ? s->midx[c][id] : 0;
          if (s->gyro[mi]) s->f[c][id] -= s->gjc[mi] * s->Jg[nxt][c][ai];
        }
      }
  s->gcur = nxt;
}

static void half_step(osim* s, int isH) {
  const dtmx_config* cf = &s->cfg;
  double dd[3] = {cf->dx, cf->dy, cf->dz};
  int64_t n = s->step;
  int sfon = tfsf_active(s, n);
  double tt = isH ? (double)n : (double)n + 0.5;
  int c0 = isH ? 3 : 0;
  /* Every component of this half step reads only the other field type, so
   * components can be updated in place one after another. */
  for (int c = c0; c < c0 + 3; c++) {
    int ilo = s->live_lo[c][0], ihi = s->live_hi[c][0];
    #pragma omp parallel for schedule(static)
    for (int i = ilo; i <= ihi; i++)
      for (int j = s->live_lo[c][1]; j <= s->live_hi[c][1]; j++)
        for (int k = s->live_lo[c][2]; k <= s->live_hi[c][2]; k++) {
          int hc[3] = {2 * i + OFF[c][0], 2 * j + OFF[c][1], 2 * k + OFF[c][2]};
          int sfact = sfon && near_box(s, hc[0], hc[1], hc[2]);
          size_t id = IDX(s, i, j, k);
          /* dif_a = signed (dt/d_a) * D_a(g), with sign + for the first curl term */
          real dif[3] = {0, 0, 0};
          for (int t = 0; t < 2; t++) {
            int a = CURL[c][t][0], g = CURL[c][t][1];
            real dv = deriv(s, c, g, a, i, j, k, sfact, isH ? tt : tt);
            real sg = (t == 0) ? 1 : -1;
            if (isH) sg = -sg;
            dif[a] = sg * (real)(cf->dt / dd[a]) * dv;
          }
          real* F = &s->f[c][id];
          if (!isH) {
            int mi = s->midx[c] ? s->midx[c][id] : 0;
            const dtmx_material* M = &s->mat[mi];
            int in_ade = i >= s->ade_box[0][0] && i < s->ade_box[0][1] && j >= s->ade_box[1][0] &&
                         j < s->ade_box[1][1] && k >= s->ade_box[2][0] && k < s->ade_box[2][1];
            if (M->npoles > 0 && in_ade) {
              /* countDisp (dispersion.cpp:85-99); rotdt = dt*curl H */
              size_t ai = ((size_t)(i - s->ade_box[0][0]) * (s->ade_box[1][1] - s->ade_box[1][0]) +
                           (j - s->ade_box[1][0])) * (s->ade_box[2][1] - s->ade_box[2][0]) + (k - s->ade_box[2][0]);
              real rot = dif[0] + dif[1] + dif[2];
              real Ep = *F, Em = s->Em[c][ai];
              real Etmp = Ep, sum = 0;
              for (int p = 0; p < M->npoles; p++)
                sum += s->kEJ[mi][c][p][0] * s->Jp[c][p][ai] + s->kEJ[mi][c][p][1] * s->Jm[c][p][ai];
              Ep = s->kE[mi][c][0] * Em + s->kE[mi][c][1] * Ep + s->kE[mi][c][2] * rot - sum;
              for (int p = 0; p < M->npoles; p++) {
                real Jt = s->Jp[c][p][ai];
                s->Jp[c][p][ai] = s->kJ[mi][c][p][0] * s->Jp[c][p][ai] + s->kJ[mi][c][p][1] * s->Jm[c][p][ai] +
                                  s->kJ[mi][c][p][2] * Ep + s->kJ[mi][c][p][3] * Em + s->kJ[mi][c][p][4] * Etmp;
                s->Jm[c][p][ai] = Jt;
              }
              s->Em[c][ai] = Etmp;
              *F = Ep;
              continue;
            }
            real ie = node_ie(s, c, mi, i, j, k);
            dif[0] *= ie; dif[1] *= ie; dif[2] *= ie;
          }
          /* absorber */
          int ins[3]; long si[3];
          int any = 0;
          for (int a = 0; a < 3; a++) {
            si[a] = -1; ins[a] = 0;
            if (s->L[a][0] + s->L[a][1] == 0) continue;
            int sl = slot_of(c, a);
            if (sl < 0) continue;
            si[a] = slab_index(s, a, i, j, k);
            if (si[a] >= 0) { ins[a] = 1; any = 1; }
          }
          if (!any || cf->absorber == DTMX_ABS_NONE) { *F += (dif[0] + dif[1] + dif[2]); continue; }
          if (cf->absorber == DTMX_ABS_CPML) {
            real add = 0;
            for (int a = 0; a < 3; a++) {
              if (dif[a] == 0 && slot_of(c, a) < 0) continue;
              if (!ins[a]) { add += dif[a]; continue; }
              real* psi = &s->aux[a][slot_of(c, a)][si[a]];
              int h = hc[a];
              *psi = (real)s->cb[a][h] * *psi + (real)s->ca[a][h] * dif[a];
              add += (real)s->cik[a][h] * dif[a] + *psi;
            }
            *F += add;
          } else {
            /* split field: F = rest + sum of stored parts; each stored part
             * p_a <- K1_a p_a + K2_a dif_a; rest gets the undamped terms */
            real rest = *F, tot = 0;
            for (int a = 0; a < 3; a++) if (ins[a]) rest -= s->aux[a][slot_of(c, a)][si[a]];
            for (int a = 0; a < 3; a++) {
              if (slot_of(c, a) < 0) continue;
              if (ins[a]) {
                real* p = &s->aux[a][slot_of(c, a)][si[a]];
                int h = hc[a];
                *p = s->k1[a][h] * *p + s->k2[a][h] * dif[a];
                tot += *p;
              } else rest += dif[a];
            }
            *F = rest + tot;
          }
        }
  }
  if (!isH) {
    /* soft point sources: E += amp*g(t_{n+1/2}) */
    for (int q = 0; q < s->npsrc; q++) {
      const dtmx_point_source* p = &s->psrc[q];
      s->f[p->comp][IDX(s, p->i, p->j, p->k)] += (real)src_wave(p, ((double)n + 0.5) * cf->dt);
    }
  }
}

/* ------------------------------------------------------------- API */

void* PFX(create)(const dtmx_config* cfg) {
  if (!cfg || cfg->nx < 4 || cfg->ny < 4 || cfg->nz < 4) return NULL;
  if (cfg->order != 2 && cfg->order != 4) return NULL;
  osim* s = calloc(1, sizeof(osim));
  s->cfg = *cfg;
  s->nx = cfg->nx; s->ny = cfg->ny; s->nz = cfg->nz;
  s->ncell = (size_t)s->nx * s->ny * s->nz;
  for (int c = 0; c < 6; c++) s->f[c] = calloc(s->ncell, sizeof(real));
  setup_boundaries(s);
  setup_absorber(s);
  s->nmat = 1;
  s->mat[0].eps[0] = s->mat[0].eps[1] = s->mat[0].eps[2] = 1.0;
  for (int c = 0; c < 3; c++) s->inv_eps[0][c] = 1;
  s->probe_cap = cfg->probe_capacity > 0 ? cfg->probe_capacity : 4096;
  return s;
}

void PFX(destroy)(void* h) {
  osim* s = h;
  if (!s) return;
  for (int c = 0; c < 6; c++) free(s->f[c]);
  for (int a = 0; a < 3; a++) {
    free(s->cb[a]); free(s->ca[a]); free(s->cik[a]); free(s->k1[a]); free(s->k2[a]);
    for (int q = 0; q < 4; q++) free(s->aux[a][q]);
    free(s->midx[a]);
  }
  for (int c = 0; c < 3; c++) {
    free(s->Em[c]);
    for (int p = 0; p < DTMX_MAX_POLES; p++) { free(s->Jp[c][p]); free(s->Jm[c][p]); }
    free(s->Jg[0][c]); free(s->Jg[1][c]); free(s->des_ie[c]);
  }
  free(s->line_e); free(s->line_h); free(s->traces);
  for (int d = 0; d < s->ndft; d++) { free(s->dft[d].omega); free(s->dft[d].acc); }
  free(s);
}

/* DispStruct::set (dispersion.cpp:41-82) for one material */
static void disp_coeffs(osim* s, int mi) {
  const dtmx_material* M = &s->mat[mi];
  double dt = s->cfg.dt;
  int mD = M->npoles;
  double alpha[DTMX_MAX_POLES], ksi[DTMX_MAX_POLES], zetp[DTMX_MAX_POLES], zetm[DTMX_MAX_POLES], zet[DTMX_MAX_POLES];
  double zms = 0, zps = 0, zs = 0;
  for (int i = 0; i < mD; i++) {
    double Deps = M->pole[i][0], wp = M->pole[i][1], gp = M->pole[i][2], gp_ = M->pole[i][3];
    /* LorenzDisp::set / setDrude (dispersion.cpp:5-22) */
    double a0 = Deps * wp * wp, a1 = Deps * gp_, b0 = M->pole_kind[i] == DTMX_POLE_DRUDE ? 0.0 : wp * wp, b1 = 2 * gp;
    alpha[i] = (4 - 2 * b0 * dt * dt) / (b1 * dt + 2);
    ksi[i] = (b1 * dt - 2) / (b1 * dt + 2);
    zetp[i] = (+a0 * dt * dt + 2 * a1 * dt) / (b1 * dt + 2);
    zetm[i] = (-a0 * dt * dt + 2 * a1 * dt) / (b1 * dt + 2);
    zet[i] = -(4 * a1 * dt) / (b1 * dt + 2);
    zms += zetm[i]; zps += zetp[i]; zs += zet[i];
  }
  double einf = M->eps_inf, sg = M->sigma;
  double C1 = (-(zms)) / (2 * einf + sg * dt + zps);
  double C2 = (2 * einf - sg * dt - zs) / (2 * einf + sg * dt + zps);
  double C3 = (2 * dt) / (2 * einf + sg * dt + zps);
  for (int xc = 0; xc < 3; xc++) {
    for (int i = 0; i < mD; i++) {
      s->kJ[mi][xc][i][0] = (real)alpha[i]; s->kJ[mi][xc][i][1] = (real)ksi[i];
      s->kJ[mi][xc][i][2] = (real)(zetp[i] / dt); s->kJ[mi][xc][i][3] = (real)(zetm[i] / dt);
      s->kJ[mi][xc][i][4] = (real)(zet[i] / dt);
      s->kEJ[mi][xc][i][0] = (real)(C3 * 0.5 * (1 + alpha[i])); s->kEJ[mi][xc][i][1] = (real)(C3 * 0.5 * ksi[i]);
    }
    /* kE[2] = C3/dt multiplies rotdt = dt*curl H */
    s->kE[mi][xc][0] = (real)C1; s->kE[mi][xc][1] = (real)C2; s->kE[mi][xc][2] = (real)(C3 / dt);
  }
}

int PFX(set_materials)(void* h, const dtmx_material* table, int nmat, const uint8_t* ix, const uint8_t* iy,
                       const uint8_t* iz) {
  osim* s = h;
  if (nmat < 1 || nmat > DTMX_MAX_MATERIALS || !ix) return DTMX_ERR_INVALID;
  s->nmat = nmat;
  memcpy(s->mat, table, nmat * sizeof(dtmx_material));
  s->has_gyro = 0;
  for (int m = 0; m < nmat; m++) {
    s->gyro[m] = table[m].gyro_wp > 0;
    if (s->gyro[m]) {
      /* magnetised-Drude current (dtmx.h, dtmx_material) */
      if (table[m].npoles > 0 || !(table[m].eps_inf > 0)) return DTMX_ERR_INVALID;
      double dt = s->cfg.dt;
      for (int c = 0; c < 3; c++) s->inv_eps[m][c] = (real)(1.0 / table[m].eps_inf);
      s->gA[m] = (real)exp(-table[m].gyro_gamma * dt);
      s->gC[m] = (real)cos(table[m].gyro_wc * dt);
      s->gS[m] = (real)sin(table[m].gyro_wc * dt);
      s->gB[m] = (real)(table[m].gyro_wp * table[m].gyro_wp * dt);
      s->gjc[m] = (real)(dt / table[m].eps_inf);
      s->has_gyro = 1;
      continue;
    }
    for (int c = 0; c < 3; c++) s->inv_eps[m][c] = (real)(1.0 / table[m].eps[c]);
    if (table[m].npoles > 0) disp_coeffs(s, m);
  }
  const uint8_t* src[3] = {ix, iy ? iy : ix, iz ? iz : ix};
  for (int c = 0; c < 3; c++) {
    free(s->midx[c]);
    s->midx[c] = malloc(s->ncell);
    memcpy(s->midx[c], src[c], s->ncell);
    for (size_t q = 0; q < s->ncell; q++) if (s->midx[c][q] >= nmat) return DTMX_ERR_INVALID;
  }
  /* bounding box of dispersive cells */
  int lo[3] = {s->nx, s->ny, s->nz}, hi[3] = {-1, -1, -1};
  for (int i = 0; i < s->nx; i++)
    for (int j = 0; j < s->ny; j++)
      for (int k = 0; k < s->nz; k++) {
        size_t id = IDX(s, i, j, k);
        int dis = 0;
        for (int c = 0; c < 3; c++) { const dtmx_material* M = &s->mat[s->midx[c][id]]; if (M->npoles > 0 || M->gyro_wp > 0) dis = 1; }
        if (!dis) continue;
        int v[3] = {i, j, k};
        for (int a = 0; a < 3; a++) { if (v[a] < lo[a]) lo[a] = v[a]; if (v[a] > hi[a]) hi[a] = v[a]; }
      }
  for (int c = 0; c < 3; c++) {
    free(s->Em[c]); s->Em[c] = NULL;
    for (int p = 0; p < DTMX_MAX_POLES; p++) { free(s->Jp[c][p]); free(s->Jm[c][p]); s->Jp[c][p] = s->Jm[c][p] = NULL; }
    for (int b = 0; b < 2; b++) { free(s->Jg[b][c]); s->Jg[b][c] = NULL; }
  }
  s->gcur = 0;
  if (hi[0] < 0) { for (int a = 0; a < 3; a++) { s->ade_box[a][0] = 0; s->ade_box[a][1] = 0; } s->ade_n = 0; return DTMX_OK; }
  s->ade_n = 1;
  for (int a = 0; a < 3; a++) { s->ade_box[a][0] = lo[a]; s->ade_box[a][1] = hi[a] + 1; s->ade_n *= (size_t)(hi[a] + 1 - lo[a]); }
  for (int c = 0; c < 3; c++) {
    s->Em[c] = calloc(s->ade_n, sizeof(real));
    for (int p = 0; p < DTMX_MAX_POLES; p++) { s->Jp[c][p] = calloc(s->ade_n, sizeof(real)); s->Jm[c][p] = calloc(s->ade_n, sizeof(real)); }
    if (s->has_gyro) for (int b = 0; b < 2; b++) s->Jg[b][c] = calloc(s->ade_n, sizeof(real));
  }
  return DTMX_OK;
}

int PFX(add_point_source)(void* h, const dtmx_point_source* p) {
  osim* s = h;
  if (s->npsrc >= 64 || p->comp < 0 || p->comp > 2) return DTMX_ERR_INVALID;
  s->psrc[s->npsrc++] = *p;
  return DTMX_OK;
}

int PFX(set_tfsf)(void* h, const dtmx_tfsf* p) {
  osim* s = h;
  /* a slab of a larger grid (dtmx.h, dtmx_tfsf.x_origin / x_cells): box and
   * line in whole-grid coordinates, half-coordinate ranges shifted to this grid */
  int xo = (int)p->x_origin, gnx = p->x_cells > 0 ? (int)p->x_cells : s->nx;
  if ((double)xo != p->x_origin || xo < 0 || xo + s->nx > gnx) return DTMX_ERR_INVALID;
  s->tfsf = *p; s->has_tfsf = 1;
  s->sf_xo = xo;
  double d[3] = {s->cfg.dx, s->cfg.dy, s->cfg.dz};
  for (int a = 0; a < 3; a++)
    sf_range(d[a], p->box_lo[a], p->box_hi[a], a == 0 ? 2 * gnx : half_max(s, a), &s->sf_lo[a], &s->sf_hi[a]);
  s->sf_lo[0] -= 2 * xo; s->sf_hi[0] -= 2 * xo;
  if (p->kind == DTMX_TFSF_PLANE_X) {
    s->line_M = 4096 + xo;
    s->line_n = gnx + 2 * 4096;
    free(s->line_e); free(s->line_h);
    s->line_e = calloc(s->line_n, sizeof(double)); s->line_h = calloc(s->line_n, sizeof(double));
    /* source point 10 cells before the box's lower x face */
    s->line_src = (s->sf_lo[0] + 2 * xo - 1) / 2 - 10 + 4096;
  }
  return DTMX_OK;
}

int PFX(add_probe)(void* h, int comp, int i, int j, int k, int mode) {
  osim* s = h;
  if (s->nprobes >= 4096 || comp < 0 || comp > 5) return -1;
  if (s->traces) return -1;
  probe_t* p = &s->probes[s->nprobes];
  p->comp = comp; p->i = i; p->j = j; p->k = k; p->mode = mode;
  return s->nprobes++;
}

int PFX(add_dft_plane)(void* h, int axis, int index, int comp_mask, int nfreq, const double* om) {
  osim* s = h;
  if (s->ndft >= 64) return -1;
  dft_t* d = &s->dft[s->ndft];
  d->axis = axis; d->index = index; d->comp_mask = comp_mask; d->nfreq = nfreq;
  d->ncomp = 0;
  for (int c = 0; c < 6; c++) if (comp_mask & (1 << c)) d->ncomp++;
  int n[3] = {s->nx, s->ny, s->nz};
  d->n1 = n[axis == 0 ? 1 : 0];
  d->n2 = n[axis == 2 ? 1 : 2];
  d->omega = malloc(nfreq * sizeof(double));
  memcpy(d->omega, om, nfreq * sizeof(double));
  d->acc = calloc((size_t)d->ncomp * nfreq * d->n1 * d->n2 * 2, sizeof(double));
  return s->ndft++;
}

static double probe_value(const osim* s, const probe_t* p) {
  int c = p->comp, x = p->i, y = p->j, z = p->k;
  #define G(cc, a, b, d) ((a) >= 0 && (a) < s->nx && (b) >= 0 && (b) < s->ny && (d) >= 0 && (d) < s->nz ? \
                           (double)s->f[cc][IDX(s, a, b, d)] : 0.0)
  if (p->mode == DTMX_PROBE_NODE) return G(c, x, y, z);
  int zM = (z == 0) ? z + 1 : z - 1;
  switch (c) {
    case DTMX_EX: return 0.25 * (G(c, x, y - 1, zM) + G(c, x, y - 1, z) + G(c, x, y, zM) + G(c, x, y, z));
    case DTMX_EY: return 0.25 * (G(c, x - 1, y, zM) + G(c, x - 1, y, z) + G(c, x, y, zM) + G(c, x, y, z));
    case DTMX_EZ: return 0.25 * (G(c, x - 1, y - 1, z) + G(c, x - 1, y, z) + G(c, x, y - 1, z) + G(c, x, y, z));
    case DTMX_HX: return 0.5 * (G(c, x - 1, y, z) + G(c, x, y, z));
    case DTMX_HY: return 0.5 * (G(c, x, y - 1, z) + G(c, x, y, z));
    /* sensor.h:73: the second Hz point (pcPnt) is never assigned for Hz
     * and reads a node outside the domain, which is zero */
    case DTMX_HZ: return 0.5 * G(c, x, y, zM);
  }
  #undef G
  return 0;
}

static void record(osim* s) {
  int pe = s->cfg.probe_every > 0 ? s->cfg.probe_every : 1;
  if (s->nprobes && (s->step % pe) == 0) {
    if (!s->traces) s->traces = calloc((size_t)s->nprobes * s->probe_cap, sizeof(real));
    if (s->nsamples < s->probe_cap) {
      for (int q = 0; q < s->nprobes; q++)
        s->traces[(size_t)q * s->probe_cap + s->nsamples] = (real)probe_value(s, &s->probes[q]);
      s->nsamples++;
    }
  }
  for (int di = 0; di < s->ndft; di++) {
    dft_t* d = &s->dft[di];
    int cidx = 0;
    for (int c = 0; c < 6; c++) {
      if (!(d->comp_mask & (1 << c))) continue;
      double t = (c < 3) ? (double)s->step * s->cfg.dt : ((double)s->step - 0.5) * s->cfg.dt;
      for (int f = 0; f < d->nfreq; f++) {
        double cr = cos(d->omega[f] * t) * s->cfg.dt, ci = -sin(d->omega[f] * t) * s->cfg.dt;
        double* acc = d->acc + ((size_t)cidx * d->nfreq + f) * d->n1 * d->n2 * 2;
        for (int u = 0; u < d->n1; u++)
          for (int v = 0; v < d->n2; v++) {
            int i, j, k;
            if (d->axis == 0) { i = d->index; j = u; k = v; }
            else if (d->axis == 1) { i = u; j = d->index; k = v; }
            else { i = u; j = v; k = d->index; }
            double val = s->f[c][IDX(s, i, j, k)];
            size_t q = ((size_t)u * d->n2 + v) * 2;
            acc[q] += val * cr; acc[q + 1] += val * ci;
          }
      }
      cidx++;
    }
  }
}

int PFX(step)(void* h, int nsteps) {
  osim* s = h;
  for (int it = 0; it < nsteps; it++) {
    int pw = s->has_tfsf && s->tfsf.kind == DTMX_TFSF_PLANE_X;
    half_step(s, 1);
    if (pw) line_update_h(s);
    gyro_pass(s);
    half_step(s, 0);
    gyro_finish(s);
    if (pw) {
      line_update_e(s);
      s->line_e[s->line_src] += line_wave(&s->tfsf, ((double)s->step + 0.5) * s->cfg.dt);
    }
    s->step++;
    record(s);
  }
  return DTMX_OK;
}

int PFX(get_field)(void* h, int comp, double* out) {
  osim* s = h;
  for (size_t q = 0; q < s->ncell; q++) out[q] = s->f[comp][q];
  return DTMX_OK;
}
int PFX(set_field)(void* h, int comp, const double* in) {
  osim* s = h;
  for (size_t q = 0; q < s->ncell; q++) s->f[comp][q] = (real)in[q];
  return DTMX_OK;
}

/* State of x planes in the library's dtmx_read_planes layout (dtmx.h):
 * section-major -- six fields, the four CPML auxiliaries of the y and z
 * slabs, then Em, Jp[P], Jm[P] of the three E components as dense planes
 * (zero off the ADE box), P the most poles of one material of the table.
 * Used by the tests' out-of-core runs with the oracle as the slab engine. */
static int plane_poles(const osim* s) {
  int p = 0;
  for (int m = 0; m < s->nmat; m++) if (s->mat[m].npoles > p) p = s->mat[m].npoles;
  return p;
}

size_t PFX(plane_state_floats)(void* h) {
  osim* s = h;
  size_t nyz = (size_t)s->ny * s->nz, n = 6 * nyz;
  if (s->aux[1][0]) n += 4 * (size_t)(s->L[1][0] + s->L[1][1]) * s->nz;
  if (s->aux[2][0]) n += 4 * (size_t)s->ny * (s->L[2][0] + s->L[2][1]);
  return n + (size_t)3 * (1 + 2 * plane_poles(s)) * nyz;
}

static int plane_copy(osim* s, int x0, int np, double* buf, int rd) {
  if (x0 < 0 || np < 0 || x0 + np > s->nx) return DTMX_ERR_INVALID;
  if (s->has_gyro || s->des_on || s->cfg.geometry != DTMX_GEOM_BOX) return DTMX_ERR_UNSUPPORTED;
  if (s->aux[0][0] && np > 0 && (x0 < s->L[0][0] || x0 + np > s->nx - s->L[0][1])) return DTMX_ERR_UNSUPPORTED;
  size_t nyz = (size_t)s->ny * s->nz;
  double* b = buf;
  for (int c = 0; c < 6; c++) {
    real* f = s->f[c] + (size_t)x0 * nyz;
    for (size_t q = 0; q < (size_t)np * nyz; q++) { if (rd) b[q] = f[q]; else f[q] = (real)b[q]; }
    b += (size_t)np * nyz;
  }
  for (int a = 1; a < 3; a++) {
    if (!s->aux[a][0]) continue;
    size_t th = (size_t)(s->L[a][0] + s->L[a][1]);
    size_t pp = a == 1 ? th * s->nz : (size_t)s->ny * th;
    for (int q = 0; q < 4; q++) {
      real* f = s->aux[a][q] + (size_t)x0 * pp;
      for (size_t u = 0; u < (size_t)np * pp; u++) { if (rd) b[u] = f[u]; else f[u] = (real)b[u]; }
      b += (size_t)np * pp;
    }
  }
  int P = plane_poles(s);
  for (int c = 0; c < 3; c++)
    for (int sec = 0; sec < 1 + 2 * P; sec++) {
      real* arr = sec == 0 ? s->Em[c] : sec <= P ? s->Jp[c][sec - 1] : s->Jm[c][sec - 1 - P];
      for (int p = 0; p < np; p++)
        for (int j = 0; j < s->ny; j++)
          for (int k = 0; k < s->nz; k++) {
            double* v = b + ((size_t)p * s->ny + j) * s->nz + k;
            long ai = arr ? ade_index(s, x0 + p, j, k) : -1;
            if (rd) *v = ai >= 0 ? arr[ai] : 0.0;
            else if (ai >= 0) arr[ai] = (real)*v;
          }
      b += (size_t)np * nyz;
    }
  return DTMX_OK;
}

int PFX(read_planes)(void* h, int x0, int np, double* out) { return plane_copy(h, x0, np, out, 1); }
int PFX(write_planes)(void* h, int x0, int np, const double* in) { return plane_copy(h, x0, np, (double*)in, 0); }

int PFX(read_probes)(void* h, double* out, int max_samples, int* ns) {
  osim* s = h;
  int n = s->nsamples < max_samples ? s->nsamples : max_samples;
  for (int q = 0; q < s->nprobes; q++)
    for (int t = 0; t < n; t++) out[(size_t)q * max_samples + t] = s->traces ? s->traces[(size_t)q * s->probe_cap + t] : 0;
  *ns = n;
  return DTMX_OK;
}

int PFX(read_dft)(void* h, int id, double* out, size_t len) {
  osim* s = h;
  if (id < 0 || id >= s->ndft) return DTMX_ERR_INVALID;
  dft_t* d = &s->dft[id];
  size_t n = (size_t)d->ncomp * d->nfreq * d->n1 * d->n2 * 2;
  if (len < n) return DTMX_ERR_INVALID;
  memcpy(out, d->acc, n * sizeof(double));
  return DTMX_OK;
}

int PFX(threads)(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}


/* ------------------------------------------------------------------ adjoint
 * Discrete adjoint of the forward step for the gradient of a Poynting-flux
 * objective with respect to per-node permittivity in a design region.
 *
 * Forward step (box geometry, CPML or none, non-dispersive):
 *   H' = H + sum_a g_a d_a + sum_slab b_a psi_a,  psi_a' = b_a psi_a + al_a d_a,
 *   d_a = s_a D_a(E)  (H half step),  then the same for E with d_a = ie s_a D_a(H'),
 * where g_a = 1 outside the axis-a slab and 1/kappa_a + al_a inside, and the
 * staggered difference operators satisfy D_E^T = -D_H (zero outside the box).
 * The adjoint step applies the transposes in reverse order.
 *
 * Dispersive (Drude/Lorentz) E nodes follow countDisp instead (no absorber
 * terms, as in the forward step):
 *   E' = kE0 Em + kE1 E + kE2 rot - sum_q (kEJ0 Jp_q + kEJ1 Jm_q),  rot = sum_a d_a,
 *   Jp_q' = kJ0 Jp_q + kJ1 Jm_q + kJ2 E' + kJ3 Em + kJ4 E,  Jm_q' = Jp_q,  Em' = E;
 * with mu = lam_E' + sum_q kJ2 lam_Jp_q' their adjoint is w_a = s_a kE2 mu and
 *   lam_E = kE1 mu + sum_q kJ4 lam_Jp_q' + lam_Em',  lam_Em = kE0 mu + sum_q kJ3 lam_Jp_q',
 *   lam_Jp_q = -kEJ0 mu + kJ0 lam_Jp_q' + lam_Jm_q',  lam_Jm_q = -kEJ1 mu + kJ1 lam_Jp_q'.
 * The design permittivity does not enter a dispersive node: its gradient is 0.
 * Gyrotropic nodes: the current J' = gA t + gB E (t_x = gC Jx + gS avg4(Jy),
 * t_y = gC Jy - gS avg4(Jx), t_z = Jz, from the old J and E) is subtracted as
 * E' -= gjc J'.  With muJ = lam_J' - gjc lam_E' and lam_t = gA muJ:
 *   lam_E += gB muJ,  lam_J = gC lam_t (own node) -/+ gS/4 lam_t of the nodes
 *   whose average holds it (x and y), lam_Jz = lam_tz;
 * the adjoint of a non-gyrotropic node's current (identically zero) is zero.
 * Objective: J = sum over the plane x = X of Re(Ey^ conj(Hz^) - Ez^ conj(Hy^)),
 * with E^ = sum_s E^s exp(-i w s dt) dt and H^ = sum_s H^{s-1/2} exp(-i w (s-1/2) dt) dt
 * (the engine's DFT convention).  Gradient: dJ/d ie_c(p) =
 * sum_s lamE_c^s(p) (E_c^s(p) - E_c^{s-1}(p)) / ie_c(p), dJ/d eps = -ie^2 dJ/d ie.
 */
int PFX(set_design)(void* h, const int* lo, const int* n, const double* eps) {
  osim* s = h;
  size_t nd = (size_t)n[0] * n[1] * n[2];
  for (int a = 0; a < 3; a++)
    if (n[a] < 1 || lo[a] < 0 || lo[a] + n[a] > (a == 0 ? s->nx : a == 1 ? s->ny : s->nz)) return DTMX_ERR_INVALID;
  for (int c = 0; c < 3; c++) {
    free(s->des_ie[c]);
    s->des_ie[c] = malloc(nd * sizeof(real));
    for (size_t q = 0; q < nd; q++) s->des_ie[c][q] = (real)(1.0 / eps[c * nd + q]);
  }
  for (int a = 0; a < 3; a++) { s->des_lo[a] = lo[a]; s->des_n[a] = n[a]; }
  s->des_on = 1;
  return DTMX_OK;
}

/* slab coefficients of axis a at half-coordinate hc: g (update gain), b, al */
static void slab_coefs(const osim* s, int a, int hc, int inslab, double* g, double* b, double* al) {
  if (!inslab) { *g = 1; *b = 0; *al = 0; return; }
  *b = s->cb[a][hc]; *al = s->ca[a][hc]; *g = s->cik[a][hc] + s->ca[a][hc];
}

static real lget(const osim* s, real* const* arr, int c, int i, int j, int k) {
  if (i < 0 || i >= s->nx || j < 0 || j >= s->ny || k < 0 || k >= s->nz) return 0;
  return arr[c][IDX(s, i, j, k)];
}

/* material of E component c at node (i,j,k) when it is dispersive and in the ADE box, else -1 */
static int ade_mat(const osim* s, int c, int i, int j, int k, long* ai) {
  int mi = s->midx[c] ? s->midx[c][IDX(s, i, j, k)] : 0;
  if (s->mat[mi].npoles <= 0) return -1;
  *ai = ade_index(s, i, j, k);
  return *ai >= 0 ? mi : -1;
}

/* w_{c,a}(p) = s_a ie(p) (g lam(p) + al lampsi(p)) for updated component c at
 * node p (the adjoint of d_a), zero outside the grid; s_a kE2 mu(p) at a
 * dispersive node */
static double adj_w(const osim* s, real* const* lam, real* const lpsi[3][4], int c, int t, int i, int j, int k) {
  if (i < 0 || i >= s->nx || j < 0 || j >= s->ny || k < 0 || k >= s->nz) return 0;
  const dtmx_config* cf = &s->cfg;
  const double dd[3] = {cf->dx, cf->dy, cf->dz};
  int a = CURL[c][t][0];
  int isH = c >= 3;
  double sg = t == 0 ? 1 : -1;
  if (isH) sg = -sg;
  double sa = sg * cf->dt / dd[a];
  size_t id = IDX(s, i, j, k);
  if (!isH && s->ade_n) {
    long ai;
    int mi = ade_mat(s, c, i, j, k, &ai);
    if (mi >= 0) return sa * (double)s->kE[mi][c][2] * (double)s->amu[c][ai];
  }
  double ie = 1;
  if (!isH) ie = node_ie(s, c, s->midx[c] ? s->midx[c][id] : 0, i, j, k);
  int sl = slot_of(c, a);
  long si = (cf->absorber == DTMX_ABS_CPML && s->L[a][0] + s->L[a][1] > 0) ? slab_index(s, a, i, j, k) : -1;
  int nn[3] = {i, j, k};
  double g, b, al;
  slab_coefs(s, a, 2 * nn[a] + OFF[c][a], si >= 0, &g, &b, &al);
  double ld = g * lam[c][id] + (si >= 0 ? al * lpsi[a][sl][si] : 0);
  return sa * ie * ld;
}

/* lam of the source field += D^T of the w of the updated field (one half step) */
static void adj_half(osim* s, real** lam, real* lpsi[3][4], int updH) {
  /* updated components cu (H if updH), sources cs */
  int cu0 = updH ? 3 : 0, cs0 = updH ? 0 : 3;
  int order = s->cfg.order;
  /* taps of the forward derivative of the updated component: offsets t0..t0+3 */
  int t0 = updH ? -2 : -1;
  const double W4[4] = {1.0 / 24, -27.0 / 24, 27.0 / 24, -1.0 / 24}, W2[4] = {0, -1, 1, 0};
  const double* W = order == 4 ? W4 : W2;
  real* add[3];
  for (int c = 0; c < 3; c++) add[c] = calloc(s->ncell, sizeof(real));
  for (int cu = cu0; cu < cu0 + 3; cu++)
    for (int t = 0; t < 2; t++) {
      int a = CURL[cu][t][0], g = CURL[cu][t][1];
      #pragma omp parallel for schedule(static)
      for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
          for (int k = 0; k < s->nz; k++) {
            /* source node q = (i,j,k) of component g receives from updated nodes p = q - (t0+o) e_a */
            double acc = 0;
            for (int o = 0; o < 4; o++) {
              if (W[o] == 0) continue;
              int m[3] = {i, j, k};
              m[a] -= t0 + o;
              acc += W[o] * adj_w(s, lam, lpsi, cu, t, m[0], m[1], m[2]);
            }
            add[g - cs0][IDX(s, i, j, k)] += (real)acc;
          }
    }
  /* slab adjoint recursion of the updated field: lampsi <- b (lam + lampsi) */
  if (s->cfg.absorber == DTMX_ABS_CPML)
    for (int cu = cu0; cu < cu0 + 3; cu++)
      for (int a = 0; a < 3; a++) {
        int sl = slot_of(cu, a);
        if (sl < 0 || s->L[a][0] + s->L[a][1] == 0) continue;
        for (int i = 0; i < s->nx; i++)
          for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
              long si = slab_index(s, a, i, j, k);
              if (si < 0) continue;
              int nn[3] = {i, j, k};
              double g, b, al;
              slab_coefs(s, a, 2 * nn[a] + OFF[cu][a], 1, &g, &b, &al);
              lpsi[a][sl][si] = (real)(b * (lam[cu][IDX(s, i, j, k)] + lpsi[a][sl][si]));
            }
      }
  for (int c = 0; c < 3; c++) {
    for (size_t q = 0; q < s->ncell; q++) lam[cs0 + c][q] += add[c][q];
    free(add[c]);
  }
}

/* mu = lam_E' + sum_q kJ2 lam_Jp_q' on the dispersive nodes */
static void ade_adjoint_mu(osim* s, real* const* lam, real* const lJp[3][DTMX_MAX_POLES]) {
  for (int c = 0; c < 3; c++)
    for (int i = s->ade_box[0][0]; i < s->ade_box[0][1]; i++)
      for (int j = s->ade_box[1][0]; j < s->ade_box[1][1]; j++)
        for (int k = s->ade_box[2][0]; k < s->ade_box[2][1]; k++) {
          long ai;
          int mi = ade_mat(s, c, i, j, k, &ai);
          if (mi < 0) continue;
          double mu = lam[c][IDX(s, i, j, k)];
          for (int q = 0; q < s->mat[mi].npoles; q++) mu += (double)s->kJ[mi][c][q][2] * lJp[c][q][ai];
          s->amu[c][ai] = (real)mu;
        }
}

/* lam_E and the adjoint ADE state of the dispersive nodes (after the E-update transposition) */
static void ade_adjoint_state(const osim* s, real** lam, real** lEm, real* lJp[3][DTMX_MAX_POLES],
                              real* lJm[3][DTMX_MAX_POLES]) {
  for (int c = 0; c < 3; c++)
    for (int i = s->ade_box[0][0]; i < s->ade_box[0][1]; i++)
      for (int j = s->ade_box[1][0]; j < s->ade_box[1][1]; j++)
        for (int k = s->ade_box[2][0]; k < s->ade_box[2][1]; k++) {
          long ai;
          int mi = ade_mat(s, c, i, j, k, &ai);
          if (mi < 0) continue;
          const double mu = s->amu[c][ai];
          double nE = (double)s->kE[mi][c][1] * mu + lEm[c][ai];
          double nEm = (double)s->kE[mi][c][0] * mu;
          for (int q = 0; q < s->mat[mi].npoles; q++) {
            const double lp = lJp[c][q][ai], lm = lJm[c][q][ai];
            nE += (double)s->kJ[mi][c][q][4] * lp;
            nEm += (double)s->kJ[mi][c][q][3] * lp;
            lJp[c][q][ai] = (real)(-(double)s->kEJ[mi][c][q][0] * mu + (double)s->kJ[mi][c][q][0] * lp + lm);
            lJm[c][q][ai] = (real)(-(double)s->kEJ[mi][c][q][1] * mu + (double)s->kJ[mi][c][q][1] * lp);
          }
          lam[c][IDX(s, i, j, k)] = (real)nE;
          lEm[c][ai] = (real)nEm;
        }
}

/* muJ = lam_J' - gjc lam_E' on the gyrotropic nodes (0 elsewhere); uses lam_E' */
static void gyro_adjoint_t(const osim* s, real* const* lam, real* const* lJg, real** lT) {
  for (int i = s->ade_box[0][0]; i < s->ade_box[0][1]; i++)
    for (int j = s->ade_box[1][0]; j < s->ade_box[1][1]; j++)
      for (int k = s->ade_box[2][0]; k < s->ade_box[2][1]; k++) {
        size_t id = IDX(s, i, j, k);
        long ai = ade_index(s, i, j, k);
        for (int c = 0; c < 3; c++) {
          int mi = s->midx[c] ? s->midx[c][id] : 0;
          lT[c][ai] = s->gyro[mi] ? (real)((double)lJg[c][ai] - (double)s->gjc[mi] * lam[c][id]) : 0;
        }
      }
}

static real adj_t_at(const osim* s, real* const* lT, int c, int i, int j, int k) {
  long ai = ade_index(s, i, j, k);
  return ai < 0 ? 0 : lT[c][ai];
}

/* lam_E += gB muJ and lam_J of the old current from lam_t = gA muJ (gathered
 * over the nodes whose 4-node average holds each current) */
static void gyro_adjoint_state(const osim* s, real** lam, real** lJg, real* const* lT) {
  for (int i = s->ade_box[0][0]; i < s->ade_box[0][1]; i++)
    for (int j = s->ade_box[1][0]; j < s->ade_box[1][1]; j++)
      for (int k = s->ade_box[2][0]; k < s->ade_box[2][1]; k++) {
        size_t id = IDX(s, i, j, k);
        long ai = ade_index(s, i, j, k);
        for (int c = 0; c < 3; c++) {
          int mi = s->midx[c] ? s->midx[c][id] : 0;
          if (!s->gyro[mi]) { lJg[c][ai] = 0; continue; }
          const double mu = lT[c][ai], t = (double)s->gA[mi] * mu;
          lam[c][id] += (real)((double)s->gB[mi] * mu);
          double v;
          if (c == 0) {
            /* Jx(i,j) enters the averages of the y nodes (i,j+1), (i-1,j+1), (i,j), (i-1,j) */
            int nb[4][2] = {{i, j + 1}, {i - 1, j + 1}, {i, j}, {i - 1, j}};
            double acc = 0;
            for (int q = 0; q < 4; q++) {
              int ii = nb[q][0], jj = nb[q][1];
              if (ii < 0 || ii >= s->nx || jj < 0 || jj >= s->ny) continue;
              int mq = s->midx[1] ? s->midx[1][IDX(s, ii, jj, k)] : 0;
              if (s->gyro[mq]) acc += 0.25 * (double)s->gS[mq] * (double)s->gA[mq] * adj_t_at(s, lT, 1, ii, jj, k);
            }
            v = (double)s->gC[mi] * t - acc;
          } else if (c == 1) {
            /* Jy(i,j) enters the averages of the x nodes (i+1,j), (i,j), (i+1,j-1), (i,j-1) */
            int nb[4][2] = {{i + 1, j}, {i, j}, {i + 1, j - 1}, {i, j - 1}};
            double acc = 0;
            for (int q = 0; q < 4; q++) {
              int ii = nb[q][0], jj = nb[q][1];
              if (ii < 0 || ii >= s->nx || jj < 0 || jj >= s->ny) continue;
              int mq = s->midx[0] ? s->midx[0][IDX(s, ii, jj, k)] : 0;
              if (s->gyro[mq]) acc += 0.25 * (double)s->gS[mq] * (double)s->gA[mq] * adj_t_at(s, lT, 0, ii, jj, k);
            }
            v = (double)s->gC[mi] * t + acc;
          } else {
            v = t;
          }
          lJg[c][ai] = (real)v;
        }
      }
}

int PFX(forward_adjoint)(void* h, int nsteps, int X, double omega, double* J_out, double* grad_out) {
  osim* s = h;
  if (!s->des_on || X < 0 || X >= s->nx || nsteps < 1) return DTMX_ERR_INVALID;
  if (s->cfg.geometry != DTMX_GEOM_BOX || s->cfg.absorber == DTMX_ABS_SPLIT_PML) return DTMX_ERR_UNSUPPORTED;
  /* the design permittivity of a gyrotropic node would enter next to its current: not carried */
  for (int c = 0; c < 3 && s->has_gyro; c++)
    for (int i = 0; i < s->des_n[0]; i++)
      for (int j = 0; j < s->des_n[1]; j++)
        for (int k = 0; k < s->des_n[2]; k++) {
          size_t id = IDX(s, s->des_lo[0] + i, s->des_lo[1] + j, s->des_lo[2] + k);
          if (s->gyro[s->midx[c] ? s->midx[c][id] : 0]) return DTMX_ERR_UNSUPPORTED;
        }
  const double dt = s->cfg.dt;
  const size_t nd = (size_t)s->des_n[0] * s->des_n[1] * s->des_n[2];
  const size_t npl = (size_t)s->ny * s->nz;
  /* forward: design-region E history and the flux DFT */
  real* hist = malloc((size_t)(nsteps + 1) * 3 * nd * sizeof(real));
  double* F = calloc(4 * npl * 2, sizeof(double));   /* Ey, Ez, Hy, Hz (re, im) */
  int64_t s0 = s->step;
  for (int st = 0; st <= nsteps; st++) {
    if (st > 0) PFX(step)(h, 1);
    for (int c = 0; c < 3; c++)
      for (int i = 0; i < s->des_n[0]; i++)
        for (int j = 0; j < s->des_n[1]; j++)
          for (int k = 0; k < s->des_n[2]; k++)
            hist[((size_t)st * 3 + c) * nd + ((size_t)i * s->des_n[1] + j) * s->des_n[2] + k] =
                s->f[c][IDX(s, s->des_lo[0] + i, s->des_lo[1] + j, s->des_lo[2] + k)];
    if (st == 0) continue;
    double sE = (double)(s->step), sH = sE - 0.5;
    double pe[2] = {cos(omega * sE * dt) * dt, -sin(omega * sE * dt) * dt};
    double ph[2] = {cos(omega * sH * dt) * dt, -sin(omega * sH * dt) * dt};
    const int comp[4] = {DTMX_EY, DTMX_EZ, DTMX_HY, DTMX_HZ};
    for (int q = 0; q < 4; q++)
      for (size_t u = 0; u < npl; u++) {
        double v = s->f[comp[q]][(size_t)X * npl + u];
        const double* pp = q < 2 ? pe : ph;
        F[(q * npl + u) * 2] += v * pp[0];
        F[(q * npl + u) * 2 + 1] += v * pp[1];
      }
  }
  /* J = sum Re(Ey conj(Hz)) - Re(Ez conj(Hy)) */
  double J = 0;
  for (size_t u = 0; u < npl; u++) {
    const double *ey = F + (0 * npl + u) * 2, *ez = F + (1 * npl + u) * 2, *hy = F + (2 * npl + u) * 2, *hz = F + (3 * npl + u) * 2;
    J += ey[0] * hz[0] + ey[1] * hz[1] - (ez[0] * hy[0] + ez[1] * hy[1]);
  }
  *J_out = J;
  /* backward */
  real* lam[6];
  for (int c = 0; c < 6; c++) lam[c] = calloc(s->ncell, sizeof(real));
  real* lpsi[3][4];
  for (int a = 0; a < 3; a++) {
    size_t th = (size_t)(s->L[a][0] + s->L[a][1]);
    size_t ns = th * (a == 0 ? npl : a == 1 ? (size_t)s->nx * s->nz : (size_t)s->nx * s->ny);
    for (int q = 0; q < 4; q++) lpsi[a][q] = calloc(ns ? ns : 1, sizeof(real));
  }
  double* grad = calloc(3 * nd, sizeof(double));
  /* adjoint of the ADE state over the ADE box */
  real *lEm[3] = {0}, *lJp[3][DTMX_MAX_POLES] = {{0}}, *lJm[3][DTMX_MAX_POLES] = {{0}};
  for (int c = 0; c < 3 && s->ade_n; c++) {
    lEm[c] = calloc(s->ade_n, sizeof(real));
    s->amu[c] = calloc(s->ade_n, sizeof(real));
    for (int q = 0; q < DTMX_MAX_POLES; q++) { lJp[c][q] = calloc(s->ade_n, sizeof(real)); lJm[c][q] = calloc(s->ade_n, sizeof(real)); }
  }
  real *lJg[3] = {0}, *lT[3] = {0};
  for (int c = 0; c < 3 && s->has_gyro && s->ade_n; c++) { lJg[c] = calloc(s->ade_n, sizeof(real)); lT[c] = calloc(s->ade_n, sizeof(real)); }
  for (int st = nsteps; st >= 1; st--) {
    double sE = (double)(s0 + st), sH = sE - 0.5;
    double pe[2] = {cos(omega * sE * dt) * dt, -sin(omega * sE * dt) * dt};
    double ph[2] = {cos(omega * sH * dt) * dt, -sin(omega * sH * dt) * dt};
    /* objective sources at x^st = (E^st, H^{st-1/2}) */
    for (size_t u = 0; u < npl; u++) {
      const double *ey = F + (0 * npl + u) * 2, *ez = F + (1 * npl + u) * 2, *hy = F + (2 * npl + u) * 2, *hz = F + (3 * npl + u) * 2;
      size_t id = (size_t)X * npl + u;
      lam[DTMX_EY][id] += (real)(pe[0] * hz[0] + pe[1] * hz[1]);
      lam[DTMX_EZ][id] -= (real)(pe[0] * hy[0] + pe[1] * hy[1]);
      lam[DTMX_HZ][id] += (real)(ey[0] * ph[0] + ey[1] * ph[1]);
      lam[DTMX_HY][id] -= (real)(ez[0] * ph[0] + ez[1] * ph[1]);
    }
    /* gradient with respect to ie of the E update of step st */
    for (int c = 0; c < 3; c++)
      for (int i = 0; i < s->des_n[0]; i++)
        for (int j = 0; j < s->des_n[1]; j++)
          for (int k = 0; k < s->des_n[2]; k++) {
            size_t di = ((size_t)i * s->des_n[1] + j) * s->des_n[2] + k;
            size_t id = IDX(s, s->des_lo[0] + i, s->des_lo[1] + j, s->des_lo[2] + k);
            long ai;
            if (s->ade_n && ade_mat(s, c, s->des_lo[0] + i, s->des_lo[1] + j, s->des_lo[2] + k, &ai) >= 0) continue;
            double dE = (double)hist[((size_t)st * 3 + c) * nd + di] - (double)hist[((size_t)(st - 1) * 3 + c) * nd + di];
            grad[c * nd + di] += (double)lam[c][id] * dE / (double)s->des_ie[c][di];
          }
    /* lam^{st-1} = A^T lam^{st}: E update transposed, then H update transposed */
    if (s->ade_n) ade_adjoint_mu(s, lam, lJp);
    if (lJg[0]) gyro_adjoint_t(s, lam, lJg, lT);
    adj_half(s, lam, lpsi, 0);
    if (s->ade_n) ade_adjoint_state(s, lam, lEm, lJp, lJm);
    if (lJg[0]) gyro_adjoint_state(s, lam, lJg, lT);
    adj_half(s, lam, lpsi, 1);
  }
  for (int c = 0; c < 3; c++) { free(lJg[c]); free(lT[c]); }
  for (int c = 0; c < 3 && s->ade_n; c++) {
    free(lEm[c]); free(s->amu[c]); s->amu[c] = NULL;
    for (int q = 0; q < DTMX_MAX_POLES; q++) { free(lJp[c][q]); free(lJm[c][q]); }
  }
  for (int c = 0; c < 3; c++)
    for (size_t q = 0; q < nd; q++) {
      double ie = s->des_ie[c][q];
      grad_out[c * nd + q] = -ie * ie * grad[c * nd + q];
    }
  for (int c = 0; c < 6; c++) free(lam[c]);
  for (int a = 0; a < 3; a++) for (int q = 0; q < 4; q++) free(lpsi[a][q]);
  free(grad); free(hist); free(F);
  return DTMX_OK;
}
