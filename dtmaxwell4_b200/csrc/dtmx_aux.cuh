// dtmx_aux.cuh -- per-step side kernels: TF/SF surface corrections, the 1-D
// incident line of the plane-wave source, soft point sources, probes, running
// DFT and the device step counter.
#pragma once
#include "dtmx_device.cuh"

namespace dtmx {

// One TF/SF correction job: component c over an index box that holds every
// node of c whose taps along one curl axis cross one face of the box.
struct TfsfJob {
  int c;
  int lo[3], hi[3];
  long long cells;
};
constexpr int MAX_TFSF_JOBS = 12;    // 3 components x 2 curl terms x 2 faces

struct TfsfDev {
  int active_cfg;            // a TF/SF source is configured
  int kind;                  // 0 dipole, 1 plane +x
  int lo[3], hi[3];          // inside-box half-coordinate ranges (inclusive)
  double ctr[3];             // dipole position (box centre, physical, whole-grid coordinates)
  int xo;                    // whole-grid cell index of plane 0 (x slabs; 0 for a whole grid)
  double hd[3];              // half cell sizes dx/2, dy/2, dz/2
  double dt, c, w, kenv, tstop;
  int ntime;
  const double* line_e; const double* line_h; int line_M, line_n;
  int njob[2];               // [0] E half step, [1] H half step
  TfsfJob job[2][MAX_TFSF_JOBS];
};

__device__ __forceinline__ bool tfsf_on(const TfsfDev& t, long long n) {
  if (t.tstop <= 0) return true;
  const long long is = n / t.ntime;
  return (double)(is + 1) * t.ntime * t.dt < t.tstop;
}

__device__ __forceinline__ bool in_box(const TfsfDev& t, int X, int Y, int Z) {
  return X >= t.lo[0] && X <= t.hi[0] && Y >= t.lo[1] && Y <= t.hi[1] && Z >= t.lo[2] && Z <= t.hi[2];
}

// Field of a z-oriented Hertzian dipole with a Hann-windowed sine moment,
// reference DipoleTFSF (signal.hpp:51-97), evaluated in double precision.
__device__ double dipole_field(const TfsfDev& t, int comp, int X, int Y, int Z, double tt) {
  const double nx = (X + 2 * t.xo) * t.hd[0] - t.ctr[0], ny = Y * t.hd[1] - t.ctr[1], nz = Z * t.hd[2] - t.ctr[2];
  const double R = sqrt(nx * nx + ny * ny + nz * nz);
  const double time = tt * t.dt, c = t.c, w = t.w, ke = t.kenv;
  const double ph = w * time - w / c * R;
  double s, co, sk, ck;
  sincos(ph, &s, &co);
  sincos(ph * ke, &sk, &ck);
  double d = s * 0.5 * (1.0 - ck);
  double ds = w * co * 0.5 - 0.5 * w * co * ck + 0.5 * s * w * ke * sk;
  double dss = -w * w * s * 0.5 + 0.5 * w * w * s * ck + w * co * w * ke * sk + 0.5 * s * w * ke * w * ke * ck;
  if (ph * ke < 0.0 || ph * ke > 2.0 * M_PI) { d = 0; ds = 0; dss = 0; }
  const double u0 = nx / R, u1 = ny / R, u2 = nz / R;
  if (comp < 3) {
    // (dss z^ x n) x n  +  3 (ds.n) n - ds  +  3 (d.n) n - d   with moments along z
    const double a0 = -dss * u1, a1 = dss * u0;
    const double cr[3] = {a1 * u2, -a0 * u2, a0 * u1 - a1 * u0};
    const double uu[3] = {u0, u1, u2};
    const double dz = comp == 2 ? 1.0 : 0.0;
    return c * (cr[comp] / (c * c * R) + (3.0 * ds * u2 * uu[comp] - ds * dz) / (c * R * R) +
                (3.0 * d * u2 * uu[comp] - d * dz) / (R * R * R));
  }
  const int q = comp - 3;
  const double b1 = q == 0 ? -dss * u1 : q == 1 ? dss * u0 : 0.0;
  const double b2 = q == 0 ? -ds * u1 : q == 1 ? ds * u0 : 0.0;
  return b1 / (c * c * R) + b2 / (c * R * R);
}

__device__ __forceinline__ double incident(const TfsfDev& t, int g, int X, int Y, int Z, double tt) {
  if (t.kind == 0) return dipole_field(t, g, X, Y, Z, tt);
  if (g == 2) { const int m = ((X - 1) >> 1) + t.line_M; return (m >= 0 && m < t.line_n) ? t.line_e[m] : 0.0; }
  if (g == 4) { const int m = (X >> 1) + t.line_M; return (m >= 0 && m < t.line_n) ? t.line_h[m] : 0.0; }
  return 0.0;
}

// curl terms of component c: {axis, source component} for (+) and (-) terms
__host__ __device__ __forceinline__ void curl_terms(int c, int& a0, int& g0, int& a1, int& g1) {
  switch (c) {
    case 0: a0 = 1; g0 = 5; a1 = 2; g1 = 4; break;
    case 1: a0 = 2; g0 = 3; a1 = 0; g1 = 5; break;
    case 2: a0 = 0; g0 = 4; a1 = 1; g1 = 3; break;
    case 3: a0 = 1; g0 = 2; a1 = 2; g1 = 1; break;
    case 4: a0 = 2; g0 = 0; a1 = 0; g1 = 2; break;
    default: a0 = 0; g0 = 1; a1 = 1; g1 = 0; break;
  }
}

// TF/SF correction of one half step (genAlg.py:209-234): a tap that crosses
// the box surface gets +inc when the updated node is outside and the tap
// inside, -inc in the opposite case.  The update is linear in the taps, so
// the correction is added after the bulk update as dt/d * D(corrections),
// summed over both curl terms of the node in double precision.
template <int ORDER>
__device__ __forceinline__ bool tfsf_node(const Params& p, const TfsfDev& t, int c, int i, int j, int k, bool isH,
                                          double tt, double& total) {
  const int t0 = isH ? -2 : -1;
  const int idx[3] = {i, j, k};
  const int Xs[3] = {2 * i + comp_off(c, 0), 2 * j + comp_off(c, 1), 2 * k + comp_off(c, 2)};
  int ax[2], gs[2];
  curl_terms(c, ax[0], gs[0], ax[1], gs[1]);
  total = 0.0;
  bool any = false;
  bool self_known = false, self_in = false;
  for (int term = 0; term < 2; term++) {
    const int a = ax[term], g = gs[term];
    // the plane wave has only Ez and Hy incident components
    if (t.kind == 1 && g != 2 && g != 4) continue;
    // a tap along a crosses the surface only if the node lies inside the box
    // range on the other two axes and within 3 half cells of a face along a
    const int b1 = (a + 1) % 3, b2 = (a + 2) % 3;
    const int gb1 = 2 * idx[b1] + comp_off(g, b1), gb2 = 2 * idx[b2] + comp_off(g, b2);
    if (gb1 < t.lo[b1] || gb1 > t.hi[b1] || gb2 < t.lo[b2] || gb2 > t.hi[b2]) continue;
    const int Xa = Xs[a];
    if (!((Xa >= t.lo[a] - 4 && Xa <= t.lo[a] + 3) || (Xa >= t.hi[a] - 3 && Xa <= t.hi[a] + 4))) continue;
    if (!self_known) { self_in = in_box(t, Xs[0], Xs[1], Xs[2]); self_known = true; }
    double v[4];
    bool hit = false;
    for (int q = 0; q < 4; q++) {
      v[q] = 0.0;
      if (ORDER == 2 && (q == 0 || q == 3)) continue;
      int m[3] = {idx[0], idx[1], idx[2]};
      m[a] += t0 + q;
      const int TX = 2 * m[0] + comp_off(g, 0), TY_ = 2 * m[1] + comp_off(g, 1), TZ_ = 2 * m[2] + comp_off(g, 2);
      const bool tin = in_box(t, TX, TY_, TZ_);
      if (tin != self_in) {
        const double inc = incident(t, g, TX, TY_, TZ_, tt);
        v[q] = self_in ? -inc : inc;
        hit = true;
      }
    }
    if (!hit) continue;
    any = true;
    double sg = term == 0 ? 1.0 : -1.0;
    if (isH) sg = -sg;
    const double dv = ORDER == 2 ? v[2] - v[1] : (27.0 * (v[2] - v[1]) - (v[3] - v[0])) / 24.0;
    total += sg * (double)p.cdt[a] * dv;
  }
  return any;
}

__device__ __forceinline__ bool in_job(const TfsfJob& jb, int i, int j, int k) {
  return i >= jb.lo[0] && i <= jb.hi[0] && j >= jb.lo[1] && j <= jb.hi[1] && k >= jb.lo[2] && k <= jb.hi[2];
}

// One thread per node of a job (blockIdx.y); a node that also lies in an
// earlier job of the same component is left to that job, so every node is
// corrected exactly once with the sum of all its crossing taps.
template <int ORDER>
__global__ void tfsf_kernel(Params p, TfsfDev t, const long long* d_step, int isH) {
  const long long n = *d_step;
  if (!tfsf_on(t, n)) return;
  const int hs = isH ? 1 : 0;
  const int r = blockIdx.y;
  if (r >= t.njob[hs]) return;
  const TfsfJob& jb = t.job[hs][r];
  // a job is a thin shell (cells < 2^31, checked when the jobs are built): 32-bit indexing
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= (int)jb.cells) return;
  const int ey = jb.hi[1] - jb.lo[1] + 1, ez = jb.hi[2] - jb.lo[2] + 1;
  const int i = jb.lo[0] + cell / (ey * ez);
  const int rest = cell - (i - jb.lo[0]) * (ey * ez);
  const int j = jb.lo[1] + rest / ez;
  const int k = jb.lo[2] + (rest - (j - jb.lo[1]) * ez);
  const int c = jb.c;
  if (!is_live(p.g, c, i, j, k)) return;
  for (int q = 0; q < r; q++)
    if (t.job[hs][q].c == c && in_job(t.job[hs][q], i, j, k)) return;
  const double tt = isH ? (double)n : (double)n + 0.5;
  double total;
  if (!tfsf_node<ORDER>(p, t, c, i, j, k, isH, tt, total)) return;
  const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
  if (!isH) {
    const int mi = p.mat[c] ? (int)p.mat[c][id] : 0;
    const long long di = design_index(p, i, j, k);
    total *= (double)(di >= 0 ? p.des_ie[c][di] : p.mt->inv_eps[mi][c]);
  }
  p.f[c][id] += (float)total;
}

// 1-D incident line (Ez at odd X, Hy at even X), same stencil and time step.
template <int ORDER>
__global__ void line_h_kernel(double* e, double* h, int n, double r) {
  for (int m = threadIdx.x + blockIdx.x * blockDim.x; m < n; m += blockDim.x * gridDim.x) {
    const double e0 = e[m], em1 = m >= 1 ? e[m - 1] : 0.0;
    double d;
    if (ORDER == 4) {
      const double ep1 = m + 1 < n ? e[m + 1] : 0.0, em2 = m >= 2 ? e[m - 2] : 0.0;
      d = (27.0 * (e0 - em1) - (ep1 - em2)) / 24.0;
    } else {
      d = e0 - em1;
    }
    h[m] += r * d;
  }
}
template <int ORDER>
__global__ void line_e_kernel(double* e, const double* h, int n, double r, int src, const long long* d_step,
                              double dt, double amp, double f0, double tau, double t0) {
  const double ts = ((double)(*d_step) + 0.5) * dt - t0;
  for (int m = threadIdx.x + blockIdx.x * blockDim.x; m < n; m += blockDim.x * gridDim.x) {
    const double h0 = h[m], hp1 = m + 1 < n ? h[m + 1] : 0.0;
    double d;
    if (ORDER == 4) {
      const double hp2 = m + 2 < n ? h[m + 2] : 0.0, hm1 = m >= 1 ? h[m - 1] : 0.0;
      d = (27.0 * (hp1 - h0) - (hp2 - hm1)) / 24.0;
    } else {
      d = hp1 - h0;
    }
    double v = e[m] + r * d;
    if (m == src) v += amp * sin(2.0 * M_PI * f0 * ts) * exp(-(ts / tau) * (ts / tau));
    e[m] = v;
  }
}

struct PointSrcDev {
  int comp; long long id; double amp, f0, tau, t0;
};

__global__ void point_source_kernel(Params p, const PointSrcDev* s, int ns, const long long* d_step, double dt) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ns) return;
  const double u = ((double)(*d_step) + 0.5) * dt - s[q].t0;
  const double v = s[q].amp * sin(2.0 * M_PI * s[q].f0 * u) * exp(-(u / s[q].tau) * (u / s[q].tau));
  p.f[s[q].comp][s[q].id] += (float)v;
}

struct ProbeDev { int comp, i, j, k, mode; };

__device__ __forceinline__ float probe_get(const Params& p, int c, int i, int j, int k) {
  if (i < 0 || i >= p.g.n[0] || j < 0 || j >= p.g.n[1] || k < 0 || k >= p.g.n[2]) return 0.f;
  return p.f[c][(long long)i * p.g.sx + (long long)j * p.g.sy + k];
}

// Reference Sensor::write averaging (sensor.h:51-83); for Hz the reference's
// second point is never assigned and reads a zero node outside the domain.
__global__ void probe_kernel(Params p, const ProbeDev* pr, int np, float* traces, int cap, const long long* d_step,
                             int every) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const long long s = *d_step + 1;
  if (q >= np || (s % every) != 0) return;
  const long long sample = s / every - 1;
  if (sample >= cap) return;
  const ProbeDev d = pr[q];
  const int c = d.comp, x = d.i, y = d.j, z = d.k;
  float v;
  if (d.mode == 0) {
    v = probe_get(p, c, x, y, z);
  } else {
    const int zM = z == 0 ? z + 1 : z - 1;
    switch (c) {
      case 0: v = 0.25f * (probe_get(p, c, x, y - 1, zM) + probe_get(p, c, x, y - 1, z) + probe_get(p, c, x, y, zM) + probe_get(p, c, x, y, z)); break;
      case 1: v = 0.25f * (probe_get(p, c, x - 1, y, zM) + probe_get(p, c, x - 1, y, z) + probe_get(p, c, x, y, zM) + probe_get(p, c, x, y, z)); break;
      case 2: v = 0.25f * (probe_get(p, c, x - 1, y - 1, z) + probe_get(p, c, x - 1, y, z) + probe_get(p, c, x, y - 1, z) + probe_get(p, c, x, y, z)); break;
      case 3: v = 0.5f * (probe_get(p, c, x - 1, y, z) + probe_get(p, c, x, y, z)); break;
      case 4: v = 0.5f * (probe_get(p, c, x, y - 1, z) + probe_get(p, c, x, y, z)); break;
      default: v = 0.5f * probe_get(p, c, x, y, zM); break;
    }
  }
  traces[(long long)q * cap + sample] = v;
}

struct DftDev {
  int axis, index, comp_mask, nfreq, n1, n2;
  int lo1, lo2;             // window origin along the two in-plane axes (slow, fast)
  const double* omega;
  double2* acc;             // [ncomp][nfreq][n1*n2]
  float* stage;             // [DFT_STAGE][ncomp][n1*n2] plane samples not yet accumulated
  long long* sstep;         // [DFT_STAGE] step number s of each staged sample
};
constexpr int DFT_STAGE = 16;

// Running DFT with FP64 accumulators: acc += f(t) exp(-i w t) dt, t = s*dt for E,
// (s-1/2)*dt for H, s = steps completed.  Every step stages the plane's values
// (dft_capture_kernel); every DFT_STAGE steps dft_flush_kernel folds the staged
// samples into the accumulators in step order, so the accumulator update
// sequence (and its rounding) is that of a per-step update while the
// accumulators are read and written once per DFT_STAGE steps.
__global__ void dft_capture_kernel(Params p, DftDev d, const long long* d_step, int slot) {
  const long long npts = (long long)d.n1 * d.n2;
  const long long pt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (pt == 0) d.sstep[slot] = *d_step + 1;
  if (pt >= npts) return;
  const int u = d.lo1 + (int)(pt / d.n2), v = d.lo2 + (int)(pt % d.n2);
  int i, j, k;
  if (d.axis == 0) { i = d.index; j = u; k = v; }
  else if (d.axis == 1) { i = u; j = d.index; k = v; }
  else { i = u; j = v; k = d.index; }
  const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
  int ci = 0;
  const int ncomp = __popc(d.comp_mask);
  for (int c = 0; c < 6; c++) {
    if (!(d.comp_mask & (1 << c))) continue;
    d.stage[((long long)slot * ncomp + ci) * npts + pt] = p.f[c][id];
    ci++;
  }
}

__global__ void __launch_bounds__(256) dft_flush_kernel(DftDev d, int nslots, double dt) {
  __shared__ double2 phE[DFT_STAGE][64], phH[DFT_STAGE][64];
  for (int q = threadIdx.x; q < nslots * d.nfreq; q += blockDim.x) {
    const int sl = q / d.nfreq, f = q - sl * d.nfreq;
    const long long s = d.sstep[sl];
    double sn, cs;
    sincos(d.omega[f] * (double)s * dt, &sn, &cs);
    phE[sl][f] = make_double2(cs * dt, -sn * dt);
    sincos(d.omega[f] * ((double)s - 0.5) * dt, &sn, &cs);
    phH[sl][f] = make_double2(cs * dt, -sn * dt);
  }
  __syncthreads();
  const long long npts = (long long)d.n1 * d.n2;
  const long long pt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (pt >= npts) return;
  const int ncomp = __popc(d.comp_mask);
  int ci = 0;
  for (int c = 0; c < 6; c++) {
    if (!(d.comp_mask & (1 << c))) continue;
    double val[DFT_STAGE];
#pragma unroll
    for (int sl = 0; sl < DFT_STAGE; sl++)
      val[sl] = sl < nslots ? (double)d.stage[((long long)sl * ncomp + ci) * npts + pt] : 0.0;
    const double2(*ph)[64] = c < 3 ? phE : phH;
    double2* acc = d.acc + (long long)ci * d.nfreq * npts + pt;
    for (int f = 0; f < d.nfreq; f++) {
      double2 a = acc[(long long)f * npts];
#pragma unroll
      for (int sl = 0; sl < DFT_STAGE; sl++) {
        if (sl < nslots) {
          a.x += val[sl] * ph[sl][f].x;
          a.y += val[sl] * ph[sl][f].y;
        }
      }
      acc[(long long)f * npts] = a;
    }
    ci++;
  }
}

// Outward Poynting flux of one face of a flux box at every frequency of its
// DFT patch: out[f] = sgn_area * sum_pts Re(E_b conj(H_c) - E_c conj(H_b)) with
// (a, b, c) = (normal, (a+1)%3, (a+2)%3), so that (b, c, a) is right-handed.
// One block per frequency; every thread sums a fixed stride of points and a
// fixed tree combines the threads, so the value does not depend on timing.
constexpr int FLUX_THREADS = 256;
__device__ __forceinline__ int dft_slot(int mask, int comp) { return __popc(mask & ((1 << comp) - 1)); }
__global__ void __launch_bounds__(FLUX_THREADS) flux_face_kernel(DftDev d, double sgn_area, double* out) {
  __shared__ double red[FLUX_THREADS];
  const int f = blockIdx.x;
  const int a = d.axis, b = (a + 1) % 3, c = (a + 2) % 3;
  const long long npts = (long long)d.n1 * d.n2;
  const double2* Eb = d.acc + ((long long)dft_slot(d.comp_mask, b) * d.nfreq + f) * npts;
  const double2* Ec = d.acc + ((long long)dft_slot(d.comp_mask, c) * d.nfreq + f) * npts;
  const double2* Hb = d.acc + ((long long)dft_slot(d.comp_mask, 3 + b) * d.nfreq + f) * npts;
  const double2* Hc = d.acc + ((long long)dft_slot(d.comp_mask, 3 + c) * d.nfreq + f) * npts;
  double s = 0.0;
  for (long long pt = threadIdx.x; pt < npts; pt += FLUX_THREADS) {
    const double2 eb = Eb[pt], ec = Ec[pt], hb = Hb[pt], hc = Hc[pt];
    s += (eb.x * hc.x + eb.y * hc.y) - (ec.x * hb.x + ec.y * hb.y);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = FLUX_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[f] = sgn_area * red[0];
}

// Near-to-far-field transform of a flux box (surface equivalence): on a face
// with outward normal n = sgn e_a the equivalent currents are J = n x H and
// M = -n x E, i.e. J_c = sgn H_b, J_b = -sgn H_c, M_c = -sgn E_b, M_b = sgn E_c
// ((a, b, c) cyclic), and the radiation vectors are
//   N = sum J(r') exp(i k rhat.r') dA,  L = sum M(r') exp(i k rhat.r') dA,
// k = omega (c = 1).  Both currents must lie on one closed surface: the
// tangential E of the face plane w sits at w + 1/2 along the normal and the
// tangential H at w, so H is averaged over the planes w and w + 1 onto the E
// surface, the box [lo + 1/2, hi + 1/2] on every axis.  In the plane every term
// keeps its component's Yee position, and the sum over a face is a quadrature
// over that box's face: along an in-plane axis, a component at integer
// positions takes the midpoints lo+1 .. hi (weight 1), one at half-integer
// positions the points lo+1/2 .. hi+1/2 with the trapezoid weights (1/2 at the
// ends); the windows hold the indices lo .. hi.  The
// DFT phasors follow x(t) = Re(X exp(i w t)), so an outgoing wave carries
// exp(-i k r) and the far field is
//   r E_theta = -i k/(4 pi) (L_phi + N_theta) e^{-ikr},  r E_phi = i k/(4 pi) (L_theta - N_phi) e^{-ikr},
// with radiation intensity U = k^2/(16 pi^2) (|L_phi + N_theta|^2 + |L_theta - N_phi|^2),
// normalised like the flux box (Re(E x H*) without the 1/2), so that the
// integral of U over the sphere equals the box's power.  One block per
// (direction, frequency); FP64 throughout, fixed-order reduction.
struct NtffFaces {
  DftDev f[6];              // tangential E and H of the face planes, windows [lo, hi] in the plane
  DftDev h[6];              // tangential H of the planes one further along each normal
  double org[3];            // the origin of r' (physical units)
  double ds[3];
  int lo[3], hi[3];         // the box (face plane indices)
};
// quadrature weight of in-plane index v for a component at v + o/2, box [lo + 1/2, hi + 1/2]
__host__ __device__ __forceinline__ double ntff_weight(int v, int o, int lo, int hi) {
  if (o == 0) return (v > lo && v <= hi) ? 1.0 : 0.0;
  if (v == lo || v == hi) return 0.5;
  return (v > lo && v < hi) ? 1.0 : 0.0;
}
__global__ void __launch_bounds__(FLUX_THREADS) ntff_kernel(NtffFaces F, const double* theta, const double* phi,
                                                            int nfreq, double* out) {
  __shared__ double red[12][FLUX_THREADS];
  const int dir = blockIdx.x, f = blockIdx.y;
  const double th = theta[dir], ph = phi[dir];
  double sth, cth, sph, cph;
  sincos(th, &sth, &cth);
  sincos(ph, &sph, &cph);
  const double rh[3] = {sth * cph, sth * sph, cth};
  double acc[12];
#pragma unroll
  for (int q = 0; q < 12; q++) acc[q] = 0.0;
  for (int q = 0; q < 6; q++) {
    const DftDev& d = F.f[q];
    const int a = d.axis, b = (a + 1) % 3, c = (a + 2) % 3;
    const double sgn = (q & 1) ? 1.0 : -1.0;
    const int s1 = a == 0 ? 1 : 0, s2 = a == 2 ? 1 : 2;
    const double k = d.omega[f];
    const double dA = F.ds[s1] * F.ds[s2];
    const long long npts = (long long)d.n1 * d.n2;
    const double2* Eb = d.acc + ((long long)dft_slot(d.comp_mask, b) * d.nfreq + f) * npts;
    const double2* Ec = d.acc + ((long long)dft_slot(d.comp_mask, c) * d.nfreq + f) * npts;
    const double2* Hb = d.acc + ((long long)dft_slot(d.comp_mask, 3 + b) * d.nfreq + f) * npts;
    const double2* Hc = d.acc + ((long long)dft_slot(d.comp_mask, 3 + c) * d.nfreq + f) * npts;
    const DftDev& d2 = F.h[q];
    const double2* Hb2 = d2.acc + ((long long)dft_slot(d2.comp_mask, 3 + b) * d2.nfreq + f) * npts;
    const double2* Hc2 = d2.acc + ((long long)dft_slot(d2.comp_mask, 3 + c) * d2.nfreq + f) * npts;
    const int srcs[4] = {3 + b, 3 + c, b, c};       // terms J_c, J_b, M_c, M_b
    for (long long pt = threadIdx.x; pt < npts; pt += FLUX_THREADS) {
      int idx[3];
      idx[a] = d.index;
      idx[s1] = d.lo1 + (int)(pt / d.n2);
      idx[s2] = d.lo2 + (int)(pt % d.n2);
      const double2 hb = Hb[pt], hb2 = Hb2[pt], hc = Hc[pt], hc2 = Hc2[pt];
      const double2 vals[4] = {make_double2(0.5 * (hb.x + hb2.x), 0.5 * (hb.y + hb2.y)),
                               make_double2(0.5 * (hc.x + hc2.x), 0.5 * (hc.y + hc2.y)), Eb[pt], Ec[pt]};
      const double wts[4] = {sgn, -sgn, -sgn, sgn};
      const int dst[4] = {c, b, c, b};
#pragma unroll
      for (int t = 0; t < 4; t++) {
        double proj = 0.0;
#pragma unroll
        for (int x = 0; x < 3; x++) {
          // along the normal every term sits on the E surface w + 1/2
          const double off = x == a ? 0.5 : 0.5 * comp_off(srcs[t], x);
          proj += rh[x] * ((idx[x] + off) * F.ds[x] - F.org[x]);
        }
        const double qw = ntff_weight(idx[s1], comp_off(srcs[t], s1), F.lo[s1], F.hi[s1]) *
                          ntff_weight(idx[s2], comp_off(srcs[t], s2), F.lo[s2], F.hi[s2]);
        if (qw == 0.0) continue;
        double sn, cs;
        sincos(k * proj, &sn, &cs);
        const double re = wts[t] * qw * dA * (vals[t].x * cs - vals[t].y * sn);
        const double im = wts[t] * qw * dA * (vals[t].x * sn + vals[t].y * cs);
        const int base = (t < 2 ? 0 : 6) + 2 * dst[t];
        acc[base] += re;
        acc[base + 1] += im;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 12; q++) red[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int w = FLUX_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int q = 0; q < 12; q++) red[q][threadIdx.x] += red[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    // N = red[0..5] (x, y, z complex), L = red[6..11]; theta/phi components
    const double tv[3] = {cth * cph, cth * sph, -sth}, pv[3] = {-sph, cph, 0.0};
    double Nt[2] = {0, 0}, Np[2] = {0, 0}, Lt[2] = {0, 0}, Lp[2] = {0, 0};
    for (int x = 0; x < 3; x++)
      for (int r = 0; r < 2; r++) {
        Nt[r] += tv[x] * red[2 * x + r][0];
        Np[r] += pv[x] * red[2 * x + r][0];
        Lt[r] += tv[x] * red[6 + 2 * x + r][0];
        Lp[r] += pv[x] * red[6 + 2 * x + r][0];
      }
    const double k = F.f[0].omega[f];
    const double s = k / (4.0 * M_PI);
    // r E_theta = -i s (Lp + Nt), r E_phi = i s (Lt - Np) (the e^{-ikr} dropped)
    const double at[2] = {Lp[0] + Nt[0], Lp[1] + Nt[1]}, ap[2] = {Lt[0] - Np[0], Lt[1] - Np[1]};
    double* o = out + ((long long)dir * nfreq + f) * 5;
    o[0] = s * s * (at[0] * at[0] + at[1] * at[1] + ap[0] * ap[0] + ap[1] * ap[1]);
    o[1] = s * at[1];
    o[2] = -s * at[0];
    o[3] = -s * ap[1];
    o[4] = s * ap[0];
  }
}

// Magnetised-Drude current over the ADE box (dtmx.h, dtmx_material):
// J^{n+1/2} into buffer 1-cur from J^{n-1/2} (buffer cur) and E^n.
__device__ __forceinline__ float gyro_old(const Params& p, int cur, int c, int i, int j, int k) {
  const int bi = i - p.ade.lo[0], bj = j - p.ade.lo[1], bk = k - p.ade.lo[2];
  if (bi < 0 || bi >= p.ade.n[0] || bj < 0 || bj >= p.ade.n[1] || bk < 0 || bk >= p.ade.n[2]) return 0.f;
  return __ldg(p.ade.Jg[cur][c] + ((long long)bi * p.ade.n[1] + bj) * p.ade.n[2] + bk);
}

// Thread layout of the passes over the ADE box: (threadIdx.x, blockIdx.x) = z,
// (threadIdx.y, blockIdx.y) = y, blockIdx.z = x (no index division).
__device__ __forceinline__ bool ade_cell(const Params& p, int& bi, int& bj, int& bk, long long& q) {
  bk = blockIdx.x * blockDim.x + threadIdx.x;
  bj = blockIdx.y * blockDim.y + threadIdx.y;
  bi = blockIdx.z;
  if (bj >= p.ade.n[1] || bk >= p.ade.n[2]) return false;
  q = ((long long)bi * p.ade.n[1] + bj) * p.ade.n[2] + bk;
  return true;
}

__global__ void gyro_current_kernel(Params p, int cur) {
  const MatTable& mt = *p.mt;
  int bi, bj, bk;
  long long q;
  if (ade_cell(p, bi, bj, bk, q)) {
    const int i = p.ade.lo[0] + bi, j = p.ade.lo[1] + bj, k = p.ade.lo[2] + bk;
    const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      // (E, the old current, materials and table are read-only in this pass)
      const int m = p.mat[c] ? (int)__ldg(p.mat[c] + id) : 0;
      if (__ldg(&mt.gjc[m]) == 0.f) continue;
      const float E = __ldg(p.f[c] + id), Jo = __ldg(p.ade.Jg[cur][c] + q);
      float t;
      if (c == 0) {
        const float avg = __fmul_rn(0.25f, __fadd_rn(__fadd_rn(__fadd_rn(gyro_old(p, cur, 1, i - 1, j, k), gyro_old(p, cur, 1, i, j, k)),
                                                               gyro_old(p, cur, 1, i - 1, j + 1, k)),
                                                     gyro_old(p, cur, 1, i, j + 1, k)));
        t = __fmaf_rn(__ldg(&mt.gC[m]), Jo, __fmul_rn(__ldg(&mt.gS[m]), avg));
      } else if (c == 1) {
        const float avg = __fmul_rn(0.25f, __fadd_rn(__fadd_rn(__fadd_rn(gyro_old(p, cur, 0, i, j - 1, k), gyro_old(p, cur, 0, i + 1, j - 1, k)),
                                                               gyro_old(p, cur, 0, i, j, k)),
                                                     gyro_old(p, cur, 0, i + 1, j, k)));
        t = __fmaf_rn(__ldg(&mt.gC[m]), Jo, -__fmul_rn(__ldg(&mt.gS[m]), avg));
      } else {
        t = Jo;
      }
      p.ade.Jg[1 - cur][c][q] = __fmaf_rn(__ldg(&mt.gA[m]), t, __fmul_rn(__ldg(&mt.gB[m]), E));
    }
  }
}

// Dispersive and gyrotropic E nodes, after e_kernel (which leaves dispersive
// nodes untouched): the ADE recursion (countDisp, dispersion.cpp:85-99) with
// rot = dt curl H recomputed from H exactly as the field kernels compute it,
// and E -= dt/eps_inf J^{n+1/2} on gyrotropic nodes.  One thread per cell of
// the ADE box; BOX: zero-outside geometry (bounds-checked taps).
template <int ORDER, bool BOX>
__global__ void ade_node_kernel(Params p) {
  const MatTable& mt = *p.mt;
  int bi, bj, bk;
  long long q;
  if (ade_cell(p, bi, bj, bk, q)) {
    const int i = p.ade.lo[0] + bi, j = p.ade.lo[1] + bj, k = p.ade.lo[2] + bk;
    const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
    const int idx[3] = {i, j, k};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (!is_live(p.g, c, i, j, k)) continue;
      // (materials, table, H and the new current are read-only in this pass)
      const int m = p.mat[c] ? (int)__ldg(p.mat[c] + id) : 0;
      const int np = __ldg(&mt.npoles[m]);
      if (np > 0) {
        float d[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int t = 0; t < 2; t++) {
          const int a = (c + 1 + t) % 3;             // curl axis of term t
          const int g = 3 + (c + 2 - t) % 3;         // source H component of term t
          float v[4];
#pragma unroll
          for (int o = 0; o < 4; o++) {
            v[o] = 0.f;
            if (ORDER == 2 && (o == 0 || o == 3)) continue;
            int m3[3] = {i, j, k};
            m3[a] += o - 1;                          // E taps at -1..+2
            if (BOX) {
              const long long sa = a == 0 ? p.g.sx : a == 1 ? p.g.sy : 1;
              v[o] = (m3[a] >= 0 && m3[a] < p.g.n[a]) ? __ldg(p.f[g] + id + (long long)(o - 1) * sa) : 0.f;
            } else {
              v[o] = fetch<1>(p, g, m3[0], m3[1], m3[2]);
            }
          }
          d[a] = __fmul_rn(t == 0 ? p.cdt[a] : -p.cdt[a], dstencil<ORDER>(v[0], v[1], v[2], v[3]));
        }
        (void)idx;
        const float E0 = p.fe_old[c] ? __ldg(p.fe_old[c] + id) : p.f[c][id];
        p.f[c][id] = ade_update(p, c, m, np, q, sum3(d[0], d[1], d[2]), E0);
      } else if (__ldg(&mt.gjc[m]) != 0.f) {
        p.f[c][id] = __fsub_rn(p.f[c][id], __fmul_rn(__ldg(&mt.gjc[m]), __ldg(p.ade.Jg[p.ade.gnew][c] + q)));
      }
    }
  }
}

__global__ void mask_nonlive_kernel(Params p, int comp, long long ncell) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q % p.g.n[2]);
    const long long r = q / p.g.n[2];
    const int j = (int)(r % p.g.n[1]);
    const int i = (int)(r / p.g.n[1]);
    if (!is_live(p.g, comp, i, j, k)) p.f[comp][(long long)i * p.g.sx + (long long)j * p.g.sy + k] = 0.f;
  }
}

__global__ void advance_step_kernel(long long* d_step) { *d_step += 1; }

__global__ void nonfinite_kernel(Params p, int comp, long long ncell, int* flag) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q % p.g.n[2]);
    const long long r = q / p.g.n[2];
    const int j = (int)(r % p.g.n[1]);
    const int i = (int)(r / p.g.n[1]);
    const float v = p.f[comp][(long long)i * p.g.sx + (long long)j * p.g.sy + k];
    if (!isfinite(v)) { atomicExch(flag, 1); return; }
  }
}

}  // namespace dtmx
