// dtmx_adjoint.cuh -- discrete adjoint of the field update for gradients with
// respect to per-node permittivity (no reference counterpart: the reference
// has no differentiation path).
//
// Forward step (box geometry, CPML or no absorber):
//   H' = H + sum_a g_a d_a + sum_slab b_a psi_a,   psi_a' = b_a psi_a + al_a d_a,
//   d_a = s_a D_a(E) for H, d_a = ie s_a D_a(H') for E,
// with g_a = 1 outside the axis-a slab and 1/kappa_a + al_a inside.  The
// adjoint step applies the transposes in reverse order: the E update (lam_H
// += D^T w_E, then lam_psiE <- b (lam_E + lam_psiE)), then the H update
// (lam_E += D^T w_H, lam_psiH <- b (lam_H + lam_psiH)), where w = s ie (g lam
// + al lam_psi) is the adjoint of d.  D^T is gathered tap by tap with the
// forward stencil weights; outside the grid every value is zero, as in the
// forward box geometry.  Dispersive (Drude/Lorentz) E nodes follow the ADE
// recursion instead (adj_ade_kernel: its transpose replaces their w and
// carries the adjoint of the ADE state).  Each kernel is a plain per-node
// gather: the adjoint is run on the recomputed segments of a checkpointed
// forward run.
#pragma once
#include "dtmx_device.cuh"

namespace dtmx {

struct AdjDev {
  float* lam[6];            // adjoint of E (0-2) and H (3-5), field layout
  float* lpsi[3][4];        // adjoint of the CPML auxiliaries, slab layout
  double* grad;             // [3][nd] dJ/d(1/eps) accumulated in double precision
  const float* hist;        // [K+1][3][nd] design-region E of the recomputed segment
  int nd;
  float* w[3][2];           // adjoint of the scaled derivative terms d of the updated field, field layout
  float* lEm[3];            // adjoint of the ADE state (Em, Jp, Jm) over the ADE box
  float* lJp[3][MAXPOLE];
  float* lJm[3][MAXPOLE];
  float* lJg[3];            // adjoint of the gyrotropic current, ADE box
  float* lT[3];             // muJ of the gyrotropic nodes during one adjoint step, ADE box
};

// curl table: updated component -> {axis, source component} of its + and - terms
__host__ __device__ __forceinline__ constexpr int curl_axis(int c, int t) {
  // Ex: y,z  Ey: z,x  Ez: x,y  (same pattern for H)
  return ((c % 3) + 1 + t) % 3;
}
__host__ __device__ __forceinline__ constexpr int curl_src(int c, int t) {
  // Ex: Hz,Hy  Ey: Hx,Hz  Ez: Hy,Hx ; Hx: Ez,Ey  Hy: Ex,Ez  Hz: Ey,Ex
  return (c < 3 ? 3 : 0) + ((c % 3) + 2 - t) % 3;
}
__device__ __forceinline__ void curl_pair(int c, int t, int& a, int& g) {
  a = curl_axis(c, t);
  g = curl_src(c, t);
}

// w of the updated field at every node (3 components x 2 curl terms):
//   w_{c,t} = sg_t cdt_a ie_c (g_a lam_c + al_a lam_psi)   (a = curl axis of term t;
//   g_a lam + al lam_psi only inside the axis-a slab, lam elsewhere),
// then the slab recursion lam_psi <- b (lam + lam_psi) (w uses the old lam_psi).
// One thread per ADJ_XP nodes along x: their lam, materials and 1/eps are
// requested together before any is used (measured on the differentiation
// workload: 2 nodes 3 % faster than 1, 4 nodes 1 %, 8 nodes 8 % slower).
// Thread layout: (threadIdx.x, blockIdx.x) = z,
// (threadIdx.y, blockIdx.y) = y, blockIdx.z = x planes [ADJ_XP z, ADJ_XP (z + 1)).
constexpr int ADJ_XP = 2;
template <int ORDER, int UPDH>
__global__ void adj_w_kernel(Params p, AdjDev A) {
  constexpr bool updH = UPDH != 0;
  const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i0 = blockIdx.z * ADJ_XP;
  if (j >= p.g.n[1] || k >= p.g.n[2]) return;
  constexpr int cu0 = updH ? 3 : 0;
  const bool cpml = p.ab.kind == 1;
  float lam[ADJ_XP][3], ie[ADJ_XP][3];
#pragma unroll
  for (int q = 0; q < ADJ_XP; q++) {
    const int i = i0 + q;
#pragma unroll
    for (int c = 0; c < 3; c++) { lam[q][c] = 0.f; ie[q][c] = 1.f; }
    if (i >= p.g.n[0]) continue;
    const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
    const long long di = updH ? -1 : design_index(p, i, j, k);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int cu = cu0 + c;
      if (!updH) {
        // (material, design and table values are constant during the adjoint: read-only path)
        const int m = p.mat[cu] ? (int)__ldg(p.mat[cu] + id) : 0;
        ie[q][c] = di >= 0 ? __ldg(p.des_ie[cu] + di) : __ldg(&p.mt->inv_eps[m][cu]);
      }
      lam[q][c] = A.lam[cu][id];
    }
  }
#pragma unroll
  for (int q = 0; q < ADJ_XP; q++) {
    const int i = i0 + q;
    if (i >= p.g.n[0]) break;
    const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
    const int idx[3] = {i, j, k};
    int si[3] = {-1, -1, -1};
    if (cpml) node_slabs(p, i, j, k, si);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int cu = cu0 + c;
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const int a = curl_axis(cu, t);
        float sg = t == 0 ? 1.f : -1.f;
        if (updH) sg = -sg;
        float ld = lam[q][c];
        if (si[a] >= 0) {
          const int h = 2 * idx[a] + comp_off(cu, a);
          const float al = __ldg(p.ab.c1[a] + h), gk = __fadd_rn(__ldg(p.ab.c2[a] + h), al);
          ld = __fmaf_rn(gk, ld, __fmul_rn(al, A.lpsi[a][slot_of(cu, a)][si[a]]));
        }
        A.w[c][t][id] = __fmul_rn(__fmul_rn(sg * p.cdt[a], ie[q][c]), ld);
      }
    }
    if (!cpml) continue;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (si[a] < 0) continue;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const int cu = cu0 + c, sl = slot_of(cu, a);
        if (sl < 0) continue;
        const float b = __ldg(p.ab.c0[a] + 2 * idx[a] + comp_off(cu, a));
        A.lpsi[a][sl][si[a]] = __fmul_rn(b, __fadd_rn(lam[q][c], A.lpsi[a][sl][si[a]]));
      }
    }
  }
}

// lam of the source field += D^T w, gathered tap by tap with the forward
// stencil weights (zero outside the grid); same thread layout as adj_w_kernel.
template <int ORDER, int UPDH>
__global__ void adj_curl_kernel(Params p, AdjDev A) {
  constexpr int updH = UPDH;
  const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, i = blockIdx.z;
  if (j >= p.g.n[1] || k >= p.g.n[2]) return;
  const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
  constexpr int t0 = updH ? -2 : -1;
  constexpr int cu0 = updH ? 3 : 0, cs0 = updH ? 0 : 3;
  const int idx[3] = {i, j, k};
  const long long st[3] = {p.g.sx, p.g.sy, 1};
#pragma unroll
  for (int gs = 0; gs < 3; gs++) {
    float acc = 0.f;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int t = 0; t < 2; t++) {
        int a, g;
        curl_pair(cu0 + c, t, a, g);
        if (g != cs0 + gs) continue;
        const float* w = A.w[c][t];
#pragma unroll
        for (int o = 0; o < 4; o++) {
          const float wgt = ORDER == 4 ? (o == 0 ? 1.f / 24.f : o == 1 ? -27.f / 24.f : o == 2 ? 27.f / 24.f : -1.f / 24.f)
                                       : (o == 1 ? -1.f : o == 2 ? 1.f : 0.f);
          if (ORDER == 2 && (o == 0 || o == 3)) continue;
          const int v = idx[a] - (t0 + o);
          if (v < 0 || v >= p.g.n[a]) continue;
          acc = __fmaf_rn(wgt, w[id - (long long)(t0 + o) * st[a]], acc);
        }
      }
    A.lam[cs0 + gs][id] = __fadd_rn(A.lam[cs0 + gs][id], acc);
  }
}

// Objective sources of step s on the plane x = X: F holds the final DFTs
// (Ey, Ez, Hy, Hz; re, im) of J = sum Re(Ey conj(Hz) - Ez conj(Hy)).
__global__ void adj_source_kernel(Params p, AdjDev A, const double* F, long long s, int X, double omega, double dt) {
  const int npl = p.g.n[1] * p.g.n[2];
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= npl) return;
  const double sE = (double)s, sH = sE - 0.5;
  double se, ce, sh, ch;
  sincos(omega * sE * dt, &se, &ce);
  sincos(omega * sH * dt, &sh, &ch);
  const double per = ce * dt, pei = -se * dt, phr = ch * dt, phi = -sh * dt;
  const double* ey = F + (0 * (long long)npl + u) * 2;
  const double* ez = F + (1 * (long long)npl + u) * 2;
  const double* hy = F + (2 * (long long)npl + u) * 2;
  const double* hz = F + (3 * (long long)npl + u) * 2;
  const int j = u / p.g.n[2], k = u % p.g.n[2];
  const long long id = (long long)X * p.g.sx + (long long)j * p.g.sy + k;
  A.lam[1][id] += (float)(per * hz[0] + pei * hz[1]);
  A.lam[2][id] -= (float)(per * hy[0] + pei * hy[1]);
  A.lam[5][id] += (float)(ey[0] * phr + ey[1] * phi);
  A.lam[4][id] -= (float)(ez[0] * phr + ez[1] * phi);
}

// Transposed ADE recursion on the dispersive E nodes, between adj_w_kernel<.,0>
// and adj_curl_kernel<.,0>.  The forward update of such a node (ade_update,
// countDisp of dispersion.cpp:85-99, no absorber terms) is linear:
//   E' = kE0 Em + kE1 E + kE2 rot - sum_q (kEJ0 Jp_q + kEJ1 Jm_q),  rot = sum_a d_a,
//   Jp_q' = kJ0 Jp_q + kJ1 Jm_q + kJ2 E' + kJ3 Em + kJ4 E,   Jm_q' = Jp_q,   Em' = E.
// With mu = lam_E' + sum_q kJ2 lam_Jp_q' (the adjoint of the intermediate E'):
//   w_{c,t} = s_t cdt_a kE2 mu   (replaces the w adj_w_kernel wrote for the node),
//   lam_E  = kE1 mu + sum_q kJ4 lam_Jp_q' + lam_Em',   lam_Em = kE0 mu + sum_q kJ3 lam_Jp_q',
//   lam_Jp_q = -kEJ0 mu + kJ0 lam_Jp_q' + lam_Jm_q',   lam_Jm_q = -kEJ1 mu + kJ1 lam_Jp_q'.
// One thread per cell of the ADE box (the ade_node_kernel layout).
__global__ void adj_ade_kernel(Params p, AdjDev A) {
  const MatTable& mt = *p.mt;
  int bi, bj, bk;
  long long q;
  if (!ade_cell(p, bi, bj, bk, q)) return;
  const int i = p.ade.lo[0] + bi, j = p.ade.lo[1] + bj, k = p.ade.lo[2] + bk;
  const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int m = p.mat[c] ? (int)__ldg(p.mat[c] + id) : 0;
    const int np = __ldg(&mt.npoles[m]);
    if (np <= 0) continue;
    float mu = A.lam[c][id];
    for (int r = 0; r < np; r++) mu = __fmaf_rn(__ldg(&mt.kJ[m][c][r][2]), A.lJp[c][r][q], mu);
    const float wk = __fmul_rn(__ldg(&mt.kE[m][c][2]), mu);
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const int a = curl_axis(c, t);
      A.w[c][t][id] = __fmul_rn(t == 0 ? p.cdt[a] : -p.cdt[a], wk);
    }
    float nE = __fmaf_rn(__ldg(&mt.kE[m][c][1]), mu, A.lEm[c][q]);
    float nEm = __fmul_rn(__ldg(&mt.kE[m][c][0]), mu);
    for (int r = 0; r < np; r++) {
      const float lp = A.lJp[c][r][q], lm = A.lJm[c][r][q];
      nE = __fmaf_rn(__ldg(&mt.kJ[m][c][r][4]), lp, nE);
      nEm = __fmaf_rn(__ldg(&mt.kJ[m][c][r][3]), lp, nEm);
      A.lJp[c][r][q] = __fmaf_rn(__ldg(&mt.kJ[m][c][r][0]), lp, __fmaf_rn(-__ldg(&mt.kEJ[m][c][r][0]), mu, lm));
      A.lJm[c][r][q] = __fmaf_rn(__ldg(&mt.kJ[m][c][r][1]), lp, -__fmul_rn(__ldg(&mt.kEJ[m][c][r][1]), mu));
    }
    A.lam[c][id] = nE;
    A.lEm[c][q] = nEm;
  }
}

// Transposed magnetised-Drude current (gyro_current_kernel, then E -= gjc J'):
//   J' = gA t + gB E,  t_x = gC Jx + gS avg4(Jy),  t_y = gC Jy - gS avg4(Jx),  t_z = Jz.
// adj_gyro_mu_kernel (after adj_w_kernel<.,0>, which reads lam_E'): muJ =
// lam_J' - gjc lam_E' on the gyrotropic nodes (0 elsewhere) into lT, and
// lam_E += gB muJ.  adj_gyro_j_kernel: the adjoint of the old current,
// lam_J = gC gA muJ (own node) -/+ gS/4 gA muJ of the nodes whose 4-node average
// holds it; a non-gyrotropic node's current is identically zero, so is its adjoint.
__global__ void adj_gyro_mu_kernel(Params p, AdjDev A) {
  const MatTable& mt = *p.mt;
  int bi, bj, bk;
  long long q;
  if (!ade_cell(p, bi, bj, bk, q)) return;
  const int i = p.ade.lo[0] + bi, j = p.ade.lo[1] + bj, k = p.ade.lo[2] + bk;
  const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int m = p.mat[c] ? (int)__ldg(p.mat[c] + id) : 0;
    const float gjc = __ldg(&mt.gjc[m]);
    if (gjc == 0.f) { A.lT[c][q] = 0.f; continue; }
    const float lE = A.lam[c][id];
    const float mu = __fmaf_rn(-gjc, lE, A.lJg[c][q]);
    A.lT[c][q] = mu;
    A.lam[c][id] = __fmaf_rn(__ldg(&mt.gB[m]), mu, lE);
  }
}

// gA gS / 4 muJ of component c at node (i, j, k) when it is gyrotropic (0 outside the box or grid)
__device__ __forceinline__ float adj_gyro_term(const Params& p, const AdjDev& A, int c, int i, int j, int k) {
  const int bi = i - p.ade.lo[0], bj = j - p.ade.lo[1], bk = k - p.ade.lo[2];
  if (bi < 0 || bi >= p.ade.n[0] || bj < 0 || bj >= p.ade.n[1] || bk < 0 || bk >= p.ade.n[2]) return 0.f;
  const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
  const int m = p.mat[c] ? (int)__ldg(p.mat[c] + id) : 0;
  if (__ldg(&p.mt->gjc[m]) == 0.f) return 0.f;
  const float mu = A.lT[c][((long long)bi * p.ade.n[1] + bj) * p.ade.n[2] + bk];
  return __fmul_rn(__fmul_rn(0.25f, __fmul_rn(__ldg(&p.mt->gS[m]), __ldg(&p.mt->gA[m]))), mu);
}

__global__ void adj_gyro_j_kernel(Params p, AdjDev A) {
  const MatTable& mt = *p.mt;
  int bi, bj, bk;
  long long q;
  if (!ade_cell(p, bi, bj, bk, q)) return;
  const int i = p.ade.lo[0] + bi, j = p.ade.lo[1] + bj, k = p.ade.lo[2] + bk;
  const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int m = p.mat[c] ? (int)__ldg(p.mat[c] + id) : 0;
    if (__ldg(&mt.gjc[m]) == 0.f) { A.lJg[c][q] = 0.f; continue; }
    const float t = __fmul_rn(__ldg(&mt.gA[m]), A.lT[c][q]);
    float v;
    if (c == 0) {
      // Jx(i,j) enters the averages of the y nodes (i,j+1), (i-1,j+1), (i,j), (i-1,j)
      const float acc = __fadd_rn(__fadd_rn(__fadd_rn(adj_gyro_term(p, A, 1, i, j + 1, k), adj_gyro_term(p, A, 1, i - 1, j + 1, k)),
                                            adj_gyro_term(p, A, 1, i, j, k)),
                                  adj_gyro_term(p, A, 1, i - 1, j, k));
      v = __fsub_rn(__fmul_rn(__ldg(&mt.gC[m]), t), acc);
    } else if (c == 1) {
      // Jy(i,j) enters the averages of the x nodes (i+1,j), (i,j), (i+1,j-1), (i,j-1)
      const float acc = __fadd_rn(__fadd_rn(__fadd_rn(adj_gyro_term(p, A, 0, i + 1, j, k), adj_gyro_term(p, A, 0, i, j, k)),
                                            adj_gyro_term(p, A, 0, i + 1, j - 1, k)),
                                  adj_gyro_term(p, A, 0, i, j - 1, k));
      v = __fmaf_rn(__ldg(&mt.gC[m]), t, acc);
    } else {
      v = t;
    }
    A.lJg[c][q] = v;
  }
}

// grad += lam_E (E^s - E^{s-1}) / ie over the design region (hist slots st, st-1);
// a design node whose material is dispersive takes no design permittivity: 0
__global__ void adj_grad_kernel(Params p, AdjDev A, int st) {
  const int nd = A.nd;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 3 * nd) return;
  const int c = q / nd, di = q - c * nd;
  const int i = p.des_lo[0] + di / (p.des_n[1] * p.des_n[2]);
  const int j = p.des_lo[1] + (di / p.des_n[2]) % p.des_n[1];
  const int k = p.des_lo[2] + di % p.des_n[2];
  const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
  if (p.mat[c] && __ldg(&p.mt->npoles[__ldg(p.mat[c] + id)]) > 0) return;
  const double dE = (double)A.hist[((long long)st * 3 + c) * nd + di] - (double)A.hist[((long long)(st - 1) * 3 + c) * nd + di];
  A.grad[q] += (double)A.lam[c][id] * dE / (double)p.des_ie[c][di];
}

// design-region E into history slot st
__global__ void design_capture_kernel(Params p, float* hist, int st, int nd) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 3 * nd) return;
  const int c = q / nd, di = q - c * nd;
  const int i = p.des_lo[0] + di / (p.des_n[1] * p.des_n[2]);
  const int j = p.des_lo[1] + (di / p.des_n[2]) % p.des_n[1];
  const int k = p.des_lo[2] + di % p.des_n[2];
  hist[((long long)st * 3 + c) * nd + di] = p.f[c][(long long)i * p.g.sx + (long long)j * p.g.sy + k];
}

}  // namespace dtmx
