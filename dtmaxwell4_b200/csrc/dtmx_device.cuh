// dtmx_device.cuh -- device-side data structures and kernels of the FDTD engine.
//
// One half step (all three H components, or all three E components) is one
// streaming kernel: a CTA owns a (z,y) tile of TZ x TY nodes and marches
// along x, keeping the x taps of the derivative in a register queue and the
// y/z taps of the current plane in shared memory.  Absorber (CPML or the
// reference split-field PML), material coefficients and the Drude/Lorentz ADE
// (reference countDisp) are fused into the same pass.
//
// Update equations (reference generator genAlg.py:182-301, defs.h:3-13):
//   H -= dt * curl E,  E += dt/eps * curl H  (c = 1),
//   D f = (27 (f[+1/2] - f[-1/2]) - (f[+3/2] - f[-3/2])) / 24   (order 4)
//   D f = f[+1/2] - f[-1/2]                                     (order 2)
// H nodes take taps at index offsets -2..+1, E nodes at -1..+2.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dtmx {

constexpr int TZ = 32;     // tile extent along z (one warp)
constexpr int TY = 8;      // tile extent along y (warps per CTA)
constexpr int NTHR = TZ * TY;
constexpr int MAXMAT = 64;
constexpr int MAXPOLE = 2;

// half-cell offset of component c along axis a (lattice in dtmx.h)
__host__ __device__ __forceinline__ int comp_off(int c, int a) { return c < 3 ? (a != c) : (a == c - 3); }

struct Grid {
  int n[3];
  long long sx, sy;          // element strides of x and y (z stride 1)
  int live_lo[6][3], live_hi[6][3];
  int btype[3][2], bplane[3][2];
  int bsE[3][2], bsH[3][2];
};

struct Absorb {
  int kind;                  // 0 none, 1 CPML, 2 split PML
  int L[3][2];               // slab thickness in cells
  float* aux[3][4];          // per axis: 4 slots (2 E comps, 2 H comps) over the slab cells
  const float* c0[3];        // CPML b      | split K1     (indexed by half-coordinate)
  const float* c1[3];        // CPML a      | split K2
  const float* c2[3];        // CPML 1/kappa
};

struct MatTable {
  float inv_eps[MAXMAT][3];
  int npoles[MAXMAT];
  float kEJ[MAXMAT][3][MAXPOLE][2];
  float kE[MAXMAT][3][3];
  float kJ[MAXMAT][3][MAXPOLE][5];
};

struct Ade {
  int lo[3], n[3];           // box of cells holding ADE state
  float* Em[3];
  float* Jp[3][MAXPOLE];
  float* Jm[3][MAXPOLE];
};

struct Params {
  Grid g;
  float* f[6];
  float cdt[3];              // dt/dx, dt/dy, dt/dz
  Absorb ab;
  const uint8_t* mat[3];     // per E component material index (nullptr -> material 0)
  const MatTable* mt;
  Ade ade;
  int x0, x1;                // planes [x0, x1) processed by this launch
  int xchunk;                // planes per CTA along x
};

// storage slot of component c for derivative axis a (-1: c has no derivative along a)
__host__ __device__ __forceinline__ int slot_of(int c, int a) {
  // Ex: y->0 z->0 ; Ey: x->0 z->1 ; Ez: x->1 y->1 ; Hx: y->2 z->2 ; Hy: x->2 z->3 ; Hz: x->3 y->3
  const int S[6][3] = {{-1, 0, 0}, {0, -1, 1}, {1, 1, -1}, {-1, 2, 2}, {2, -1, 3}, {3, 3, -1}};
  return S[c][a];
}

// Map index v of component c along axis a to the stored index, applying the
// boundary rule outside the live range; returns -1 when the value is zero.
__device__ __forceinline__ int map_idx(const Grid& g, int c, int a, int v, float& sgn) {
  int lo = g.live_lo[c][a], hi = g.live_hi[c][a];
  if (v >= lo && v <= hi) return v;
  int side = v < lo ? 0 : 1;
  if (g.btype[a][side] == 0) return (v >= 0 && v < g.n[a]) ? v : -1;   // non-live cells hold zero
  int o = comp_off(c, a);
  int h2 = 2 * g.bplane[a][side] - (2 * v + o);
  int v2 = (h2 - o) >> 1;
  sgn *= (float)((c < 3) ? g.bsE[a][side] : g.bsH[a][side]);
  if (v2 < lo || v2 > hi) return -1;
  return v2;
}

__device__ __forceinline__ float fetch(const Params& p, int c, int i, int j, int k) {
  float s = 1.f;
  int ii = map_idx(p.g, c, 0, i, s);
  int jj = map_idx(p.g, c, 1, j, s);
  int kk = map_idx(p.g, c, 2, k, s);
  if ((ii | jj | kk) < 0) return 0.f;
  return s * __ldg(p.f[c] + ii * p.g.sx + jj * p.g.sy + kk);
}

template <int ORDER>
__device__ __forceinline__ float dstencil(float v0, float v1, float v2, float v3) {
  if (ORDER == 2) return v2 - v1;
  return (27.f * (v2 - v1) - (v3 - v0)) * (1.f / 24.f);
}

__device__ __forceinline__ bool is_live(const Grid& g, int c, int i, int j, int k) {
  return i >= g.live_lo[c][0] && i <= g.live_hi[c][0] && j >= g.live_lo[c][1] && j <= g.live_hi[c][1] &&
         k >= g.live_lo[c][2] && k <= g.live_hi[c][2];
}

__device__ __forceinline__ long long slab_index(const Params& p, int a, int i, int j, int k) {
  const int n = p.g.n[a];
  const int c = a == 0 ? i : a == 1 ? j : k;
  const int lo = p.ab.L[a][0], hi = p.ab.L[a][1];
  int cs;
  if (c < lo) cs = c;
  else if (c >= n - hi) cs = lo + (c - (n - hi));
  else return -1;
  const int th = lo + hi;
  if (a == 0) return ((long long)cs * p.g.n[1] + j) * p.g.n[2] + k;
  if (a == 1) return ((long long)i * th + cs) * p.g.n[2] + k;
  return ((long long)i * p.g.n[1] + j) * th + cs;
}

// Apply the absorber to component c at cell (i,j,k): dif[a] are the signed,
// scaled derivative terms; returns the new value given the old value F.
__device__ __forceinline__ float absorb_update(const Params& p, int c, int i, int j, int k, const float dif[3], float F) {
  if (p.ab.kind == 0) return F + dif[0] + dif[1] + dif[2];
  long long si[3];
  bool any = false;
  const int idx[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    si[a] = -1;
    if (slot_of(c, a) < 0 || (p.ab.L[a][0] + p.ab.L[a][1]) == 0) continue;
    si[a] = slab_index(p, a, i, j, k);
    any |= si[a] >= 0;
  }
  if (!any) return F + dif[0] + dif[1] + dif[2];
  if (p.ab.kind == 1) {
    float add = 0.f;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int sl = slot_of(c, a);
      if (sl < 0) continue;
      if (si[a] < 0) { add += dif[a]; continue; }
      const int h = 2 * idx[a] + comp_off(c, a);
      float* psi = p.ab.aux[a][sl] + si[a];
      const float nv = __ldg(p.ab.c0[a] + h) * *psi + __ldg(p.ab.c1[a] + h) * dif[a];
      *psi = nv;
      add += __ldg(p.ab.c2[a] + h) * dif[a] + nv;
    }
    return F + add;
  }
  // split field: F = rest + sum of stored directional parts
  float rest = F, tot = 0.f;
#pragma unroll
  for (int a = 0; a < 3; a++)
    if (si[a] >= 0) rest -= p.ab.aux[a][slot_of(c, a)][si[a]];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int sl = slot_of(c, a);
    if (sl < 0) continue;
    if (si[a] >= 0) {
      const int h = 2 * idx[a] + comp_off(c, a);
      float* pp = p.ab.aux[a][sl] + si[a];
      const float nv = __ldg(p.ab.c0[a] + h) * *pp + __ldg(p.ab.c1[a] + h) * dif[a];
      *pp = nv;
      tot += nv;
    } else {
      rest += dif[a];
    }
  }
  return rest + tot;
}

// Shared-memory tile of one component of plane i with halo (ZL,ZH) in z and (YL,YH) in y.
template <int ZL, int ZH, int YL, int YH>
struct Tile {
  static constexpr int W = TZ + ZL + ZH;
  static constexpr int H = TY + YL + YH;
  static constexpr int N = W * H;
  __device__ static void load(float* sm, const Params& p, int c, int i, int j0, int k0, int tid) {
    for (int e = tid; e < N; e += NTHR) {
      const int zz = e % W, yy = e / W;
      sm[e] = fetch(p, c, i, j0 - YL + yy, k0 - ZL + zz);
    }
  }
  __device__ static float at(const float* sm, int ty, int tz, int dy, int dz) {
    return sm[(ty + YL + dy) * W + (tz + ZL + dz)];
  }
};

// ---------------------------------------------------------------- H half step
// Hx -= dt (dy Ez - dz Ey),  Hy -= dt (dz Ex - dx Ez),  Hz -= dt (dx Ey - dy Ex)
template <int ORDER>
__global__ void __launch_bounds__(NTHR) h_kernel(Params p) {
  constexpr int R = ORDER / 2;                 // taps below: 2R-? ; H taps -R..R-1
  using TEx = Tile<R, R - 1, R, R - 1>;        // dy and dz taps of Ex
  using TEy = Tile<R, R - 1, 0, 0>;            // dz taps of Ey
  using TEz = Tile<0, 0, R, R - 1>;            // dy taps of Ez
  __shared__ float sEx[TEx::N], sEy[TEy::N], sEz[TEz::N];
  const int tz = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tz;
  const int k0 = blockIdx.x * TZ, j0 = blockIdx.y * TY;
  const int k = k0 + tz, j = j0 + ty;
  const int xa = p.x0 + blockIdx.z * p.xchunk;
  const int xb = min(xa + p.xchunk, p.x1);
  const bool in = (j < p.g.n[1]) && (k < p.g.n[2]);
  // register queues of Ey, Ez along x: q[0..3] = planes i-2..i+1 (order 4), i-1..i (order 2)
  float qy[4], qz[4];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    qy[q + 1] = in ? fetch(p, 1, xa - 2 + q, j, k) : 0.f;
    qz[q + 1] = in ? fetch(p, 2, xa - 2 + q, j, k) : 0.f;
  }
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  for (int i = xa; i < xb; i++) {
#pragma unroll
    for (int q = 0; q < 3; q++) { qy[q] = qy[q + 1]; qz[q] = qz[q + 1]; }
    qy[3] = in ? fetch(p, 1, i + 1, j, k) : 0.f;
    qz[3] = in ? fetch(p, 2, i + 1, j, k) : 0.f;
    TEx::load(sEx, p, 0, i, j0, k0, tid);
    TEy::load(sEy, p, 1, i, j0, k0, tid);
    TEz::load(sEz, p, 2, i, j0, k0, tid);
    __syncthreads();
    if (in) {
      // taps v0..v3 at offsets -2..+1 (order 4) ; order 2 uses v1, v2 = offsets -1, 0
      float a0, a1, a2, a3;
      // ---- Hx
      if (is_live(p.g, 3, i, j, k)) {
        a0 = ORDER == 4 ? TEz::at(sEz, ty, tz, -2, 0) : 0.f; a1 = TEz::at(sEz, ty, tz, -1, 0);
        a2 = TEz::at(sEz, ty, tz, 0, 0); a3 = ORDER == 4 ? TEz::at(sEz, ty, tz, 1, 0) : 0.f;
        const float dyEz = dstencil<ORDER>(a0, a1, a2, a3);
        a0 = ORDER == 4 ? TEy::at(sEy, ty, tz, 0, -2) : 0.f; a1 = TEy::at(sEy, ty, tz, 0, -1);
        a2 = TEy::at(sEy, ty, tz, 0, 0); a3 = ORDER == 4 ? TEy::at(sEy, ty, tz, 0, 1) : 0.f;
        const float dzEy = dstencil<ORDER>(a0, a1, a2, a3);
        float dif[3] = {0.f, -cy * dyEz, cz * dzEy};
        float* ph = p.f[3] + i * p.g.sx + j * p.g.sy + k;
        *ph = absorb_update(p, 3, i, j, k, dif, *ph);
      }
      // ---- Hy
      if (is_live(p.g, 4, i, j, k)) {
        a0 = ORDER == 4 ? TEx::at(sEx, ty, tz, 0, -2) : 0.f; a1 = TEx::at(sEx, ty, tz, 0, -1);
        a2 = TEx::at(sEx, ty, tz, 0, 0); a3 = ORDER == 4 ? TEx::at(sEx, ty, tz, 0, 1) : 0.f;
        const float dzEx = dstencil<ORDER>(a0, a1, a2, a3);
        const float dxEz = dstencil<ORDER>(qz[0], qz[1], qz[2], qz[3]);
        float dif[3] = {cx * dxEz, 0.f, -cz * dzEx};
        float* ph = p.f[4] + i * p.g.sx + j * p.g.sy + k;
        *ph = absorb_update(p, 4, i, j, k, dif, *ph);
      }
      // ---- Hz
      if (is_live(p.g, 5, i, j, k)) {
        const float dxEy = dstencil<ORDER>(qy[0], qy[1], qy[2], qy[3]);
        a0 = ORDER == 4 ? TEx::at(sEx, ty, tz, -2, 0) : 0.f; a1 = TEx::at(sEx, ty, tz, -1, 0);
        a2 = TEx::at(sEx, ty, tz, 0, 0); a3 = ORDER == 4 ? TEx::at(sEx, ty, tz, 1, 0) : 0.f;
        const float dyEx = dstencil<ORDER>(a0, a1, a2, a3);
        float dif[3] = {-cx * dxEy, cy * dyEx, 0.f};
        float* ph = p.f[5] + i * p.g.sx + j * p.g.sy + k;
        *ph = absorb_update(p, 5, i, j, k, dif, *ph);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- E half step
// ADE branch restates countDisp (dispersion.cpp:85-99).
__device__ __forceinline__ float e_node(const Params& p, int c, int i, int j, int k, float dif[3], float F) {
  const long long id = (long long)i * p.g.sx + (long long)j * p.g.sy + k;
  const int m = p.mat[c] ? (int)__ldg(p.mat[c] + id) : 0;
  const MatTable& mt = *p.mt;
  const int np = mt.npoles[m];
  if (np > 0) {
    const int bi = i - p.ade.lo[0], bj = j - p.ade.lo[1], bk = k - p.ade.lo[2];
    if (bi >= 0 && bi < p.ade.n[0] && bj >= 0 && bj < p.ade.n[1] && bk >= 0 && bk < p.ade.n[2]) {
      const long long ai = ((long long)bi * p.ade.n[1] + bj) * p.ade.n[2] + bk;
      const float rot = dif[0] + dif[1] + dif[2];
      float Ep = F;
      const float Em = p.ade.Em[c][ai];
      const float Etmp = Ep;
      float sum = 0.f;
      float jp[MAXPOLE], jm[MAXPOLE];
      for (int q = 0; q < np; q++) {
        jp[q] = p.ade.Jp[c][q][ai]; jm[q] = p.ade.Jm[c][q][ai];
        sum += mt.kEJ[m][c][q][0] * jp[q] + mt.kEJ[m][c][q][1] * jm[q];
      }
      Ep = mt.kE[m][c][0] * Em + mt.kE[m][c][1] * Ep + mt.kE[m][c][2] * rot - sum;
      for (int q = 0; q < np; q++) {
        p.ade.Jp[c][q][ai] = mt.kJ[m][c][q][0] * jp[q] + mt.kJ[m][c][q][1] * jm[q] + mt.kJ[m][c][q][2] * Ep +
                             mt.kJ[m][c][q][3] * Em + mt.kJ[m][c][q][4] * Etmp;
        p.ade.Jm[c][q][ai] = jp[q];
      }
      p.ade.Em[c][ai] = Etmp;
      return Ep;
    }
  }
  const float ie = mt.inv_eps[m][c];
  dif[0] *= ie; dif[1] *= ie; dif[2] *= ie;
  return absorb_update(p, c, i, j, k, dif, F);
}

// Ex += dt/eps (dy Hz - dz Hy), Ey += dt/eps (dz Hx - dx Hz), Ez += dt/eps (dx Hy - dy Hx)
template <int ORDER>
__global__ void __launch_bounds__(NTHR) e_kernel(Params p) {
  constexpr int R = ORDER / 2;                 // E taps -(R-1)..R  -> halo R-1 below, R above
  using THx = Tile<R - 1, R, R - 1, R>;        // dz and dy taps of Hx
  using THy = Tile<R - 1, R, 0, 0>;            // dz taps of Hy
  using THz = Tile<0, 0, R - 1, R>;            // dy taps of Hz
  __shared__ float sHx[THx::N], sHy[THy::N], sHz[THz::N];
  const int tz = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tz;
  const int k0 = blockIdx.x * TZ, j0 = blockIdx.y * TY;
  const int k = k0 + tz, j = j0 + ty;
  const int xa = p.x0 + blockIdx.z * p.xchunk;
  const int xb = min(xa + p.xchunk, p.x1);
  const bool in = (j < p.g.n[1]) && (k < p.g.n[2]);
  // q[0..3] = planes i-1..i+2
  float qy[4], qz[4];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    qy[q + 1] = in ? fetch(p, 4, xa - 1 + q, j, k) : 0.f;
    qz[q + 1] = in ? fetch(p, 5, xa - 1 + q, j, k) : 0.f;
  }
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  for (int i = xa; i < xb; i++) {
#pragma unroll
    for (int q = 0; q < 3; q++) { qy[q] = qy[q + 1]; qz[q] = qz[q + 1]; }
    qy[3] = in ? fetch(p, 4, i + 2, j, k) : 0.f;
    qz[3] = in ? fetch(p, 5, i + 2, j, k) : 0.f;
    THx::load(sHx, p, 3, i, j0, k0, tid);
    THy::load(sHy, p, 4, i, j0, k0, tid);
    THz::load(sHz, p, 5, i, j0, k0, tid);
    __syncthreads();
    if (in) {
      float a0, a1, a2, a3;
      // ---- Ex
      if (is_live(p.g, 0, i, j, k)) {
        a0 = ORDER == 4 ? THz::at(sHz, ty, tz, -1, 0) : 0.f; a1 = THz::at(sHz, ty, tz, 0, 0);
        a2 = THz::at(sHz, ty, tz, 1, 0); a3 = ORDER == 4 ? THz::at(sHz, ty, tz, 2, 0) : 0.f;
        const float dyHz = dstencil<ORDER>(a0, a1, a2, a3);
        a0 = ORDER == 4 ? THy::at(sHy, ty, tz, 0, -1) : 0.f; a1 = THy::at(sHy, ty, tz, 0, 0);
        a2 = THy::at(sHy, ty, tz, 0, 1); a3 = ORDER == 4 ? THy::at(sHy, ty, tz, 0, 2) : 0.f;
        const float dzHy = dstencil<ORDER>(a0, a1, a2, a3);
        float dif[3] = {0.f, cy * dyHz, -cz * dzHy};
        float* pe = p.f[0] + i * p.g.sx + j * p.g.sy + k;
        *pe = e_node(p, 0, i, j, k, dif, *pe);
      }
      // ---- Ey
      if (is_live(p.g, 1, i, j, k)) {
        a0 = ORDER == 4 ? THx::at(sHx, ty, tz, 0, -1) : 0.f; a1 = THx::at(sHx, ty, tz, 0, 0);
        a2 = THx::at(sHx, ty, tz, 0, 1); a3 = ORDER == 4 ? THx::at(sHx, ty, tz, 0, 2) : 0.f;
        const float dzHx = dstencil<ORDER>(a0, a1, a2, a3);
        const float dxHz = dstencil<ORDER>(qz[0], qz[1], qz[2], qz[3]);
        float dif[3] = {-cx * dxHz, 0.f, cz * dzHx};
        float* pe = p.f[1] + i * p.g.sx + j * p.g.sy + k;
        *pe = e_node(p, 1, i, j, k, dif, *pe);
      }
      // ---- Ez
      if (is_live(p.g, 2, i, j, k)) {
        const float dxHy = dstencil<ORDER>(qy[0], qy[1], qy[2], qy[3]);
        a0 = ORDER == 4 ? THx::at(sHx, ty, tz, -1, 0) : 0.f; a1 = THx::at(sHx, ty, tz, 0, 0);
        a2 = THx::at(sHx, ty, tz, 1, 0); a3 = ORDER == 4 ? THx::at(sHx, ty, tz, 2, 0) : 0.f;
        const float dyHx = dstencil<ORDER>(a0, a1, a2, a3);
        float dif[3] = {cx * dxHy, -cy * dyHx, 0.f};
        float* pe = p.f[2] + i * p.g.sx + j * p.g.sy + k;
        *pe = e_node(p, 2, i, j, k, dif, *pe);
      }
    }
    __syncthreads();
  }
}

}  // namespace dtmx
