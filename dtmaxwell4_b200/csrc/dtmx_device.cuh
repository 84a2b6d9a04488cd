// dtmx_device.cuh -- device-side data structures and per-plane field updates.
//
// The unit of work is one (z,y) tile of one x-plane: TZ = 32 nodes along z
// (one warp, coalesced 128-byte rows) by TYT = 16 nodes along y (8 warps, two
// rows per thread).  The y/z taps of the derivatives come from shared-memory
// copies of the neighbouring field's plane tile; the x taps come from the
// caller (a register queue when a CTA streams along x, direct loads in the
// wavefront engine).  Absorber (CPML or the reference split-field PML),
// material coefficients and the Drude/Lorentz ADE (reference countDisp) are
// applied in the same pass.
//
// Update equations (reference generator genAlg.py:182-301, defs.h:3-13):
//   H -= dt * curl E,  E += dt/eps * curl H  (c = 1),
//   D f = (27 (f[+1/2] - f[-1/2]) - (f[+3/2] - f[-3/2])) / 24   (order 4)
//   D f = f[+1/2] - f[-1/2]                                     (order 2)
// H nodes take taps at index offsets -2..+1, E nodes at -1..+2.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace dtmx {

constexpr int TZ = 32;          // tile extent along z (one warp)
constexpr int TW = 8;           // warps per CTA
constexpr int RY = 2;           // y rows per thread
constexpr int TYT = TW * RY;    // tile extent along y
constexpr int NTHR = TZ * TW;
constexpr int MAXMAT = 64;
constexpr int MAXPOLE = 2;

// half-cell offset of component c along axis a (lattice in dtmx.h)
__host__ __device__ __forceinline__ int comp_off(int c, int a) { return c < 3 ? (a != c) : (a == c - 3); }

struct Grid {
  int n[3];
  long long sx, sy;          // element strides of x and y (z stride 1)
  int live_lo[6][3], live_hi[6][3];
  int all_lo[3], all_hi[3];  // index range live for every component
  int safe_lo[3], safe_hi[3];// index range whose taps need no mirror mapping (zero sides unbounded)
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
  int x0, x1;                // planes [x0, x1) processed by a streaming launch
  int xchunk;                // planes per CTA along x
  int* err;                  // device error word (bounded waits that gave up)
};

// TMA descriptors of one context: source tiles (40 z x rows y x 1 plane),
// own-value tiles (32 x 16 x 1) of every component and material tiles.
struct TmaMaps {
  CUtensorMap src[6];
  CUtensorMap own[6];
  CUtensorMap mat[3];
};

// storage slot of component c for derivative axis a (-1: c has no derivative along a)
__host__ __device__ __forceinline__ int slot_of(int c, int a) {
  // Ex: y->0 z->0 ; Ey: x->0 z->1 ; Ez: x->1 y->1 ; Hx: y->2 z->2 ; Hy: x->2 z->3 ; Hz: x->3 y->3
  const int S[6][3] = {{-1, 0, 0}, {0, -1, 1}, {1, 1, -1}, {-1, 2, 2}, {2, -1, 3}, {3, 3, -1}};
  return S[c][a];
}

// Loads: LD = 0 read-only path (field not written during the launch),
// LD = 1 L2-coherent path (written by other CTAs of the same launch).
template <int LD>
__device__ __forceinline__ float ldf(const float* q) { return LD ? __ldcg(q) : __ldg(q); }

// Map index v of component c along axis a to the stored index, applying the
// boundary rule outside the live range; returns -1 when the value is zero.
__device__ __forceinline__ int map_idx(const Grid& g, int c, int a, int v, float& sgn) {
  const int lo = g.live_lo[c][a], hi = g.live_hi[c][a];
  if (v >= lo && v <= hi) return v;
  const int side = v < lo ? 0 : 1;
  if (g.btype[a][side] == 0) return (v >= 0 && v < g.n[a]) ? v : -1;   // non-live cells hold zero
  const int o = comp_off(c, a);
  const int h2 = 2 * g.bplane[a][side] - (2 * v + o);
  const int v2 = (h2 - o) >> 1;
  sgn *= (float)((c < 3) ? g.bsE[a][side] : g.bsH[a][side]);
  if (v2 < lo || v2 > hi) return -1;
  return v2;
}

template <int LD>
__device__ __forceinline__ float fetch(const Params& p, int c, int i, int j, int k) {
  float s = 1.f;
  const int ii = map_idx(p.g, c, 0, i, s);
  const int jj = map_idx(p.g, c, 1, j, s);
  const int kk = map_idx(p.g, c, 2, k, s);
  if ((ii | jj | kk) < 0) return 0.f;
  return s * ldf<LD>(p.f[c] + ii * p.g.sx + jj * p.g.sy + kk);
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

__device__ __forceinline__ bool in_slab(const Params& p, int a, int v) {
  return v < p.ab.L[a][0] || v >= p.g.n[a] - p.ab.L[a][1];
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

// Absorber update of component c at cell (i,j,k), which lies in at least one
// absorber slab: dif[a] are the signed, scaled derivative terms; returns the
// new value given the old value F.
__device__ __forceinline__ float absorb_update(const Params& p, int c, int i, int j, int k, const float* dif, float F) {
  long long si[3];
  const int idx[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    si[a] = -1;
    if (slot_of(c, a) < 0 || (p.ab.L[a][0] + p.ab.L[a][1]) == 0) continue;
    si[a] = slab_index(p, a, i, j, k);
  }
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

// ---- asynchronous global -> shared copies (16-byte, L2 only: coherent with
// writes made by other CTAs of the same launch)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Shared-memory copy of one component's plane tile: rows of TW_ROW floats
// covering z in [k0-4, k0+36) (16-byte aligned), with YL/YH halo rows in y.
constexpr int ZO = 4;                 // z offset of node k0 inside a row
constexpr int TW_ROW = TZ + 2 * ZO;   // 40 floats = 10 x 16 bytes
template <int YL, int YH>
struct Tile {
  static constexpr int H = TYT + YL + YH;
  static constexpr int NV = TW_ROW * H;                 // floats written by a load
  static constexpr int N = (NV + 31) / 32 * 32;         // footprint, 128-byte multiple
  // fast: every element is an in-array interior value -> async 16-byte copies
  __device__ static void load_async(float* sm, const Params& p, int c, int i, int j0, int k0) {
    const float* base = p.f[c] + (long long)i * p.g.sx + (long long)(j0 - YL) * p.g.sy + (k0 - ZO);
    const int tid = threadIdx.y * TZ + threadIdx.x;
    for (int q = tid; q < H * (TW_ROW / 4); q += NTHR) {
      const int r = q / (TW_ROW / 4), col = q - r * (TW_ROW / 4);
      cp_async16(sm + r * TW_ROW + col * 4, base + (long long)r * p.g.sy + col * 4);
    }
  }
  // boundary tiles: element-wise with the boundary rules (z halo of 2 each side)
  template <int LD>
  __device__ static void load_slow(float* sm, const Params& p, int c, int i, int j0, int k0) {
    const int lane = threadIdx.x, w = threadIdx.y;
    for (int r = w; r < H; r += TW) {
      const int j = j0 - YL + r;
      sm[r * TW_ROW + ZO + lane] = fetch<LD>(p, c, i, j, k0 + lane);
      if (lane < 2 * ZO) {
        const int dz = lane < ZO ? lane - ZO : TZ + lane - ZO;   // -4..-1 and 32..35
        sm[r * TW_ROW + ZO + dz] = fetch<LD>(p, c, i, j, k0 + dz);
      }
    }
  }
  // (y, z) tile-local node coordinates, (dy, dz) tap offsets
  __device__ static float at(const float* sm, int y, int z, int dy, int dz) {
    return sm[(y + YL + dy) * TW_ROW + (z + ZO + dz)];
  }
};

// fast-path test: all taps of the tile at plane i are live for every component
__device__ __forceinline__ bool tile_interior(const Grid& g, int i, int j0, int k0) {
  return i - 2 >= g.all_lo[0] && i + 2 <= g.all_hi[0] && j0 - 2 >= g.all_lo[1] && j0 + TYT + 1 <= g.all_hi[1] &&
         k0 - 2 >= g.all_lo[2] && k0 + TZ + 1 <= g.all_hi[2];
}

// The three source-component tiles of one plane (one pipeline stage).
template <int ORDER, bool ISH>
struct Stage {
  static constexpr int R = ORDER / 2;
  static constexpr int YL = ISH ? R : R - 1, YH = ISH ? R - 1 : R;
  using TA = Tile<YL, YH>;                     // Ex (H step) / Hx (E step): y and z taps
  using TB = Tile<0, 0>;                       // Ey / Hy: z taps and own value
  using TC = Tile<YL, YH>;                     // Ez / Hz: y taps and own value
  static constexpr int N = TA::N + TB::N + TC::N;
  static constexpr int c0 = ISH ? 0 : 3;       // first source component
  template <int LD>
  __device__ static void load(float* sm, const Params& p, int i, int j0, int k0, bool fast) {
    if (fast) {
      TA::load_async(sm, p, c0, i, j0, k0);
      TB::load_async(sm + TA::N, p, c0 + 1, i, j0, k0);
      TC::load_async(sm + TA::N + TB::N, p, c0 + 2, i, j0, k0);
    } else {
      TA::template load_slow<LD>(sm, p, c0, i, j0, k0);
      TB::template load_slow<LD>(sm + TA::N, p, c0 + 1, i, j0, k0);
      TC::template load_slow<LD>(sm + TA::N + TB::N, p, c0 + 2, i, j0, k0);
    }
  }
  __device__ static float own_b(const float* sm, int y, int z) { return TB::at(sm + TA::N, y, z, 0, 0); }
  __device__ static float own_c(const float* sm, int y, int z) { return TC::at(sm + TA::N + TB::N, y, z, 0, 0); }
};

// Per-thread absorber context of one node: which slabs hold it.
__device__ __forceinline__ bool node_in_absorber(const Params& p, bool inx, int j, int k) {
  return p.ab.kind != 0 && (inx || in_slab(p, 1, j) || in_slab(p, 2, k));
}

// ---------------------------------------------------------------- H half step
// Hx -= dt (dy Ez - dz Ey),  Hy -= dt (dz Ex - dx Ez),  Hz -= dt (dx Ey - dy Ex)
// qy[r][0..3], qz[r][0..3]: Ey, Ez of the thread's node r at planes i-2..i+1.
// own-value tile: 3 components x TYT rows x TZ floats; material tile: 3 x TYT x TZ bytes
constexpr int OWN_N = TYT * TZ;
__device__ __forceinline__ float own_at(const float* so, int c, int y, int z) { return so[c * OWN_N + y * TZ + z]; }
__device__ __forceinline__ int mat_at(const uint8_t* sm, int c, int y, int z) { return sm[c * OWN_N + y * TZ + z]; }

template <int ORDER, int LD>
__device__ __forceinline__ void h_plane(const Params& p, int i, int j0, int k0, const float* sm, const float (&qy)[RY][4],
                                        const float (&qz)[RY][4], bool fast, const float* so) {
  using S = Stage<ORDER, true>;
  const float* sEx = sm;
  const float* sEy = sEx + S::TA::N;
  const float* sEz = sEy + S::TB::N;
  const int tz = threadIdx.x, w = threadIdx.y;
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  const bool inx = p.ab.kind != 0 && in_slab(p, 0, i);
  const long long pbase = (long long)i * p.g.sx;
#pragma unroll
  for (int r = 0; r < RY; r++) {
    const int y = w + TW * r;
    const int j = j0 + y, k = k0 + tz;
    if (!fast && (j >= p.g.n[1] || k >= p.g.n[2])) continue;
    const long long off = pbase + (long long)j * p.g.sy + k;
    const bool ab = node_in_absorber(p, inx, j, k);
    float a0, a1, a2, a3;
    // ---- Hx
    if (fast || is_live(p.g, 3, i, j, k)) {
      a0 = ORDER == 4 ? S::TC::at(sEz, y, tz, -2, 0) : 0.f; a1 = S::TC::at(sEz, y, tz, -1, 0);
      a2 = S::TC::at(sEz, y, tz, 0, 0); a3 = ORDER == 4 ? S::TC::at(sEz, y, tz, 1, 0) : 0.f;
      const float dyEz = dstencil<ORDER>(a0, a1, a2, a3);
      a0 = ORDER == 4 ? S::TB::at(sEy, y, tz, 0, -2) : 0.f; a1 = S::TB::at(sEy, y, tz, 0, -1);
      a2 = S::TB::at(sEy, y, tz, 0, 0); a3 = ORDER == 4 ? S::TB::at(sEy, y, tz, 0, 1) : 0.f;
      const float dzEy = dstencil<ORDER>(a0, a1, a2, a3);
      const float dif[3] = {0.f, -cy * dyEz, cz * dzEy};
      const float F0 = own_at(so, 0, y, tz);
      p.f[3][off] = ab ? absorb_update(p, 3, i, j, k, dif, F0) : F0 + dif[0] + dif[1] + dif[2];
    }
    // ---- Hy
    if (fast || is_live(p.g, 4, i, j, k)) {
      a0 = ORDER == 4 ? S::TA::at(sEx, y, tz, 0, -2) : 0.f; a1 = S::TA::at(sEx, y, tz, 0, -1);
      a2 = S::TA::at(sEx, y, tz, 0, 0); a3 = ORDER == 4 ? S::TA::at(sEx, y, tz, 0, 1) : 0.f;
      const float dzEx = dstencil<ORDER>(a0, a1, a2, a3);
      const float dxEz = dstencil<ORDER>(qz[r][0], qz[r][1], qz[r][2], qz[r][3]);
      const float dif[3] = {cx * dxEz, 0.f, -cz * dzEx};
      const float F1 = own_at(so, 1, y, tz);
      p.f[4][off] = ab ? absorb_update(p, 4, i, j, k, dif, F1) : F1 + dif[0] + dif[1] + dif[2];
    }
    // ---- Hz
    if (fast || is_live(p.g, 5, i, j, k)) {
      const float dxEy = dstencil<ORDER>(qy[r][0], qy[r][1], qy[r][2], qy[r][3]);
      a0 = ORDER == 4 ? S::TA::at(sEx, y, tz, -2, 0) : 0.f; a1 = S::TA::at(sEx, y, tz, -1, 0);
      a2 = S::TA::at(sEx, y, tz, 0, 0); a3 = ORDER == 4 ? S::TA::at(sEx, y, tz, 1, 0) : 0.f;
      const float dyEx = dstencil<ORDER>(a0, a1, a2, a3);
      const float dif[3] = {-cx * dxEy, cy * dyEx, 0.f};
      const float F2 = own_at(so, 2, y, tz);
      p.f[5][off] = ab ? absorb_update(p, 5, i, j, k, dif, F2) : F2 + dif[0] + dif[1] + dif[2];
    }
  }
}

// ---------------------------------------------------------------- E half step
// ADE branch restates countDisp (dispersion.cpp:85-99).
__device__ __forceinline__ float ade_update(const Params& p, int c, int m, int np, long long ai, float rot, float F) {
  const MatTable& mt = *p.mt;
  const float Em = p.ade.Em[c][ai];
  const float Etmp = F;
  float sum = 0.f;
  float jp[MAXPOLE], jm[MAXPOLE];
  for (int q = 0; q < np; q++) {
    jp[q] = p.ade.Jp[c][q][ai]; jm[q] = p.ade.Jm[c][q][ai];
    sum += __ldg(&mt.kEJ[m][c][q][0]) * jp[q] + __ldg(&mt.kEJ[m][c][q][1]) * jm[q];
  }
  const float Ep = __ldg(&mt.kE[m][c][0]) * Em + __ldg(&mt.kE[m][c][1]) * F + __ldg(&mt.kE[m][c][2]) * rot - sum;
  for (int q = 0; q < np; q++) {
    p.ade.Jp[c][q][ai] = __ldg(&mt.kJ[m][c][q][0]) * jp[q] + __ldg(&mt.kJ[m][c][q][1]) * jm[q] +
                         __ldg(&mt.kJ[m][c][q][2]) * Ep + __ldg(&mt.kJ[m][c][q][3]) * Em +
                         __ldg(&mt.kJ[m][c][q][4]) * Etmp;
    p.ade.Jm[c][q][ai] = jp[q];
  }
  p.ade.Em[c][ai] = Etmp;
  return Ep;
}

// Material coefficients used on the common path, staged in shared memory.
struct MatShared {
  float inv_eps[MAXMAT][3];
  int npoles[MAXMAT];
};

__device__ __forceinline__ void load_matshared(MatShared& ms, const Params& p) {
  const int tid = threadIdx.y * TZ + threadIdx.x;
  for (int q = tid; q < MAXMAT * 3; q += NTHR) (&ms.inv_eps[0][0])[q] = __ldg(&p.mt->inv_eps[0][0] + q);
  for (int q = tid; q < MAXMAT; q += NTHR) ms.npoles[q] = __ldg(&p.mt->npoles[q]);
}

__device__ __forceinline__ float e_node(const Params& p, const MatShared& ms, int c, int m, int i, int j, int k, bool ab,
                                        float (&dif)[3], float F) {
  const int np = ms.npoles[m];
  if (np > 0) {
    const int bi = i - p.ade.lo[0], bj = j - p.ade.lo[1], bk = k - p.ade.lo[2];
    if (bi >= 0 && bi < p.ade.n[0] && bj >= 0 && bj < p.ade.n[1] && bk >= 0 && bk < p.ade.n[2]) {
      const long long ai = ((long long)bi * p.ade.n[1] + bj) * p.ade.n[2] + bk;
      return ade_update(p, c, m, np, ai, dif[0] + dif[1] + dif[2], F);
    }
  }
  const float ie = ms.inv_eps[m][c];
  dif[0] *= ie; dif[1] *= ie; dif[2] *= ie;
  return ab ? absorb_update(p, c, i, j, k, dif, F) : F + dif[0] + dif[1] + dif[2];
}

// Ex += dt/eps (dy Hz - dz Hy), Ey += dt/eps (dz Hx - dx Hz), Ez += dt/eps (dx Hy - dy Hx)
// qy[r][0..3], qz[r][0..3]: Hy, Hz of the thread's node r at planes i-1..i+2.
template <int ORDER, int LD>
__device__ __forceinline__ void e_plane(const Params& p, int i, int j0, int k0, const float* sm, const float (&qy)[RY][4],
                                        const float (&qz)[RY][4], bool fast, const float* so, const uint8_t* smat,
                                        const MatShared& ms) {
  using S = Stage<ORDER, false>;
  const float* sHx = sm;
  const float* sHy = sHx + S::TA::N;
  const float* sHz = sHy + S::TB::N;
  const int tz = threadIdx.x, w = threadIdx.y;
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  const bool inx = p.ab.kind != 0 && in_slab(p, 0, i);
  const long long pbase = (long long)i * p.g.sx;
#pragma unroll
  for (int r = 0; r < RY; r++) {
    const int y = w + TW * r;
    const int j = j0 + y, k = k0 + tz;
    if (!fast && (j >= p.g.n[1] || k >= p.g.n[2])) continue;
    const long long off = pbase + (long long)j * p.g.sy + k;
    const bool ab = node_in_absorber(p, inx, j, k);
    float a0, a1, a2, a3;
    // ---- Ex
    if (fast || is_live(p.g, 0, i, j, k)) {
      a0 = ORDER == 4 ? S::TC::at(sHz, y, tz, -1, 0) : 0.f; a1 = S::TC::at(sHz, y, tz, 0, 0);
      a2 = S::TC::at(sHz, y, tz, 1, 0); a3 = ORDER == 4 ? S::TC::at(sHz, y, tz, 2, 0) : 0.f;
      const float dyHz = dstencil<ORDER>(a0, a1, a2, a3);
      a0 = ORDER == 4 ? S::TB::at(sHy, y, tz, 0, -1) : 0.f; a1 = S::TB::at(sHy, y, tz, 0, 0);
      a2 = S::TB::at(sHy, y, tz, 0, 1); a3 = ORDER == 4 ? S::TB::at(sHy, y, tz, 0, 2) : 0.f;
      const float dzHy = dstencil<ORDER>(a0, a1, a2, a3);
      float dif[3] = {0.f, cy * dyHz, -cz * dzHy};
      p.f[0][off] = e_node(p, ms, 0, mat_at(smat, 0, y, tz), i, j, k, ab, dif, own_at(so, 0, y, tz));
    }
    // ---- Ey
    if (fast || is_live(p.g, 1, i, j, k)) {
      a0 = ORDER == 4 ? S::TA::at(sHx, y, tz, 0, -1) : 0.f; a1 = S::TA::at(sHx, y, tz, 0, 0);
      a2 = S::TA::at(sHx, y, tz, 0, 1); a3 = ORDER == 4 ? S::TA::at(sHx, y, tz, 0, 2) : 0.f;
      const float dzHx = dstencil<ORDER>(a0, a1, a2, a3);
      const float dxHz = dstencil<ORDER>(qz[r][0], qz[r][1], qz[r][2], qz[r][3]);
      float dif[3] = {-cx * dxHz, 0.f, cz * dzHx};
      p.f[1][off] = e_node(p, ms, 1, mat_at(smat, 1, y, tz), i, j, k, ab, dif, own_at(so, 1, y, tz));
    }
    // ---- Ez
    if (fast || is_live(p.g, 2, i, j, k)) {
      const float dxHy = dstencil<ORDER>(qy[r][0], qy[r][1], qy[r][2], qy[r][3]);
      a0 = ORDER == 4 ? S::TA::at(sHx, y, tz, -1, 0) : 0.f; a1 = S::TA::at(sHx, y, tz, 0, 0);
      a2 = S::TA::at(sHx, y, tz, 1, 0); a3 = ORDER == 4 ? S::TA::at(sHx, y, tz, 2, 0) : 0.f;
      const float dyHx = dstencil<ORDER>(a0, a1, a2, a3);
      float dif[3] = {cx * dxHy, -cy * dyHx, 0.f};
      p.f[2][off] = e_node(p, ms, 2, mat_at(smat, 2, y, tz), i, j, k, ab, dif, own_at(so, 2, y, tz));
    }
  }
}

// x taps of the thread's nodes: component c at plane ip (fast: direct load)
template <int LD>
__device__ __forceinline__ void load_xtaps(const Params& p, int c, int ip, int j0, int k0, bool fast, float (&out)[RY]) {
  const int tz = threadIdx.x, w = threadIdx.y;
#pragma unroll
  for (int r = 0; r < RY; r++) {
    const int j = j0 + w + TW * r, k = k0 + tz;
    if (fast) out[r] = ldf<LD>(p.f[c] + (long long)ip * p.g.sx + (long long)j * p.g.sy + k);
    else out[r] = (j < p.g.n[1] && k < p.g.n[2]) ? fetch<LD>(p, c, ip, j, k) : 0.f;
  }
}

}  // namespace dtmx

#include "dtmx_stream.cuh"
