// dtmx_device.cuh -- device-side data structures and per-plane field updates.
//
// The unit of work is one (z,y) tile of one x-plane: TZ = 32 nodes along z
// (one warp, coalesced 128-byte rows) by TYT = 16 nodes along y (8 warps, two
// rows per thread).  The y/z taps of the derivatives come from shared-memory
// copies of the neighbouring field's plane tile; the x taps come from the
// caller (a register queue when a CTA streams along x, direct loads in the
// wavefront engine).  Absorber (CPML or the reference split-field PML) and
// material coefficients are applied in the same pass; the Drude/Lorentz ADE
// nodes (reference countDisp) and the gyrotropic current are finished by a
// pass over the dispersive box after the E half step.
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
  int box;                   // box geometry: every node of the array is live, zero outside
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
  // magnetised-Drude (gyrotropic) current: decay, rotation cos/sin, E drive, dt/eps_inf (0: not gyrotropic)
  float gA[MAXMAT], gC[MAXMAT], gS[MAXMAT], gB[MAXMAT], gjc[MAXMAT];
};

struct Ade {
  int lo[3], n[3];           // box of cells holding ADE state
  float* Em[3];
  float* Jp[3][MAXPOLE];
  float* Jm[3][MAXPOLE];
  float* Jg[2][3];           // gyrotropic current, double-buffered
  int gnew;                  // buffer holding J^{n+1/2} during the E half step
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
  long long wait_limit;      // polls of one bounded wait (2^26; lowered only to test the timeout paths)
  // per (plane, y tile, z tile): the single non-dispersive material of all E
  // nodes of that plane tile, or -1 when mixed/dispersive
  const signed char* umat;
  int ntz, nty;              // tiles along z and y
  // E of the previous step when a pass reads it from another buffer than the
  // one it writes (the single-sweep engine's ADE pass); nullptr: in place
  const float* fe_old[3];
  // design region: per-node 1/eps of the E components over a cell box
  const float* des_ie[3];
  int des_lo[3], des_n[3];
  int des_on;
};

__host__ __device__ __forceinline__ long long design_index(const Params& p, int i, int j, int k) {
  if (!p.des_on) return -1;
  const int a = i - p.des_lo[0], b = j - p.des_lo[1], c = k - p.des_lo[2];
  if (a < 0 || a >= p.des_n[0] || b < 0 || b >= p.des_n[1] || c < 0 || c >= p.des_n[2]) return -1;
  return ((long long)a * p.des_n[1] + b) * p.des_n[2] + c;
}

// TMA descriptors of one context: source tiles (40 z x rows y x 1 plane),
// own-value tiles (32 x 16 x 1) of every component and material tiles.
struct TmaMaps {
  CUtensorMap src[6];
  CUtensorMap own[6];
  CUtensorMap mat[3];
};

// storage slot of component c for derivative axis a (-1: c has no derivative along a)
__host__ __device__ __forceinline__ constexpr int slot_of(int c, int a) {
  // Ex: y->0 z->0 ; Ey: x->0 z->1 ; Ez: x->1 y->1 ; Hx: y->2 z->2 ; Hy: x->2 z->3 ; Hz: x->3 y->3
  // (a conditional expression: a table indexed by a run-time c would live in local memory)
  return c == 0 ? (a == 0 ? -1 : 0)
       : c == 1 ? (a == 0 ? 0 : a == 1 ? -1 : 1)
       : c == 2 ? (a == 2 ? -1 : 1)
       : c == 3 ? (a == 0 ? -1 : 2)
       : c == 4 ? (a == 0 ? 2 : a == 1 ? -1 : 3)
                : (a == 2 ? -1 : 3);
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

// The node update is written with explicitly rounded operations (__fadd_rn,
// __fmul_rn, __fmaf_rn: no compiler contraction), so every kernel that
// evaluates it -- the per-half-step kernels and the wavefront engine -- gets
// bit-identical results whatever code surrounds it.
template <int ORDER>
__device__ __forceinline__ float dstencil(float v0, float v1, float v2, float v3) {
  if (ORDER == 2) return __fsub_rn(v2, v1);
  return __fmul_rn(__fmaf_rn(27.f, __fsub_rn(v2, v1), __fsub_rn(v0, v3)), 1.f / 24.f);
}
__device__ __forceinline__ float sum3(float a, float b, float c) { return __fadd_rn(__fadd_rn(a, b), c); }

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

// ---- asynchronous global -> shared copies (16-byte, L2 only: coherent with
// writes made by other CTAs of the same launch)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// own-value tile: 3 components x TYT rows x TZ floats; material tile: 3 x TYT x TZ bytes
constexpr int OWN_N = TYT * TZ;
__device__ __forceinline__ float own_at(const float* so, int c, int y, int z) { return so[c * OWN_N + y * TZ + z]; }
__device__ __forceinline__ int mat_at(const uint8_t* sm, int c, int y, int z) { return sm[c * OWN_N + y * TZ + z]; }

// Absorber correction of component c at a slab node: the update is
// F_new = F + dif[0] + dif[1] + dif[2] + correction, where for every slab axis a
//   CPML:  correction_a = (1/kappa_a - 1) dif_a + psi_a,  psi_a <- b psi_a + a dif_a
//   split: correction_a = (K1_a - 1) p_a + (K2_a - 1) dif_a,  p_a <- K1_a p_a + K2_a dif_a
// (the split form follows from F = rest + sum p_a with rest += undamped terms).
// Split into a load and an apply step so that callers can issue the slab
// loads early: absorb_load reads the auxiliary value of every slab axis of the
// node (0 elsewhere), absorb_apply computes the correction from those values
// and stores the new ones.
__device__ __forceinline__ void absorb_load(const Params& p, int c, int i, int j, int k, float (&old)[3]) {
  const int idx[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    old[a] = 0.f;
    const int sl = slot_of(c, a);
    if (sl < 0 || !in_slab(p, a, idx[a])) continue;
    old[a] = p.ab.aux[a][sl][slab_index(p, a, i, j, k)];
  }
}
__device__ __forceinline__ float absorb_apply(const Params& p, int c, int i, int j, int k, const float* dif,
                                              const float (&old)[3]) {
  const int idx[3] = {i, j, k};
  float corr = 0.f;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int sl = slot_of(c, a);
    if (sl < 0 || !in_slab(p, a, idx[a])) continue;
    const long long si = slab_index(p, a, i, j, k);
    const int h = 2 * idx[a] + comp_off(c, a);
    const float k0 = __ldg(p.ab.c0[a] + h), k1 = __ldg(p.ab.c1[a] + h);
    const float nv = __fmaf_rn(k0, old[a], __fmul_rn(k1, dif[a]));
    p.ab.aux[a][sl][si] = nv;
    if (p.ab.kind == 1) corr = __fadd_rn(corr, __fmaf_rn(__fsub_rn(__ldg(p.ab.c2[a] + h), 1.f), dif[a], nv));
    else corr = __fadd_rn(corr, __fsub_rn(__fsub_rn(nv, old[a]), dif[a]));
  }
  return corr;
}

// The same two steps for the streaming kernels, with the node's slab indices
// along the three axes computed once per node (-1 outside that slab) and
// shared by its three components; 32-bit (every slab array holds fewer than
// 2^31 values, checked when the absorber is set up).  Same arithmetic as
// absorb_load / absorb_apply.
__device__ __forceinline__ int slab_index32(const Params& p, int a, int i, int j, int k) {
  const int n = p.g.n[a], v = a == 0 ? i : a == 1 ? j : k;
  const int lo = p.ab.L[a][0], hi = p.ab.L[a][1];
  int cs;
  if (v < lo) cs = v;
  else if (v >= n - hi) cs = lo + (v - (n - hi));
  else return -1;
  if (a == 0) return (cs * p.g.n[1] + j) * p.g.n[2] + k;
  if (a == 1) return (i * (lo + hi) + cs) * p.g.n[2] + k;
  return (i * p.g.n[1] + j) * (lo + hi) + cs;
}
// slab indices of node (i,j,k); true when it lies in any slab
__device__ __forceinline__ bool node_slabs(const Params& p, int i, int j, int k, int (&si)[3]) {
  si[0] = slab_index32(p, 0, i, j, k);
  si[1] = slab_index32(p, 1, i, j, k);
  si[2] = slab_index32(p, 2, i, j, k);
  return (si[0] & si[1] & si[2]) >= 0;
}
__device__ __forceinline__ void absorb_load3(const Params& p, int c, const int (&si)[3], float (&old)[3]) {
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int sl = slot_of(c, a);
    old[a] = (sl >= 0 && si[a] >= 0) ? p.ab.aux[a][sl][si[a]] : 0.f;
  }
}
__device__ __forceinline__ float absorb_apply3(const Params& p, int c, const int (&idx)[3], const int (&si)[3],
                                               const float* dif, const float (&old)[3]) {
  float corr = 0.f;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int sl = slot_of(c, a);
    if (sl < 0 || si[a] < 0) continue;
    const int h = 2 * idx[a] + comp_off(c, a);
    const float k0 = __ldg(p.ab.c0[a] + h), k1 = __ldg(p.ab.c1[a] + h);
    const float nv = __fmaf_rn(k0, old[a], __fmul_rn(k1, dif[a]));
    p.ab.aux[a][sl][si[a]] = nv;
    if (p.ab.kind == 1) corr = __fadd_rn(corr, __fmaf_rn(__fsub_rn(__ldg(p.ab.c2[a] + h), 1.f), dif[a], nv));
    else corr = __fadd_rn(corr, __fsub_rn(__fsub_rn(nv, old[a]), dif[a]));
  }
  return corr;
}

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

// CTA-uniform tests: does the tile at plane i touch an absorber slab / the ADE box?
__device__ __forceinline__ bool tile_absorber(const Params& p, int i, int j0, int k0) {
  if (p.ab.kind == 0) return false;
  return in_slab(p, 0, i) || j0 < p.ab.L[1][0] || j0 + TYT > p.g.n[1] - p.ab.L[1][1] || k0 < p.ab.L[2][0] ||
         k0 + TZ > p.g.n[2] - p.ab.L[2][1];
}
__device__ __forceinline__ bool tile_ade(const Params& p, int i, int j0, int k0) {
  return i >= p.ade.lo[0] && i < p.ade.lo[0] + p.ade.n[0] && j0 + TYT > p.ade.lo[1] && j0 < p.ade.lo[1] + p.ade.n[1] &&
         k0 + TZ > p.ade.lo[2] && k0 < p.ade.lo[2] + p.ade.n[2];
}

// Per-thread absorber context of one node: which slabs hold it.
__device__ __forceinline__ bool node_in_absorber(const Params& p, bool inx, int j, int k) {
  return p.ab.kind != 0 && (inx || in_slab(p, 1, j) || in_slab(p, 2, k));
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
    sum = __fadd_rn(sum, __fmaf_rn(__ldg(&mt.kEJ[m][c][q][0]), jp[q], __fmul_rn(__ldg(&mt.kEJ[m][c][q][1]), jm[q])));
  }
  const float Ep = __fsub_rn(__fmaf_rn(__ldg(&mt.kE[m][c][0]), Em,
                                       __fmaf_rn(__ldg(&mt.kE[m][c][1]), F, __fmul_rn(__ldg(&mt.kE[m][c][2]), rot))),
                             sum);
  for (int q = 0; q < np; q++) {
    float a = __fmul_rn(__ldg(&mt.kJ[m][c][q][4]), Etmp);
    a = __fmaf_rn(__ldg(&mt.kJ[m][c][q][3]), Em, a);
    a = __fmaf_rn(__ldg(&mt.kJ[m][c][q][2]), Ep, a);
    a = __fmaf_rn(__ldg(&mt.kJ[m][c][q][1]), jm[q], a);
    p.ade.Jp[c][q][ai] = __fmaf_rn(__ldg(&mt.kJ[m][c][q][0]), jp[q], a);
    p.ade.Jm[c][q][ai] = jp[q];
  }
  p.ade.Em[c][ai] = Etmp;
  return Ep;
}

// Material coefficients used on the common path, staged in shared memory.
struct MatShared {
  float inv_eps[MAXMAT][3];
  int npoles[MAXMAT];
  float gjc[MAXMAT];
};

__device__ __forceinline__ void load_matshared(MatShared& ms, const Params& p) {
  const int tid = threadIdx.y * TZ + threadIdx.x;
  for (int q = tid; q < MAXMAT * 3; q += NTHR) (&ms.inv_eps[0][0])[q] = __ldg(&p.mt->inv_eps[0][0] + q);
  for (int q = tid; q < MAXMAT; q += NTHR) { ms.npoles[q] = __ldg(&p.mt->npoles[q]); ms.gjc[q] = __ldg(&p.mt->gjc[q]); }
}

// E -= dt/eps_inf J^{n+1/2} on a gyrotropic node (J computed by gyro_current_kernel)
__device__ __forceinline__ float gyro_subtract(const Params& p, int c, int i, int j, int k, float gjc, float nv) {
  const int bi = i - p.ade.lo[0], bj = j - p.ade.lo[1], bk = k - p.ade.lo[2];
  if (bi < 0 || bi >= p.ade.n[0] || bj < 0 || bj >= p.ade.n[1] || bk < 0 || bk >= p.ade.n[2]) return nv;
  const long long ai = ((long long)bi * p.ade.n[1] + bj) * p.ade.n[2] + bk;
  return __fsub_rn(nv, __fmul_rn(gjc, p.ade.Jg[p.ade.gnew][c][ai]));
}

// Absorber auxiliaries of the thread's nodes in plane i (absorber tiles only).
// They do not depend on the staged tiles, so the streaming loop issues these
// loads before it waits for the plane's stage, hiding their latency.
template <bool ISH>
__device__ __forceinline__ void absorb_prefetch(const Params& p, int i, int j0, int k0, float (&old)[RY][3][3]) {
  const int cf = ISH ? 3 : 0;
#pragma unroll
  for (int r = 0; r < RY; r++) {
    const int j = j0 + threadIdx.y + TW * r, k = k0 + threadIdx.x;
    int si[3];
    if (j >= p.g.n[1] || k >= p.g.n[2] || !node_slabs(p, i, j, k, si)) continue;
#pragma unroll
    for (int c = 0; c < 3; c++) absorb_load3(p, cf + c, si, old[r][c]);
  }
}

// Update of one plane tile (all three components of the half step).  Common
// path: F + sum of the signed derivative terms (times 1/eps for E); slab
// nodes add the absorber correction, dispersive nodes (E step, tiles touching
// the ADE box) are replaced by the ADE recursion, non-live nodes are skipped.
//   um >= 0: every E node of the tile has non-dispersive material um
// MODE 1 (simple): every node live, no absorber, uniform material um (>= 0);
// MODE 2 (absorber): the same with absorber slabs in the tile;
// MODE 0: the general path.  All three evaluate the same expressions.
template <int ORDER, bool ISH, int MODE>
__device__ __forceinline__ void plane_update(const Params& p, int i, int j0, int k0, const float* sm,
                                             const float (&qb)[RY][4], const float (&qc)[RY][4], const float* so,
                                             const uint8_t* smat, const MatShared& ms, bool fast, int um,
                                             const float (&old)[RY][3][3]) {
  constexpr bool SIMPLE = MODE == 1, ABSU = MODE == 2;
  using S = Stage<ORDER, ISH>;
  const float* sA = sm;
  const float* sB = sA + S::TA::N;
  const float* sC = sB + S::TB::N;
  const int tz = threadIdx.x, w = threadIdx.y;
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  const int cf = ISH ? 3 : 0;
  const long long pbase = (long long)i * p.g.sx;
  const bool tab = ABSU || (!SIMPLE && tile_absorber(p, i, j0, k0));
  const bool tade = MODE == 0 && !ISH && tile_ade(p, i, j0, k0);
  float iu[3] = {1.f, 1.f, 1.f};
  if ((SIMPLE || ABSU) && !ISH) { iu[0] = ms.inv_eps[um][0]; iu[1] = ms.inv_eps[um][1]; iu[2] = ms.inv_eps[um][2]; }
  constexpr int o0 = ISH ? -2 : -1, o1 = o0 + 1, o2 = o0 + 2, o3 = o0 + 3;
#pragma unroll
  for (int r = 0; r < RY; r++) {
    const int y = w + TW * r;
    const int j = j0 + y, k = k0 + tz;
    if (MODE == 0 && !fast && (j >= p.g.n[1] || k >= p.g.n[2])) continue;
    const long long off = pbase + (long long)j * p.g.sy + k;
    const float dyC = dstencil<ORDER>(ORDER == 4 ? S::TC::at(sC, y, tz, o0, 0) : 0.f, S::TC::at(sC, y, tz, o1, 0),
                                      S::TC::at(sC, y, tz, o2, 0), ORDER == 4 ? S::TC::at(sC, y, tz, o3, 0) : 0.f);
    const float dzB = dstencil<ORDER>(ORDER == 4 ? S::TB::at(sB, y, tz, 0, o0) : 0.f, S::TB::at(sB, y, tz, 0, o1),
                                      S::TB::at(sB, y, tz, 0, o2), ORDER == 4 ? S::TB::at(sB, y, tz, 0, o3) : 0.f);
    const float dzA = dstencil<ORDER>(ORDER == 4 ? S::TA::at(sA, y, tz, 0, o0) : 0.f, S::TA::at(sA, y, tz, 0, o1),
                                      S::TA::at(sA, y, tz, 0, o2), ORDER == 4 ? S::TA::at(sA, y, tz, 0, o3) : 0.f);
    const float dyA = dstencil<ORDER>(ORDER == 4 ? S::TA::at(sA, y, tz, o0, 0) : 0.f, S::TA::at(sA, y, tz, o1, 0),
                                      S::TA::at(sA, y, tz, o2, 0), ORDER == 4 ? S::TA::at(sA, y, tz, o3, 0) : 0.f);
    const float dxC = dstencil<ORDER>(qc[r][0], qc[r][1], qc[r][2], qc[r][3]);
    const float dxB = dstencil<ORDER>(qb[r][0], qb[r][1], qb[r][2], qb[r][3]);
    // signed, scaled derivative terms per component, [comp][axis]
    float d[3][3];
    if (ISH) {
      // Hx -= dt(dy Ez - dz Ey); Hy -= dt(dz Ex - dx Ez); Hz -= dt(dx Ey - dy Ex)
      d[0][0] = 0.f;                  d[0][1] = __fmul_rn(-cy, dyC); d[0][2] = __fmul_rn(cz, dzB);
      d[1][0] = __fmul_rn(cx, dxC);   d[1][1] = 0.f;                 d[1][2] = __fmul_rn(-cz, dzA);
      d[2][0] = __fmul_rn(-cx, dxB);  d[2][1] = __fmul_rn(cy, dyA);  d[2][2] = 0.f;
    } else {
      // Ex += dt/eps(dy Hz - dz Hy); Ey += dt/eps(dz Hx - dx Hz); Ez += dt/eps(dx Hy - dy Hx)
      d[0][0] = 0.f;                  d[0][1] = __fmul_rn(cy, dyC);  d[0][2] = __fmul_rn(-cz, dzB);
      d[1][0] = __fmul_rn(-cx, dxC);  d[1][1] = 0.f;                 d[1][2] = __fmul_rn(cz, dzA);
      d[2][0] = __fmul_rn(cx, dxB);   d[2][1] = __fmul_rn(-cy, dyA); d[2][2] = 0.f;
    }
    int si[3] = {-1, -1, -1};
    const bool ab = tab && node_slabs(p, i, j, k, si);
    const int idx3[3] = {i, j, k};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (MODE == 0 && !fast && !is_live(p.g, cf + c, i, j, k)) continue;
      float F = own_at(so, c, y, tz);
      if (SIMPLE || ABSU) {
        if (!ISH) { d[c][0] = __fmul_rn(d[c][0], iu[c]); d[c][1] = __fmul_rn(d[c][1], iu[c]); d[c][2] = __fmul_rn(d[c][2], iu[c]); }
        float inc = sum3(d[c][0], d[c][1], d[c][2]);
        if (ABSU && ab) inc = __fadd_rn(inc, absorb_apply3(p, cf + c, idx3, si, d[c], old[r][c]));
        p.f[cf + c][off] = __fadd_rn(F, inc);
        continue;
      }
      int m = 0;
      if (!ISH) {
        m = um >= 0 ? um : mat_at(smat, c, y, tz);
        if (tade && ms.npoles[m] > 0) {
          // dispersive node: left to ade_node_kernel, which runs after this kernel
          const int bi = i - p.ade.lo[0], bj = j - p.ade.lo[1], bk = k - p.ade.lo[2];
          if (bi >= 0 && bi < p.ade.n[0] && bj >= 0 && bj < p.ade.n[1] && bk >= 0 && bk < p.ade.n[2]) continue;
        }
        float ie = ms.inv_eps[m][c];
        if (p.des_on) {
          const long long di = design_index(p, i, j, k);
          if (di >= 0) ie = p.des_ie[c][di];
        }
        d[c][0] = __fmul_rn(d[c][0], ie); d[c][1] = __fmul_rn(d[c][1], ie); d[c][2] = __fmul_rn(d[c][2], ie);
      }
      float inc = sum3(d[c][0], d[c][1], d[c][2]);
      if (ab) inc = __fadd_rn(inc, absorb_apply3(p, cf + c, idx3, si, d[c], old[r][c]));
      float nv = __fadd_rn(F, inc);
      p.f[cf + c][off] = nv;
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
