// dtmx_fused.cuh -- single-sweep engine: one launch per time step advances H
// and then E, plane by plane, reading the old fields once and writing the new
// ones once.
//
// The fields are kept twice (A, B).  A step reads A and writes B, and the next
// step the other way round, so no CTA can see a value that another CTA of the
// same launch has already advanced.  That lets a CTA recompute, redundantly,
// the new H on the one-node halo its E update needs (the row above the tile
// and the column beyond it) instead of waiting for the neighbour that owns
// those nodes.  The per-step engine makes two passes over the grid per step
// (H, then E), each reading the field the other one writes; this engine makes
// one.
//
// Tile: the per-step kernels' 32 (z, lanes) x 16 (y, 8 warps x 2 rows) node
// tile, walked upwards along an x chunk.  Iteration t of the walk consumes the
// stage of plane pc = x0 + t and
//   * computes the new H of plane pc on the own nodes (and, split over warps
//     0-3, the halo: Hz and Hx of row 16, Hy and Hx of column 32) from the old
//     E of planes pc (staged) and pc - 1 (registers) and the old H of plane pc
//     (staged); the own values go to B and, with the halo, to a shared-memory
//     plane buffer;
//   * computes the new E of plane pc - 1 on the own nodes from its old E
//     (registers), the new H of plane pc - 1 (the other shared-memory plane
//     buffer; own nodes from registers) and of plane pc (registers).
// Each old value is therefore read from HBM once per step (the halo rows and
// columns of the TMA boxes come from L2), and every plane costs one CTA
// barrier.  One elected thread issues the TMA copies (cp.async.bulk.tensor,
// no multicast) of a plane's E box (18 rows x 40 floats per component), old-H
// boxes and, when the E update of the previous plane needs them, that plane's
// material tiles, into a 3-stage ring (two planes in flight).  Everything
// outside the grid reads as zero (TMA fill; new H forced to zero outside),
// which is the box geometry; other geometries use the per-step engine.
//
// The node updates are the expressions of plane_update (dtmx_device.cuh), in
// the same order with the same explicitly rounded operations, so without a
// TF/SF source this engine's fields are bit-identical to the per-step
// engine's.  With one, the H correction is added to the old H before the sweep
// (the update is linear in it), which rounds differently at the box faces.
#pragma once
#include "dtmx_stream.cuh"

namespace dtmx {

constexpr int FE_W = 40;                     // E box: z in [k0-4, k0+36) (16-byte aligned start)
constexpr int FHX_W = 36, FHY_W = 36, FHZ_W = 32;
constexpr int F_NST = 3;
constexpr int HN_P = TZ + 1;                 // new-H plane buffer: z in [k0, k0+33)
constexpr int FX_MAX = 64;                   // longest x chunk
constexpr int F_MROWS = 16;                  // material tiles: the per-step kernels' 32 x 16 boxes
__host__ __device__ constexpr int f_up32(int v) { return (v + 31) / 32 * 32; }

// Shared-memory layout of a tile of NR rows per warp (8 NR rows), in floats.
template <int NR>
struct FL {
  static constexpr int TY = TW * NR;                 // own rows of a tile (16 or 8)
  static constexpr int FE_R = TY + 2;                // E box rows: y in [j0-1, j0+TY+1)
  static constexpr int FE_N = f_up32(FE_R * FE_W);
  static constexpr int FHX_R = TY + 1, FHY_R = TY, FHZ_R = TY + 1;   // old-H boxes
  static constexpr int OFF_HX = 3 * FE_N;
  static constexpr int OFF_HY = OFF_HX + f_up32(FHX_W * FHX_R);
  static constexpr int OFF_HZ = OFF_HY + f_up32(FHY_W * FHY_R);
  static constexpr int OFF_M = OFF_HZ + f_up32(FHZ_W * FHZ_R);
  static constexpr int STAGE = OFF_M + 3 * F_MROWS * TZ / 4;
  static constexpr unsigned BYTES = (3 * FE_W * FE_R + FHX_W * FHX_R + FHY_W * FHY_R + FHZ_W * FHZ_R) * 4;
  static constexpr unsigned BYTES_MAT = 3 * F_MROWS * TZ;
  static constexpr int HN_N = (TY + 1) * HN_P;       // new-H plane, per component: y in [j0, j0+TY+1)
  static constexpr int HN = f_up32(3 * HN_N);
  static constexpr size_t SMEM = (size_t)(F_NST * STAGE + 2 * HN) * 4 + sizeof(MatShared) + F_NST * 8 + 128;
};
static_assert(FL<2>::STAGE == 4352 && FL<2>::OFF_HX == 2208, "16-row layout");

// TMA descriptors of one buffer set for one tile height
struct FusedMaps {
  CUtensorMap e[3];                          // 40 x (TY+2) E boxes
  CUtensorMap hx, hy, hz;                    // old-H boxes
  CUtensorMap mat[3];                        // 32 x 16 material tiles (the per-step kernels' maps)
};

// Per-launch arguments beyond Params (which describes the source buffer A)
struct FusedArgs {
  float* dst[6];                             // buffer B
  float* hsrc[3][2];                         // CPML auxiliaries of H (slots 2, 3) in A
  float* hdst[3][2];                         // ... and in B
};

// staged-tile accessors (tile-local y, z)
template <int NR>
__device__ __forceinline__ float fE(const float* st, int c, int y, int z) {
  return st[c * FL<NR>::FE_N + (y + 1) * FE_W + z + 4];
}
template <int NR> __device__ __forceinline__ float fHx(const float* st, int y, int z) { return st[FL<NR>::OFF_HX + y * FHX_W + z]; }
template <int NR> __device__ __forceinline__ float fHy(const float* st, int y, int z) { return st[FL<NR>::OFF_HY + y * FHY_W + z]; }
template <int NR> __device__ __forceinline__ float fHz(const float* st, int y, int z) { return st[FL<NR>::OFF_HZ + y * FHZ_W + z]; }
template <int NR>
__device__ __forceinline__ int fM(const float* st, int c, int y, int z) {
  return reinterpret_cast<const uint8_t*>(st + FL<NR>::OFF_M)[c * F_MROWS * TZ + y * TZ + z];
}
template <int NR>
__device__ __forceinline__ float& fN(float* hn, int q, int y, int z) { return hn[q * FL<NR>::HN_N + y * HN_P + z]; }
template <int NR>
__device__ __forceinline__ float fN(const float* hn, int q, int y, int z) { return hn[q * FL<NR>::HN_N + y * HN_P + z]; }

// CPML correction of component C at node (i, j, k) with slab indices si
// (absorb_apply3 of the CPML form); H auxiliaries read from A and written to
// B, E auxiliaries in place.  store false: a node whose new value this CTA
// does not own (halo, the plane after the chunk) reads its auxiliaries only.
template <int C>
__device__ __forceinline__ float fused_cpml(const Params& p, const FusedArgs& fa, const int (&idx)[3], const int (&si)[3],
                                            const float (&dif)[3], bool store) {
  float corr = 0.f;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int sl = slot_of(C, a);
    if (sl < 0 || si[a] < 0) continue;
    const int h = 2 * idx[a] + comp_off(C, a);
    const float k0 = __ldg(p.ab.c0[a] + h), k1 = __ldg(p.ab.c1[a] + h);
    const float old = C >= 3 ? __ldg(fa.hsrc[a][sl - 2] + si[a]) : p.ab.aux[a][sl][si[a]];
    const float nv = __fmaf_rn(k0, old, __fmul_rn(k1, dif[a]));
    if (store) (C >= 3 ? fa.hdst[a][sl - 2] : p.ab.aux[a][sl])[si[a]] = nv;
    corr = __fadd_rn(corr, __fmaf_rn(__fsub_rn(__ldg(p.ab.c2[a] + h), 1.f), dif[a], nv));
  }
  return corr;
}

// new H component C (3..5) = old + sum of the derivative terms d (+ CPML)
template <int C, bool ABS>
__device__ __forceinline__ float fused_hnode(const Params& p, const FusedArgs& fa, float old, float d0, float d1, float d2,
                                             bool slab, const int (&idx)[3], const int (&si)[3], bool store) {
  float inc = sum3(d0, d1, d2);
  if (ABS && slab) {
    const float dif[3] = {d0, d1, d2};
    inc = __fadd_rn(inc, fused_cpml<C>(p, fa, idx, si, dif, store));
  }
  return __fadd_rn(old, inc);
}

// ---- absorber tiles
// CPML coefficients are staged per CTA in shared memory, 6 floats per node
// coordinate v of an axis: b, a, 1/kappa - 1 at half-coordinate 2v (the H
// components' offset along a derivative axis) and at 2v + 1 (the E
// components').  Rows: x planes x0-1 .. x0+FX_MAX, y rows j0 .. j0+16, z
// columns k0 .. k0+32.
constexpr int FCO_X = 0, FCO_Y = (FX_MAX + 2) * 6, FCO_Z = FCO_Y + (F_MROWS + 1) * 6, FCO_N = FCO_Z + (TZ + 1) * 6;

// index of coordinate v in the slab of its axis (-1 outside)
__device__ __forceinline__ int slab_cs(const Params& p, int a, int v) {
  const int n = p.g.n[a], lo = p.ab.L[a][0], hi = p.ab.L[a][1];
  return v < lo ? v : (v >= n - hi ? lo + v - (n - hi) : -1);
}

// slab indices of node (i, j, k) along the axes of AXM (bit a: axis a may hold
// a slab), from its slab coordinates xs, ys, zs (-1 outside); the slab_index32 layouts
template <int AXM>
__device__ __forceinline__ void fused_slabs(const Params& p, int i, int j, int k, int xs, int ys, int zs, int (&si)[3]) {
  si[0] = ((AXM & 1) && xs >= 0) ? (xs * p.g.n[1] + j) * p.g.n[2] + k : -1;
  si[1] = ((AXM & 2) && ys >= 0) ? (i * (p.ab.L[1][0] + p.ab.L[1][1]) + ys) * p.g.n[2] + k : -1;
  si[2] = ((AXM & 4) && zs >= 0) ? (i * p.g.n[1] + j) * (p.ab.L[2][0] + p.ab.L[2][1]) + zs : -1;
}

// the old auxiliaries of one node for one half of the update: per slab axis a
// the two slots of that axis (H: slots 2, 3 from A; E: slots 0, 1 in place)
template <int AXM, bool ISH>
__device__ __forceinline__ void fused_aux_load(const Params& p, const FusedArgs& fa, const int (&si)[3], float (&old)[3][2]) {
#pragma unroll
  for (int a = 0; a < 3; a++) {
    old[a][0] = 0.f; old[a][1] = 0.f;
    if (!((AXM >> a) & 1) || si[a] < 0) continue;
    if (ISH) { old[a][0] = __ldg(fa.hsrc[a][0] + si[a]); old[a][1] = __ldg(fa.hsrc[a][1] + si[a]); }
    else { old[a][0] = p.ab.aux[a][0][si[a]]; old[a][1] = p.ab.aux[a][1][si[a]]; }
  }
}

// CPML correction of component C from preloaded auxiliaries and staged
// coefficients (the arithmetic of absorb_apply3, CPML form); store: the new
// auxiliaries belong to this CTA.  Every axis of AXM takes part without a
// branch: off its slab a node reads 0 and the coefficients there are b = 1,
// a = 0, 1/kappa - 1 = 0, so its term is exactly zero and nothing is stored.
template <int C, int AXM>
__device__ __forceinline__ float fused_aux_apply(const Params& p, const FusedArgs& fa, const int (&si)[3],
                                                 const float (&old)[3][2], const float (&dif)[3], const float* cx,
                                                 const float* cy, const float* cz, bool store) {
  float corr = 0.f;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int sl = slot_of(C, a);
    if (sl < 0 || !((AXM >> a) & 1)) continue;
    const int q = sl & 1;
    const float* cf = (a == 0 ? cx : a == 1 ? cy : cz) + (C >= 3 ? 0 : 3);
    const float nv = __fmaf_rn(cf[0], old[a][q], __fmul_rn(cf[1], dif[a]));
    if (store && si[a] >= 0) (C >= 3 ? fa.hdst[a][q] : p.ab.aux[a][q])[si[a]] = nv;
    corr = __fadd_rn(corr, __fmaf_rn(cf[2], dif[a], nv));
  }
  return corr;
}

// New H of plane i on the thread's own nodes: hc (registers), hn (shared
// plane buffer), B (when the chunk owns plane i).  ec gets the old E of the
// own nodes (the next plane's x taps and its E update); ep holds those of
// plane i - 1.  AXM: the slab axes of the tile-plane (0: no absorber); the
// slab coordinates xs (plane), ys (rows), zs (column) are per-thread constants.
template <int NR, int AXM>
__device__ __forceinline__ void fused_h_own(const Params& p, const FusedArgs& fa, const float* st, float* hn, int i,
                                            int j0, int k0, bool store, const bool (&ok)[NR], const float (&ep)[NR][3],
                                            float (&hc)[NR][3], float (&ec)[NR][3], const float* fco, int xs,
                                            const int (&ys)[NR], int zs) {
  const int lane = threadIdx.x, w = threadIdx.y;
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  const long long pb = (long long)i * p.g.sx;
  int si[NR][3];
  float old[NR][3][2];
  if (AXM) {
    // every auxiliary of the thread's nodes is requested before any is used
#pragma unroll
    for (int r = 0; r < NR; r++) {
      fused_slabs<AXM>(p, i, j0 + w + TW * r, k0 + lane, xs, ys[r], zs, si[r]);
      if (!ok[r]) si[r][0] = si[r][1] = si[r][2] = -1;
      fused_aux_load<AXM, true>(p, fa, si[r], old[r]);
    }
  }
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int y = w + TW * r, j = j0 + y, k = k0 + lane;
    const float ez = fE<NR>(st, 2, y, lane), ey = fE<NR>(st, 1, y, lane), ex = fE<NR>(st, 0, y, lane);
    ec[r][0] = ex; ec[r][1] = ey; ec[r][2] = ez;
    // Hx -= dt(dy Ez - dz Ey); Hy -= dt(dz Ex - dx Ez); Hz -= dt(dx Ey - dy Ex)
    const float dhx[3] = {0.f, __fmul_rn(-cy, __fsub_rn(ez, fE<NR>(st, 2, y - 1, lane))),
                         __fmul_rn(cz, __fsub_rn(ey, fE<NR>(st, 1, y, lane - 1)))};
    const float dhy[3] = {__fmul_rn(cx, __fsub_rn(ez, ep[r][2])), 0.f,
                         __fmul_rn(-cz, __fsub_rn(ex, fE<NR>(st, 0, y, lane - 1)))};
    const float dhz[3] = {__fmul_rn(-cx, __fsub_rn(ey, ep[r][1])), __fmul_rn(cy, __fsub_rn(ex, fE<NR>(st, 0, y - 1, lane))),
                         0.f};
    float ix = sum3(dhx[0], dhx[1], dhx[2]), iy = sum3(dhy[0], dhy[1], dhy[2]), iz = sum3(dhz[0], dhz[1], dhz[2]);
    if (AXM && (si[r][0] & si[r][1] & si[r][2]) >= 0) {
      const float* fx = fco + FCO_X + (i - p.x0 - blockIdx.z * p.xchunk + 1) * 6;
      const float* fy = fco + FCO_Y + y * 6;
      const float* fz = fco + FCO_Z + lane * 6;
      ix = __fadd_rn(ix, fused_aux_apply<3, AXM>(p, fa, si[r], old[r], dhx, fx, fy, fz, store));
      iy = __fadd_rn(iy, fused_aux_apply<4, AXM>(p, fa, si[r], old[r], dhy, fx, fy, fz, store));
      iz = __fadd_rn(iz, fused_aux_apply<5, AXM>(p, fa, si[r], old[r], dhz, fx, fy, fz, store));
    }
    float vx = __fadd_rn(fHx<NR>(st, y, lane), ix), vy = __fadd_rn(fHy<NR>(st, y, lane), iy), vz = __fadd_rn(fHz<NR>(st, y, lane), iz);
    if (!ok[r]) { vx = 0.f; vy = 0.f; vz = 0.f; }
    hc[r][0] = vx; hc[r][1] = vy; hc[r][2] = vz;
    fN<NR>(hn, 0, y, lane) = vx;
    fN<NR>(hn, 1, y, lane) = vy;
    fN<NR>(hn, 2, y, lane) = vz;
    if (store && ok[r]) {
      const long long off = pb + (long long)j * p.g.sy + k;
      fa.dst[3][off] = vx;
      fa.dst[4][off] = vy;
      fa.dst[5][off] = vz;
    }
  }
}

// The halo of the new-H plane buffer (values the E update of the tile reads
// beyond its own nodes), one component per warp:
//   warp 0: Hz of row 16      warp 1: Hx of row 16
//   warp 2: Hy of column 32   warp 3: Hx of column 32 (lanes 0-15)
// xe: the warp's old E of the previous plane at its halo node (x tap), updated.
// A CPML slab node takes the correction with the auxiliaries read, not written.
template <int NR, bool ABS>
__device__ __forceinline__ void fused_h_halo(const Params& p, const FusedArgs& fa, const float* st, float* hn, int i,
                                             int j0, int k0, float& xe) {
  const int lane = threadIdx.x, w = threadIdx.y;
  if (w > 3 || (w > 1 && lane >= FL<NR>::TY)) return;
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  const bool row = w < 2;
  const int y = row ? FL<NR>::TY : lane, z = row ? lane : TZ;
  const int j = j0 + y, k = k0 + z;
  const bool ok = j < p.g.n[1] && k < p.g.n[2];
  int si[3] = {-1, -1, -1};
  const int idx[3] = {i, j, k};
  const bool slab = ABS && ok && node_slabs(p, i, j, k, si);
  float v;
  if (w == 0) {
    const float ey = fE<NR>(st, 1, y, z);
    const float d0 = __fmul_rn(-cx, __fsub_rn(ey, xe));
    const float d1 = __fmul_rn(cy, __fsub_rn(fE<NR>(st, 0, y, z), fE<NR>(st, 0, y - 1, z)));
    v = fused_hnode<5, ABS>(p, fa, fHz<NR>(st, y, z), d0, d1, 0.f, slab, idx, si, false);
    xe = ey;
  } else if (w == 2) {
    const float ez = fE<NR>(st, 2, y, z);
    const float d0 = __fmul_rn(cx, __fsub_rn(ez, xe));
    const float d2 = __fmul_rn(-cz, __fsub_rn(fE<NR>(st, 0, y, z), fE<NR>(st, 0, y, z - 1)));
    v = fused_hnode<4, ABS>(p, fa, fHy<NR>(st, y, z), d0, 0.f, d2, slab, idx, si, false);
    xe = ez;
  } else {
    const float d1 = __fmul_rn(-cy, __fsub_rn(fE<NR>(st, 2, y, z), fE<NR>(st, 2, y - 1, z)));
    const float d2 = __fmul_rn(cz, __fsub_rn(fE<NR>(st, 1, y, z), fE<NR>(st, 1, y, z - 1)));
    v = fused_hnode<3, ABS>(p, fa, fHx<NR>(st, y, z), 0.f, d1, d2, slab, idx, si, false);
  }
  fN<NR>(hn, w == 0 ? 2 : w == 2 ? 1 : 0, y, z) = ok ? v : 0.f;
}

// New E of plane i on the own nodes.  ep: old E (registers), hn: new H of
// plane i (shared), hc: new H of plane i + 1 (own nodes).
//   MODE 1: uniform non-dispersive material um
//   MODE 0: general (mixed materials, dispersive nodes left to the ADE pass,
//           design region)
// AXM: the slab axes of the tile-plane (0: no absorber).
template <int NR, int MODE, int AXM>
__device__ __forceinline__ void fused_e_own(const Params& p, const FusedArgs& fa, const float* st, const float* hn,
                                            const MatShared& ms, int um, int i, int j0, int k0, const bool (&ok)[NR],
                                            const float (&ep)[NR][3], const float (&hc)[NR][3], const float* fco, int xs,
                                            const int (&ys)[NR], int zs) {
  const int lane = threadIdx.x, w = threadIdx.y;
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  float iu[3] = {1.f, 1.f, 1.f};
  if (MODE != 0) { iu[0] = ms.inv_eps[um][0]; iu[1] = ms.inv_eps[um][1]; iu[2] = ms.inv_eps[um][2]; }
  const long long pb = (long long)i * p.g.sx;
  int si[NR][3];
  float old[NR][3][2];
  if (AXM) {
#pragma unroll
    for (int r = 0; r < NR; r++) {
      fused_slabs<AXM>(p, i, j0 + w + TW * r, k0 + lane, xs, ys[r], zs, si[r]);
      if (!ok[r]) si[r][0] = si[r][1] = si[r][2] = -1;
      fused_aux_load<AXM, false>(p, fa, si[r], old[r]);
    }
  }
#pragma unroll
  for (int r = 0; r < NR; r++) {
    if (!ok[r]) continue;
    const int y = w + TW * r, j = j0 + y, k = k0 + lane;
    const long long off = pb + (long long)j * p.g.sy + k;
    const float hx = fN<NR>(hn, 0, y, lane), hy = fN<NR>(hn, 1, y, lane), hz = fN<NR>(hn, 2, y, lane);
    // Ex += dt/eps(dy Hz - dz Hy); Ey += dt/eps(dz Hx - dx Hz); Ez += dt/eps(dx Hy - dy Hx)
    float d[3][3];
    d[0][0] = 0.f;
    d[0][1] = __fmul_rn(cy, __fsub_rn(fN<NR>(hn, 2, y + 1, lane), hz));
    d[0][2] = __fmul_rn(-cz, __fsub_rn(fN<NR>(hn, 1, y, lane + 1), hy));
    d[1][0] = __fmul_rn(-cx, __fsub_rn(hc[r][2], hz));
    d[1][1] = 0.f;
    d[1][2] = __fmul_rn(cz, __fsub_rn(fN<NR>(hn, 0, y, lane + 1), hx));
    d[2][0] = __fmul_rn(cx, __fsub_rn(hc[r][1], hy));
    d[2][1] = __fmul_rn(-cy, __fsub_rn(fN<NR>(hn, 0, y + 1, lane), hx));
    d[2][2] = 0.f;
    const bool slab = AXM && (si[r][0] & si[r][1] & si[r][2]) >= 0;
    const float* fx = fco + FCO_X + (i - p.x0 - blockIdx.z * p.xchunk + 1) * 6;
    const float* fy = fco + FCO_Y + y * 6;
    const float* fz = fco + FCO_Z + lane * 6;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float ie = iu[c];
      if (MODE == 0) {
        const int m = um >= 0 ? um : fM<NR>(st, c, y, lane);
        if (ms.npoles[m] > 0) continue;              // dispersive node: the ADE pass writes it
        ie = ms.inv_eps[m][c];
        if (p.des_on) {
          const long long di = design_index(p, i, j, k);
          if (di >= 0) ie = p.des_ie[c][di];
        }
      }
      d[c][0] = __fmul_rn(d[c][0], ie); d[c][1] = __fmul_rn(d[c][1], ie); d[c][2] = __fmul_rn(d[c][2], ie);
      float inc = sum3(d[c][0], d[c][1], d[c][2]);
      if (slab) {
        if (c == 0) inc = __fadd_rn(inc, fused_aux_apply<0, AXM>(p, fa, si[r], old[r], d[0], fx, fy, fz, true));
        else if (c == 1) inc = __fadd_rn(inc, fused_aux_apply<1, AXM>(p, fa, si[r], old[r], d[1], fx, fy, fz, true));
        else inc = __fadd_rn(inc, fused_aux_apply<2, AXM>(p, fa, si[r], old[r], d[2], fx, fy, fz, true));
      }
      fa.dst[c][off] = __fadd_rn(ep[r][c], inc);
    }
  }
}

// Issue the copies of stage s (plane x0 - 1 + s; the material tiles of the
// plane before it, whose E update runs while this stage is current).
template <int NR>
__device__ __forceinline__ void fused_issue(const FusedMaps& m, float* st, uint64_t* bar, int ip, int j0, int k0,
                                            bool want_mat) {
  mbar_arrive_expect_tx(bar, FL<NR>::BYTES + (want_mat ? FL<NR>::BYTES_MAT : 0u));
#pragma unroll
  for (int c = 0; c < 3; c++) tma_load_3d(st + c * FL<NR>::FE_N, &m.e[c], k0 - 4, j0 - 1, ip, bar);
  tma_load_3d(st + FL<NR>::OFF_HX, &m.hx, k0, j0, ip, bar);
  tma_load_3d(st + FL<NR>::OFF_HY, &m.hy, k0, j0, ip, bar);
  tma_load_3d(st + FL<NR>::OFF_HZ, &m.hz, k0, j0, ip, bar);
  if (want_mat)
#pragma unroll
    for (int c = 0; c < 3; c++)
      tma_load_3d(reinterpret_cast<uint8_t*>(st + FL<NR>::OFF_M) + c * F_MROWS * TZ, &m.mat[c], k0, j0, ip - 1, bar);
}

// H of plane i over the own nodes for the tile-plane's slab axes m (bit 0: x
// slab plane, bit 1: y slab rows, bit 2: z slab columns).  Tile-planes with
// any slab take one general variant: variants per slab combination were
// measured slower on every workload (a larger kernel).
template <int NR>
__device__ __forceinline__ void fused_h_dispatch(int m, const Params& p, const FusedArgs& fa, const float* st, float* hn,
                                                 int i, int j0, int k0, bool store, const bool (&ok)[NR],
                                                 const float (&ep)[NR][3], float (&hc)[NR][3], float (&ec)[NR][3],
                                                 const float* fco, int xs, const int (&ys)[NR], int zs) {
  switch (m) {
    case 0: fused_h_own<NR, 0>(p, fa, st, hn, i, j0, k0, store, ok, ep, hc, ec, fco, xs, ys, zs); break;
    default: fused_h_own<NR, 7>(p, fa, st, hn, i, j0, k0, store, ok, ep, hc, ec, fco, xs, ys, zs); break;
  }
}
template <int NR, int MODE>
__device__ __forceinline__ void fused_e_dispatch(int m, const Params& p, const FusedArgs& fa, const float* st,
                                                 const float* hn, const MatShared& ms, int um, int i, int j0, int k0,
                                                 const bool (&ok)[NR], const float (&ep)[NR][3], const float (&hc)[NR][3],
                                                 const float* fco, int xs, const int (&ys)[NR], int zs) {
  switch (m) {
    case 0: fused_e_own<NR, MODE, 0>(p, fa, st, hn, ms, um, i, j0, k0, ok, ep, hc, fco, xs, ys, zs); break;
    default: fused_e_own<NR, MODE, 7>(p, fa, st, hn, ms, um, i, j0, k0, ok, ep, hc, fco, xs, ys, zs); break;
  }
}

// 3 CTAs per SM (shared memory: a 3-stage ring and two new-H planes)
template <int NR>
__global__ void __launch_bounds__(NTHR, NR == 2 ? 3 : 4)
    fused_kernel(const __grid_constant__ Params p, const __grid_constant__ FusedArgs fa,
                 const __grid_constant__ FusedMaps m) {
  extern __shared__ __align__(128) float fsm[];
  float* hnb = fsm + F_NST * FL<NR>::STAGE;                      // two new-H planes
  MatShared& ms = *reinterpret_cast<MatShared*>(hnb + 2 * FL<NR>::HN);
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(&ms) + sizeof(MatShared));
  __shared__ signed char umc[FX_MAX];
  __shared__ float fco[FCO_N];
  __shared__ int gave_up;
  const int lane = threadIdx.x, w = threadIdx.y, tid = w * TZ + lane;
  const int k0 = blockIdx.x * TZ, j0 = blockIdx.y * FL<NR>::TY;
  const int x0 = p.x0 + blockIdx.z * p.xchunk;
  const int x1 = min(x0 + p.xchunk, p.x1);
  const int len = x1 - x0;
  const int slast = len + 1;                               // stages 0 .. len + 1: planes x0 - 1 .. x1
  const bool cpml = p.ab.kind == 1;
  if (tid == 0) {
    for (int q = 0; q < F_NST; q++) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    gave_up = 0;
  }
  load_matshared(ms, p);
  for (int q = tid; q < len; q += NTHR)
    umc[q] = __ldg(p.umat + ((long long)(x0 + q) * p.nty + j0 / F_MROWS) * p.ntz + blockIdx.x);
  if (cpml)
    for (int q = tid; q < FCO_N / 6; q += NTHR) {
      // row q: x plane x0 - 1 + q, y row j0 + q - (FX_MAX + 2), z column k0 + q - (FX_MAX + F_MROWS + 3)
      const int a = q < FX_MAX + 2 ? 0 : q < FX_MAX + F_MROWS + 3 ? 1 : 2;
      const int v = a == 0 ? x0 - 1 + q : a == 1 ? j0 + q - (FX_MAX + 2) : k0 + q - (FX_MAX + F_MROWS + 3);
#pragma unroll
      for (int o = 0; o < 2; o++) {
        const int h = 2 * v + o;
        const bool in = h >= 0 && h < 2 * p.g.n[a] + 2;
        fco[q * 6 + 3 * o + 0] = in ? __ldg(p.ab.c0[a] + h) : 1.f;
        fco[q * 6 + 3 * o + 1] = in ? __ldg(p.ab.c1[a] + h) : 0.f;
        fco[q * 6 + 3 * o + 2] = in ? __fsub_rn(__ldg(p.ab.c2[a] + h), 1.f) : 0.f;
      }
    }
  __syncthreads();
  auto issue = [&](int s) {
    const int ip = x0 - 1 + s;
    fused_issue<NR>(m, fsm + (s % F_NST) * FL<NR>::STAGE, &bars[s % F_NST], ip, j0, k0, ip - 1 >= x0 && umc[ip - 1 - x0] < 0);
  };
  int issued = -1;
  if (tid == 0)
    for (int s = 0; s < F_NST && s <= slast; s++) { issue(s); issued = s; }
  // per-thread constants of the walk
  bool ok[NR];
  int ys[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) {
    ok[r] = j0 + w + TW * r < p.g.n[1] && k0 + lane < p.g.n[2];
    ys[r] = cpml ? slab_cs(p, 1, j0 + w + TW * r) : -1;
  }
  const int zs = cpml ? slab_cs(p, 2, k0 + lane) : -1;
  // slab axes of the own nodes (y, z: fixed for the walk) and of the halo (row 16, column 32)
  const int myz = cpml ? ((j0 < p.ab.L[1][0] || j0 + FL<NR>::TY > p.g.n[1] - p.ab.L[1][1]) ? 2 : 0) |
                             ((k0 < p.ab.L[2][0] || k0 + TZ > p.g.n[2] - p.ab.L[2][1]) ? 4 : 0)
                       : 0;
  const bool halo_yz = cpml && (j0 < p.ab.L[1][0] || j0 + FL<NR>::TY + 1 > p.g.n[1] - p.ab.L[1][1] || k0 < p.ab.L[2][0] ||
                                k0 + TZ + 1 > p.g.n[2] - p.ab.L[2][1]);
  float ep[NR][3], hc[NR][3], ec[NR][3];
  float xe = 0.f;
  // stage 0 (plane x0 - 1): the old E of the own nodes and of the halo nodes (x taps)
  if (tid == 0 && !mbar_wait(&bars[0], 0u, p.err, p.wait_limit)) gave_up = 1;
  __syncthreads();
  int t = 0, swait = 0;                                    // swait: the stage waited for last
  if (!gave_up) {
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
      for (int c = 0; c < 3; c++) ep[r][c] = fE<NR>(fsm, c, w + TW * r, lane);
    if (w == 0) xe = fE<NR>(fsm, 1, FL<NR>::TY, lane);
    else if (w == 2 && lane < FL<NR>::TY) xe = fE<NR>(fsm, 2, lane, TZ);
    for (; t <= len; t++) {
      const int s = t + 1, pc = x0 + t;
      swait = s;
      if (tid == 0 && !mbar_wait(&bars[s % F_NST], (unsigned)((s / F_NST) & 1), p.err, p.wait_limit)) gave_up = 1;
      // every thread is past iteration t - 1: the slot of stage t and the new-H
      // plane written two iterations ago are free
      __syncthreads();
      if (gave_up) break;
      if (tid == 0 && t + F_NST <= slast) { issue(t + F_NST); issued = t + F_NST; }
      const float* st = fsm + (s % F_NST) * FL<NR>::STAGE;
      float* hn1 = hnb + (t & 1) * FL<NR>::HN;                   // new H of plane pc
      const float* hn0 = hnb + ((t + 1) & 1) * FL<NR>::HN;       // new H of plane pc - 1
      if (pc < p.g.n[0]) {
        const int xs = cpml ? slab_cs(p, 0, pc) : -1;
        fused_h_dispatch<NR>(myz | (xs >= 0 ? 1 : 0), p, fa, st, hn1, pc, j0, k0, t < len, ok, ep, hc, ec, fco, xs, ys, zs);
        if (halo_yz || xs >= 0) fused_h_halo<NR, true>(p, fa, st, hn1, pc, j0, k0, xe);
        else fused_h_halo<NR, false>(p, fa, st, hn1, pc, j0, k0, xe);
      } else {
        // beyond the last plane of the grid: H is zero there
#pragma unroll
        for (int r = 0; r < NR; r++)
#pragma unroll
          for (int c = 0; c < 3; c++) { hc[r][c] = 0.f; ec[r][c] = 0.f; }
      }
      if (t >= 1) {
        const int pe = pc - 1;
        const int um = umc[pe - x0];
        const int xs = cpml ? slab_cs(p, 0, pe) : -1;
        const int mm = myz | (xs >= 0 ? 1 : 0);
        if (um >= 0) fused_e_dispatch<NR, 1>(mm, p, fa, st, hn0, ms, um, pe, j0, k0, ok, ep, hc, fco, xs, ys, zs);
        else fused_e_dispatch<NR, 0>(mm, p, fa, st, hn0, ms, um, pe, j0, k0, ok, ep, hc, fco, xs, ys, zs);
      }
#pragma unroll
      for (int r = 0; r < NR; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) ep[r][c] = ec[r][c];
    }
  }
  if (gave_up && tid == 0) {
    // a wait gave up: no further copies were issued; wait (bounded) for those in flight, then leave
    for (int s = swait; s <= issued; s++) mbar_wait(&bars[s % F_NST], (unsigned)((s / F_NST) & 1), nullptr, DRAIN_POLLS);
  }
}

}  // namespace dtmx
