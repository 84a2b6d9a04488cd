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
// Tile: a CTA owns 15 y rows x 32 z columns of an x chunk, walked upwards.
// Its 8 warps compute the new H on 16 rows (the 15 own rows and the halo row
// above), 32 lanes per row; the halo column beyond the tile (Hy and Hx of
// z = k0+32, needed by the E update of the last lane) is shared out over the
// warps.  For plane i of the walk:
//   H(i+1) on the 16 x 33 region  <- E_old(i+1), E_old(i) (staged), H_old(i+1)
//   E(i)   on the 15 x 32 tile    <- E_old(i), H(i) and H(i+1) (shared memory)
// One thread issues the TMA copies (cp.async.bulk.tensor, no multicast) of each
// plane's E (17 rows: the row below the tile for the H taps), old H (16 rows)
// and, on mixed planes, material tiles into a 3-stage ring; the new H of two
// planes sits in a shared-memory double buffer.  Everything outside the grid
// reads as zero (TMA fill, or forced for the new H), which is the box
// geometry; other geometries use the per-step engine.
//
// The node updates are the expressions of plane_update (dtmx_device.cuh), in
// the same order with the same explicitly rounded operations, so without a
// TF/SF source this engine's fields are bit-identical to the per-step
// engine's.  With one, the H correction is added to the old H before the sweep
// (the update is linear in it), which rounds differently at the box faces.
#pragma once
#include "dtmx_stream.cuh"

namespace dtmx {

constexpr int FZ = 32;                      // tile columns (lanes)
constexpr int FW = 8;                       // warps
constexpr int FTY = 15;                     // own rows of a tile
constexpr int FHR = 16;                     // rows with a new H: own + the halo row
constexpr int FNTHR = FZ * FW;
constexpr int FROW = 40;                    // staged row: z in [k0-4, k0+36), 16-byte aligned
constexpr int FZO = 4;                      // z offset of k0 in a staged row
constexpr int FE_ROWS = FHR + 1;            // E rows j0-1 .. j0+15
constexpr int FH_ROWS = FHR;                // old H rows j0 .. j0+15
constexpr int FE_N = 704;                   // 17 x 40 = 680 floats, rounded to 128 bytes
constexpr int FH_N = 640;                   // 16 x 40
constexpr int FM_N = 3 * FHR * FZ / 4;      // material tiles (bytes as floats): 3 x 16 x 32
constexpr int F_OFF_E = 0, F_OFF_H = 3 * FE_N, F_OFF_M = F_OFF_H + 3 * FH_N;
constexpr int F_STAGE = F_OFF_M + FM_N;     // 4416 floats = 17664 bytes (138 x 128)
constexpr unsigned F_BYTES = (3 * FE_ROWS * FROW + 3 * FH_ROWS * FROW) * 4;
constexpr unsigned F_BYTES_MAT = 3 * FHR * FZ;
constexpr int F_NST = 3;
constexpr int HN_P = 33;                    // new-H row pitch: z in [k0, k0+33)
constexpr int HN_N = FHR * HN_P;            // per component
constexpr int F_HN = ((3 * HN_N + 31) / 32) * 32;
constexpr size_t F_SMEM_BYTES = (size_t)(F_NST * F_STAGE + 2 * F_HN) * 4 + sizeof(MatShared) + F_NST * 8 + 128;

// TMA descriptors of one buffer set: E tiles (40 x 17) and old H tiles (40 x 16)
struct FusedMaps {
  CUtensorMap e[3];
  CUtensorMap h[3];
  CUtensorMap mat[3];                       // 32 x 16 material tiles (rows j0 .. j0+15)
};

// Per-launch arguments beyond Params (which describes the source buffer A)
struct FusedArgs {
  float* dst[6];                            // buffer B
  float* hsrc[3][2];                        // CPML auxiliaries of H (slots 2, 3) in A
  float* hdst[3][2];                        // ... and in B
  const signed char* umat;                  // uniform material per (plane, 15-row tile, z tile)
  int nty, ntz;
};

// CPML correction of component c at a slab node (absorb_apply3 with the H
// auxiliaries read from A and written to B; E auxiliaries in place).
template <bool STORE>
__device__ __forceinline__ float fused_absorb(const Params& p, const FusedArgs& fa, int c, const int (&idx)[3],
                                              const int (&si)[3], const float* dif) {
  float corr = 0.f;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int sl = slot_of(c, a);
    if (sl < 0 || si[a] < 0) continue;
    const float* src = c >= 3 ? fa.hsrc[a][sl - 2] : p.ab.aux[a][sl];
    const float old = src[si[a]];
    const int h = 2 * idx[a] + comp_off(c, a);
    const float k0 = __ldg(p.ab.c0[a] + h), k1 = __ldg(p.ab.c1[a] + h);
    const float nv = __fmaf_rn(k0, old, __fmul_rn(k1, dif[a]));
    if (STORE) (c >= 3 ? fa.hdst[a][sl - 2] : p.ab.aux[a][sl])[si[a]] = nv;
    corr = __fadd_rn(corr, __fmaf_rn(__fsub_rn(__ldg(p.ab.c2[a] + h), 1.f), dif[a], nv));
  }
  return corr;
}

// staged-tile accessors: E rows y in [-1, 15], old H rows y in [0, 15], z in [-4, 35]
__device__ __forceinline__ float fE(const float* st, int c, int y, int z) {
  return st[F_OFF_E + c * FE_N + (y + 1) * FROW + z + FZO];
}
__device__ __forceinline__ float fH(const float* st, int c, int y, int z) {
  return st[F_OFF_H + c * FH_N + y * FROW + z + FZO];
}
__device__ __forceinline__ int fM(const float* st, int c, int y, int z) {
  return reinterpret_cast<const uint8_t*>(st + F_OFF_M)[c * FHR * FZ + y * FZ + z];
}

// New H of component hc (3..5) at tile node (y, z) of plane i (stage cur, plane
// i-1 in stage prv): the H expressions of plane_update, H taps at -1..0.
// CPML slab nodes add the absorber correction (ABS).
template <bool ABS, bool STORE>
__device__ __forceinline__ float fused_h(const Params& p, const FusedArgs& fa, const float* cur, const float* prv,
                                         int hc, int y, int z, int i, int j, int k) {
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  float d[3];
  if (hc == 3) {        // Hx -= dt (dy Ez - dz Ey)
    d[0] = 0.f;
    d[1] = __fmul_rn(-cy, __fsub_rn(fE(cur, 2, y, z), fE(cur, 2, y - 1, z)));
    d[2] = __fmul_rn(cz, __fsub_rn(fE(cur, 1, y, z), fE(cur, 1, y, z - 1)));
  } else if (hc == 4) { // Hy -= dt (dz Ex - dx Ez)
    d[0] = __fmul_rn(cx, __fsub_rn(fE(cur, 2, y, z), fE(prv, 2, y, z)));
    d[1] = 0.f;
    d[2] = __fmul_rn(-cz, __fsub_rn(fE(cur, 0, y, z), fE(cur, 0, y, z - 1)));
  } else {              // Hz -= dt (dx Ey - dy Ex)
    d[0] = __fmul_rn(-cx, __fsub_rn(fE(cur, 1, y, z), fE(prv, 1, y, z)));
    d[1] = __fmul_rn(cy, __fsub_rn(fE(cur, 0, y, z), fE(cur, 0, y - 1, z)));
    d[2] = 0.f;
  }
  float inc = sum3(d[0], d[1], d[2]);
  if (ABS) {
    int si[3];
    if (node_slabs(p, i, j, k, si)) {
      const int idx[3] = {i, j, k};
      inc = __fadd_rn(inc, fused_absorb<STORE>(p, fa, hc, idx, si, d));
    }
  }
  return __fadd_rn(fH(cur, hc - 3, y, z), inc);
}

// New H of plane i over the 16 x 33 region into hn (and the own nodes into B).
// cur: stage of plane i, prv: stage of plane i-1.  Values outside the grid are
// zero; STORE_B: plane i belongs to this chunk.
template <bool ABS>
__device__ __forceinline__ void fused_h_plane(const Params& p, const FusedArgs& fa, const float* cur, const float* prv,
                                              float* hn, int i, int j0, int k0, bool store_b) {
  const int lane = threadIdx.x, w = threadIdx.y;
  const int k = k0 + lane;
  const bool in_x = i < p.g.n[0];
  const long long pb = (long long)i * p.g.sx;
#pragma unroll
  for (int r = 0; r < 2; r++) {
    const int y = w + FW * r, j = j0 + y;
    const bool ok = in_x && j < p.g.n[1] && k < p.g.n[2];
    const bool own = y < FTY && store_b && ok;
    const long long off = pb + (long long)j * p.g.sy + k;
#pragma unroll
    for (int hc = 3; hc < 6; hc++) {
      float v = 0.f;
      if (ok) {
        v = own ? fused_h<ABS, true>(p, fa, cur, prv, hc, y, lane, i, j, k)
                : fused_h<ABS, false>(p, fa, cur, prv, hc, y, lane, i, j, k);
        if (own) fa.dst[hc][off] = v;
      }
      hn[(hc - 3) * HN_N + y * HN_P + lane] = v;
    }
  }
  // the halo column z = k0+32: Hy on rows 0-14 by warps 0-3, Hx by warps 4-7 (lanes 0-3)
  {
    const int hc = w < 4 ? 4 : 3;
    const int y = (w & 3) * 4 + lane;
    if (lane < 4 && y < FTY) {
      const int j = j0 + y, kk = k0 + FZ;
      const bool ok = in_x && j < p.g.n[1] && kk < p.g.n[2];
      hn[(hc - 3) * HN_N + y * HN_P + FZ] = ok ? fused_h<ABS, false>(p, fa, cur, prv, hc, y, FZ, i, j, kk) : 0.f;
    }
  }
}

// New E of plane i on the own nodes: the E expressions of plane_update, E taps
// at 0..+1, from the new H of planes i (h0) and i+1 (h1).
//   MODE 1: uniform non-dispersive material um, no absorber
//   MODE 2: uniform material um, absorber slabs in the tile
//   MODE 0: general (mixed materials, dispersive nodes left to the ADE pass,
//           design region, absorber)
template <int MODE>
__device__ __forceinline__ void fused_e_plane(const Params& p, const FusedArgs& fa, const float* cur, const float* h0,
                                              const float* h1, const MatShared& ms, int um, int i, int j0, int k0) {
  const int lane = threadIdx.x, w = threadIdx.y;
  const int k = k0 + lane;
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  if (i >= p.g.n[0] || k >= p.g.n[2]) return;
  float iu[3] = {1.f, 1.f, 1.f};
  if (MODE != 0) { iu[0] = ms.inv_eps[um][0]; iu[1] = ms.inv_eps[um][1]; iu[2] = ms.inv_eps[um][2]; }
  const long long pb = (long long)i * p.g.sx;
#pragma unroll
  for (int r = 0; r < 2; r++) {
    const int y = w + FW * r, j = j0 + y;
    if (y >= FTY || j >= p.g.n[1]) continue;
    const long long off = pb + (long long)j * p.g.sy + k;
    const float* hx = h0;
    const float* hy = h0 + HN_N;
    const float* hz = h0 + 2 * HN_N;
    const int q = y * HN_P + lane;
    float d[3][3];
    // Ex += dt/eps (dy Hz - dz Hy); Ey += dt/eps (dz Hx - dx Hz); Ez += dt/eps (dx Hy - dy Hx)
    d[0][0] = 0.f;
    d[0][1] = __fmul_rn(cy, __fsub_rn(hz[q + HN_P], hz[q]));
    d[0][2] = __fmul_rn(-cz, __fsub_rn(hy[q + 1], hy[q]));
    d[1][0] = __fmul_rn(-cx, __fsub_rn(h1[2 * HN_N + q], hz[q]));
    d[1][1] = 0.f;
    d[1][2] = __fmul_rn(cz, __fsub_rn(hx[q + 1], hx[q]));
    d[2][0] = __fmul_rn(cx, __fsub_rn(h1[HN_N + q], hy[q]));
    d[2][1] = __fmul_rn(-cy, __fsub_rn(hx[q + HN_P], hx[q]));
    d[2][2] = 0.f;
    int si[3] = {-1, -1, -1};
    const bool ab = (MODE != 1) && p.ab.kind != 0 && node_slabs(p, i, j, k, si);
    const int idx3[3] = {i, j, k};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float F = fE(cur, c, y, lane);
      float ie = iu[c];
      if (MODE == 0) {
        const int m = um >= 0 ? um : fM(cur, c, y, lane);
        if (ms.npoles[m] > 0) continue;               // dispersive node: the ADE pass writes it
        ie = ms.inv_eps[m][c];
        if (p.des_on) {
          const long long di = design_index(p, i, j, k);
          if (di >= 0) ie = p.des_ie[c][di];
        }
      }
      d[c][0] = __fmul_rn(d[c][0], ie); d[c][1] = __fmul_rn(d[c][1], ie); d[c][2] = __fmul_rn(d[c][2], ie);
      float inc = sum3(d[c][0], d[c][1], d[c][2]);
      if (ab) inc = __fadd_rn(inc, fused_absorb<true>(p, fa, c, idx3, si, d[c]));
      fa.dst[c][off] = __fadd_rn(F, inc);
    }
  }
}

// Issue the copies of plane ip into a stage (one thread).
__device__ __forceinline__ void fused_stage(const FusedMaps& m, float* st, uint64_t* bar, int ip, int j0, int k0,
                                            bool want_mat) {
  mbar_arrive_expect_tx(bar, F_BYTES + (want_mat ? F_BYTES_MAT : 0u));
#pragma unroll
  for (int c = 0; c < 3; c++) tma_load_3d(st + F_OFF_E + c * FE_N, &m.e[c], k0 - FZO, j0 - 1, ip, bar);
#pragma unroll
  for (int c = 0; c < 3; c++) tma_load_3d(st + F_OFF_H + c * FH_N, &m.h[c], k0 - FZO, j0, ip, bar);
  if (want_mat)
#pragma unroll
    for (int c = 0; c < 3; c++)
      tma_load_3d(reinterpret_cast<uint8_t*>(st + F_OFF_M) + c * FHR * FZ, &m.mat[c], k0, j0, ip, bar);
}

// the plane's absorber test over the region whose new H the CTA computes (y
// up to j0+15, z up to k0+32) -- a superset of the E tile
__device__ __forceinline__ bool fused_tile_abs(const Params& p, int i, int j0, int k0) {
  if (p.ab.kind == 0) return false;
  return in_slab(p, 0, i) || j0 < p.ab.L[1][0] || j0 + FHR > p.g.n[1] - p.ab.L[1][1] || k0 < p.ab.L[2][0] ||
         k0 + FZ + 1 > p.g.n[2] - p.ab.L[2][1];
}

// 3 CTAs per SM (68 KB of shared memory each)
__global__ void __launch_bounds__(FNTHR, 3)
    fused_kernel(const __grid_constant__ Params p, const __grid_constant__ FusedArgs fa,
                 const __grid_constant__ FusedMaps m) {
  extern __shared__ __align__(128) float fsm[];
  float* hnb = fsm + F_NST * F_STAGE;                      // two new-H planes
  MatShared& ms = *reinterpret_cast<MatShared*>(hnb + 2 * F_HN);
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(&ms) + sizeof(MatShared));
  __shared__ int gave_up;
  const int lane = threadIdx.x, w = threadIdx.y, tid = w * FZ + lane;
  const int k0 = blockIdx.x * FZ, ty = blockIdx.y, j0 = ty * FTY;
  const int x0 = p.x0 + blockIdx.z * p.xchunk;
  const int x1 = min(x0 + p.xchunk, p.x1);
  const int len = x1 - x0;
  // stage number s holds plane x0 - 1 + s; planes x0-1 .. x1 (len + 2 stages)
  const int slast = len + 1;
  auto umat = [&](int ip) -> int {
    return (ip >= 0 && ip < p.g.n[0]) ? (int)__ldg(fa.umat + ((long long)ip * fa.nty + ty) * fa.ntz + blockIdx.x) : 0;
  };
  if (tid == 0) {
    for (int q = 0; q < F_NST; q++) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    gave_up = 0;
  }
  load_matshared(ms, p);
  __syncthreads();
  if (tid == 0)
    for (int s = 0; s <= 2 && s <= slast; s++) {
      const int ip = x0 - 1 + s;
      fused_stage(m, fsm + (s % F_NST) * F_STAGE, &bars[s % F_NST], ip, j0, k0, ip >= x0 && ip < x1 && umat(ip) < 0);
    }
  // prologue: the new H of plane x0 (needs planes x0-1 and x0)
  const bool ok = mbar_wait(&bars[0], 0u, p.err, p.wait_limit) && mbar_wait(&bars[1], 0u, p.err, p.wait_limit);
  if (__syncthreads_or(!ok)) gave_up = 1;
  int issued = min(2, slast);
  if (!gave_up) {
    const float* prv = fsm;
    const float* cur = fsm + F_STAGE;
    if (fused_tile_abs(p, x0, j0, k0)) fused_h_plane<true>(p, fa, cur, prv, hnb, x0, j0, k0, true);
    else fused_h_plane<false>(p, fa, cur, prv, hnb, x0, j0, k0, true);
  }
  for (int t = 0; t < len && !gave_up; t++) {
    const int i = x0 + t;
    // the stage of plane i+1 (every thread waits: the barrier phase completes for all at once)
    const int sw = t + 2;
    const bool got = mbar_wait(&bars[sw % F_NST], (unsigned)((sw / F_NST) & 1), p.err, p.wait_limit);
    // every thread is past step t-1 here: the stage of plane i-1 and new-H buffer t+1 are free
    if (__syncthreads_or(!got)) { gave_up = 1; break; }
    const int s_next = t + 3;                               // stage of plane i+2
    if (tid == 0 && s_next <= slast) {
      const int ip = x0 - 1 + s_next;
      fused_stage(m, fsm + (s_next % F_NST) * F_STAGE, &bars[s_next % F_NST], ip, j0, k0, ip < x1 && umat(ip) < 0);
      issued = s_next;
    }
    const float* sti = fsm + ((t + 1) % F_NST) * F_STAGE;  // plane i
    const float* st1 = fsm + (sw % F_NST) * F_STAGE;       // plane i+1
    const float* h0 = hnb + (t & 1) * F_HN;                 // new H of plane i
    float* h1 = hnb + ((t + 1) & 1) * F_HN;                 // new H of plane i+1
    // new H of plane i+1 (stored to B only when the chunk owns it)
    if (fused_tile_abs(p, i + 1, j0, k0)) fused_h_plane<true>(p, fa, st1, sti, h1, i + 1, j0, k0, i + 1 < x1);
    else fused_h_plane<false>(p, fa, st1, sti, h1, i + 1, j0, k0, i + 1 < x1);
    __syncthreads();
    const int um = umat(i);
    const bool eab = p.ab.kind != 0 && (in_slab(p, 0, i) || j0 < p.ab.L[1][0] || j0 + FTY > p.g.n[1] - p.ab.L[1][1] ||
                                        k0 < p.ab.L[2][0] || k0 + FZ > p.g.n[2] - p.ab.L[2][1]);
    if (um >= 0 && !eab) fused_e_plane<1>(p, fa, sti, h0, h1, ms, um, i, j0, k0);
    else if (um >= 0) fused_e_plane<2>(p, fa, sti, h0, h1, ms, um, i, j0, k0);
    else fused_e_plane<0>(p, fa, sti, h0, h1, ms, um, i, j0, k0);
  }
  if (gave_up) {
    // a wait gave up: no further copies were issued; wait (bounded) for those in flight, then leave
    if (tid == 0)
      for (int s = max(0, issued - 2); s <= issued; s++)
        mbar_wait(&bars[s % F_NST], (unsigned)((s / F_NST) & 1), nullptr, DRAIN_POLLS);
  }
}

}  // namespace dtmx
