// dtmx_torre.cuh -- wavefront ("torre") engine: T time steps per launch with
// the working set held in L2.
//
// The reference advances DiamondTorre tiles (diamond.cu:72-273, window.hpp:
// 108-176): each CUDA block climbs a tower of time levels over a small x-t
// diamond so that a rag is loaded once for several steps.  On B200 the same
// temporal blocking is laid out as a wavefront along x: one persistent CTA
// owns one (y, z) tile column for the whole launch, and the 2T half-step
// levels of that column advance together, level l working on plane
// x = s - off[l] at wave step s.  The planes between the first and the last
// level (tens of MB for a 384^2 cross-section) stay in L2, so DRAM sees each
// field about once per launch instead of twice per step.
//
// Fields are updated in place.  A CTA reads the y/z halo rows of its
// neighbours' tiles; the level offsets are spaced so that, with each CTA
// loading step s only after its four neighbours have published step s-2,
// every halo it reads has been written at the right level and none has been
// overwritten by the next level (read-after-write: off[l] - off[l-1] >=
// reach_l + 2; write-after-read: off[l+1] - off[l] > back_l).  Completion of a
// wave step is published per tile with a release store after all of the
// step's field stores; the producer warp acquires its neighbours' counters,
// orders the async proxy after them (fence.proxy.async) and only then issues
// the TMA loads of the next step.  All tiles must be co-resident (cooperative
// launch); every wait is bounded and records a timeout in p.err.
//
// Within a CTA: one producer warp stages each level-plane item (source tiles
// with y/z halos, the three own components, the material tile and the two
// components whose x taps feed the register queues) into a ring of NS
// shared-memory stages by TMA; eight (TY/4) consumer warps compute, each
// thread four consecutive z nodes of one y row (float4 shared-memory reads,
// float4 global stores).  x taps come from per-level register queues that
// advance one plane per wave step.  Arithmetic is that of plane_update (same
// expressions in the same order), so the engine is bit-identical to the
// one-launch-per-half-step engine.
#pragma once
#include "dtmx_device.cuh"
#include "dtmx_stream.cuh"

namespace dtmx {

constexpr int TT_Z = 32;           // tile extent along z
constexpr int TT_NS = 5;           // stages in the ring
constexpr int TT_K = 2;            // wave steps a producer may run ahead of its slowest neighbour
constexpr int TT_NPUB = 4;         // step-completion barriers (> TT_K + 1)

struct TorreMaps {
  CUtensorMap A[2];     // Ex / Hx: 40 z x (TY + 2R-1) y    (y and z halo)
  CUtensorMap B[2];     // Ey / Hy: 40 z x TY y              (z halo)
  CUtensorMap C[2];     // Ez / Hz: 32 z x (TY + 2R-1) y    (y halo)
  CUtensorMap core[6];  // 32 z x TY y of every component
  CUtensorMap mat[3];   // 32 z x TY y material bytes
};

struct TorreArgs {
  int* ctr;             // [nty][ntz] completed wave steps of each tile
  int ntz, nty;
  int nsteps;           // wave steps of the launch
};

template <int ORDER>
struct TorreGeom {
  static constexpr int R = ORDER / 2;
  // forward (a) and backward (b) x reach of the taps: H reads E at -R..R-1,
  // E reads H at -(R-1)..R
  static constexpr int AH = R - 1, BH = R, AE = R, BE = R - 1;
  static constexpr int NQ = 2 * R;               // x taps per derivative
  // read-after-write with TT_K steps of prefetch: gap >= reach + TT_K + 1;
  // write-after-read: gap(l+1) - back(l) >= TT_K holds then as well
  static constexpr int GAP_H = AH + TT_K + 1, GAP_E = AE + TT_K + 1;
  __host__ __device__ static constexpr int off(int l) {
    // l even: H level, odd: E level; level 0 starts AH planes early so that
    // its first items can fill the x-tap queue
    return l == 0 ? AH : off(l - 1) + ((l & 1) ? GAP_E : GAP_H);
  }
};

template <int ORDER, int TY>
struct TorreLayout {
  static constexpr int R = ORDER / 2;
  static constexpr int R2 = 2 * R - 1;
  static constexpr int AW = 40, CW = 32;
  static constexpr int al(int b) { return (b + 127) / 128 * 128; }
  static constexpr int SZ_A = al(AW * (TY + R2) * 4);
  static constexpr int SZ_B = al(AW * TY * 4);
  static constexpr int SZ_C = al(CW * (TY + R2) * 4);
  static constexpr int SZ_Q = al(TT_Z * TY * 4);
  static constexpr int SZ_M = al(TT_Z * TY);
  static constexpr int O_A = 0, O_B = O_A + SZ_A, O_C = O_B + SZ_B, O_BQ = O_C + SZ_C, O_CQ = O_BQ + SZ_Q;
  static constexpr int O_OWN = O_CQ + SZ_Q, O_MAT = O_OWN + 3 * SZ_Q;
  static constexpr int STAGE = O_MAT + 3 * SZ_M;
  static constexpr int NCW = TY / 4;                       // consumer warps
  static constexpr int NTHR = 32 * (NCW + 2);              // + producer warp + publisher warp
  static constexpr size_t SMEM = (size_t)TT_NS * STAGE + sizeof(MatShared) + (2 * TT_NS + TT_NPUB) * 8 + TT_NS * 4 + 128;
  static constexpr unsigned BYTES_Q = 2u * TT_Z * TY * 4;
  static constexpr unsigned BYTES_SRC = (unsigned)(AW * (TY + R2) * 4 + AW * TY * 4 + CW * (TY + R2) * 4 + 3 * TT_Z * TY * 4);
  static constexpr unsigned BYTES_MAT = 3u * TT_Z * TY;
};

__device__ __forceinline__ int ld_acquire(const int* q) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(q) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* q, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;\n" ::"l"(q), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }
__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ float4 lds4(const float* q) { return *reinterpret_cast<const float4*>(q); }
__device__ __forceinline__ float f4(const float4& v, int j) { return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w; }

// Is item (s, l) live, and which plane does it work on?  Items with
// -reach <= x < 0 only feed the x-tap queue.
template <int ORDER>
__device__ __forceinline__ bool item_live(int s, int l, int nx, int& x) {
  using G = TorreGeom<ORDER>;
  x = s - G::off(l);
  const int a = (l & 1) ? G::AE : G::AH;
  return x >= -a && x < nx;
}

// Producer warp: wait until this tile and its four neighbours have completed
// at least `need` wave steps.  Lane q watches tile q; the five counters are
// read in parallel and a lane re-reads only while its cached value is short.
// Bounded: gives up after wait_limit/16 rounds (2^22) and records the timeout.
__device__ __forceinline__ bool wait_tiles(const Params& p, const TorreArgs& ta, int ty, int tz, int need, int& seen) {
  const int lane = threadIdx.x & 31;
  const int* c = nullptr;
  if (lane < 5) {
    const int dy = lane == 1 ? -1 : lane == 2 ? 1 : 0, dz = lane == 3 ? -1 : lane == 4 ? 1 : 0;
    const int y = ty + dy, z = tz + dz;
    if (y >= 0 && y < ta.nty && z >= 0 && z < ta.ntz) c = ta.ctr + y * ta.ntz + z;
  }
  if (!c) seen = 1 << 30;
  bool ok = true;
  for (long long it = 0;; it++) {
    if (seen < need) seen = ld_acquire(c);
    if (__all_sync(0xffffffffu, seen >= need)) break;
    if (it > (p.wait_limit >> 4)) {
      if (lane == 0) atomicExch(p.err, 2);
      ok = false;
      break;
    }
    __nanosleep(32);
  }
  __syncwarp();
  return ok;
}

template <int ORDER, int TY>
__device__ __forceinline__ void issue_item(const Params& p, const TorreMaps& m, unsigned char* stg, uint64_t* full,
                                           int l, int x, int y0, int z0, bool want_mat) {
  using L = TorreLayout<ORDER, TY>;
  using G = TorreGeom<ORDER>;
  const bool isH = !(l & 1);
  const int h = isH ? 0 : 1;
  const int cs = isH ? 0 : 3, cf = isH ? 3 : 0;
  const int YL = isH ? G::R : G::R - 1;
  const int a = isH ? G::AH : G::AE;
  unsigned bytes = L::BYTES_Q;
  if (x >= 0) bytes += L::BYTES_SRC + (want_mat ? L::BYTES_MAT : 0u);
  mbar_arrive_expect_tx(full, bytes);
  tma_load_3d(stg + L::O_BQ, &m.core[cs + 1], z0, y0, x + a, full);
  tma_load_3d(stg + L::O_CQ, &m.core[cs + 2], z0, y0, x + a, full);
  if (x < 0) return;
  tma_load_3d(stg + L::O_A, &m.A[h], z0 - 4, y0 - YL, x, full);
  tma_load_3d(stg + L::O_B, &m.B[h], z0 - 4, y0, x, full);
  tma_load_3d(stg + L::O_C, &m.C[h], z0, y0 - YL, x, full);
#pragma unroll
  for (int c = 0; c < 3; c++) tma_load_3d(stg + L::O_OWN + c * L::SZ_Q, &m.core[cf + c], z0, y0, x, full);
  if (want_mat)
#pragma unroll
    for (int c = 0; c < 3; c++) tma_load_3d(stg + L::O_MAT + c * L::SZ_M, &m.mat[c], z0, y0, x, full);
}

// Material of a torre tile plane: uniform non-dispersive material of all E
// nodes (>= 0) or -1, combined from the 16-row tiles of the per-plane table.
template <int TY>
__device__ __forceinline__ int torre_umat(const Params& p, int x, int ty, int tz) {
  int u = -2;
#pragma unroll
  for (int q = 0; q < TY / TYT; q++) {
    const int yt = ty * (TY / TYT) + q;
    if (yt >= p.nty) break;
    const int v = (int)__ldg(p.umat + ((long long)x * p.nty + yt) * p.ntz + tz);
    u = (u == -2 || u == v) ? v : -1;
  }
  return u < 0 ? -1 : u;
}

// derivative from the NQ taps of one node (order 4: v0..v3, order 2: v1, v2)
template <int ORDER>
__device__ __forceinline__ float dtap(float t0, float t1, float t2, float t3) {
  if (ORDER == 4) return dstencil<4>(t0, t1, t2, t3);
  return dstencil<2>(0.f, t0, t1, 0.f);
}

// New value of one component at the thread's four nodes.  d[a][e]: the signed,
// scaled derivative term along axis a (0 where the component has none).
template <int ORDER, bool ISH, int TY>
__device__ __forceinline__ void torre_store(const Params& p, const unsigned char* stg, int c, float (&d)[3][4], int x,
                                            int j, int y, int z, int z0, int um, bool general, const MatShared& ms,
                                            long long off0) {
  using L = TorreLayout<ORDER, TY>;
  const int cf = ISH ? 3 : 0;
  const float4 o4 = lds4(reinterpret_cast<const float*>(stg + L::O_OWN + c * L::SZ_Q) + y * TT_Z + z);
  float out[4];
  if (!general) {
#pragma unroll
    for (int e = 0; e < 4; e++) {
      if (!ISH) {
        const float iu = ms.inv_eps[um][c];
        d[0][e] = __fmul_rn(d[0][e], iu); d[1][e] = __fmul_rn(d[1][e], iu); d[2][e] = __fmul_rn(d[2][e], iu);
      }
      out[e] = __fadd_rn(f4(o4, e), sum3(d[0][e], d[1][e], d[2][e]));
    }
    *reinterpret_cast<float4*>(p.f[cf + c] + off0) = make_float4(out[0], out[1], out[2], out[3]);
    return;
  }
  // general node: partial tile, absorber slab, dispersive or mixed materials.
  // The slab auxiliaries of the four nodes are loaded together first.
  const bool inx = p.ab.kind != 0 && in_slab(p, 0, x);
  const uint8_t* smat = stg + L::O_MAT;
  float old[4][3];
  bool inab[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int k = z0 + z + e;
    inab[e] = j < p.g.n[1] && k < p.g.n[2] && node_in_absorber(p, inx, j, k);
    if (inab[e]) absorb_load(p, cf + c, x, j, k, old[e]);
  }
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int k = z0 + z + e;
    const float F = f4(o4, e);
    out[e] = F;
    if (j >= p.g.n[1] || k >= p.g.n[2]) continue;
    float dd[3] = {d[0][e], d[1][e], d[2][e]};
    if (!ISH) {
      const int m = um >= 0 ? um : (int)smat[c * L::SZ_M + y * TT_Z + z + e];
      if (ms.npoles[m] > 0) {
        const int bi = x - p.ade.lo[0], bj = j - p.ade.lo[1], bk = k - p.ade.lo[2];
        if (bi >= 0 && bi < p.ade.n[0] && bj >= 0 && bj < p.ade.n[1] && bk >= 0 && bk < p.ade.n[2]) {
          const long long ai = ((long long)bi * p.ade.n[1] + bj) * p.ade.n[2] + bk;
          out[e] = ade_update(p, c, m, ms.npoles[m], ai, sum3(dd[0], dd[1], dd[2]), F);
          continue;
        }
      }
      float ie = ms.inv_eps[m][c];
      if (p.des_on) {
        const long long di = design_index(p, x, j, k);
        if (di >= 0) ie = p.des_ie[c][di];
      }
      dd[0] = __fmul_rn(dd[0], ie); dd[1] = __fmul_rn(dd[1], ie); dd[2] = __fmul_rn(dd[2], ie);
    }
    float inc = sum3(dd[0], dd[1], dd[2]);
    if (inab[e]) inc = __fadd_rn(inc, absorb_apply(p, cf + c, x, j, k, dd, old[e]));
    out[e] = __fadd_rn(F, inc);
  }
  if (j < p.g.n[1] && z0 + z + 3 < p.g.n[2]) {
    *reinterpret_cast<float4*>(p.f[cf + c] + off0) = make_float4(out[0], out[1], out[2], out[3]);
  } else if (j < p.g.n[1]) {
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (z0 + z + e < p.g.n[2]) p.f[cf + c][off0 + e] = out[e];
  }
}

// One level-plane item of a consumer thread: push the new x taps, then (x >= 0)
// update its four nodes of the three components of the half step, one
// component at a time (Hx: dy C, dz B; Hy: dx C, dz A; Hz: dx B, dy A and the
// same pattern for E), each finished with one float4 store.
template <int ORDER, bool ISH, int TY>
__device__ __forceinline__ void torre_item(const Params& p, const unsigned char* stg, float (&qb)[ORDER][4],
                                           float (&qc)[ORDER][4], int x, int y0, int z0, int um, bool general,
                                           const MatShared& ms) {
  using L = TorreLayout<ORDER, TY>;
  using G = TorreGeom<ORDER>;
  constexpr int NQ = G::NQ;
  constexpr int YL = ISH ? G::R : G::R - 1;
  constexpr int o0 = ISH ? -G::R : -(G::R - 1);   // first tap offset
  constexpr int I1 = NQ > 1 ? 1 : 0, I2 = NQ > 2 ? 2 : NQ - 1, I3 = NQ - 1;
  const int t = threadIdx.x, w = t >> 5, ln = t & 31;
  const int y = w * 4 + (ln >> 3), z = (ln & 7) * 4;
  {
    const float4 nb = lds4(reinterpret_cast<const float*>(stg + L::O_BQ) + y * TT_Z + z);
    const float4 nc = lds4(reinterpret_cast<const float*>(stg + L::O_CQ) + y * TT_Z + z);
#pragma unroll
    for (int q = 0; q < NQ - 1; q++)
#pragma unroll
      for (int e = 0; e < 4; e++) { qb[q][e] = qb[q + 1][e]; qc[q][e] = qc[q + 1][e]; }
#pragma unroll
    for (int e = 0; e < 4; e++) { qb[NQ - 1][e] = f4(nb, e); qc[NQ - 1][e] = f4(nc, e); }
  }
  if (x < 0) return;
  const float* sA = reinterpret_cast<const float*>(stg + L::O_A);
  const float* sB = reinterpret_cast<const float*>(stg + L::O_B);
  const float* sC = reinterpret_cast<const float*>(stg + L::O_C);
  const float cx = p.cdt[0], cy = p.cdt[1], cz = p.cdt[2];
  // H -= dt curl E, E += dt/eps curl H: signed coefficients (negation is exact)
  const float cyp = ISH ? -cy : cy, czp = ISH ? -cz : cz, cxp = ISH ? -cx : cx;
  const int j = y0 + y;
  const long long off0 = (long long)x * p.g.sx + (long long)j * p.g.sy + z0 + z;
  constexpr int zb = 4 + o0;              // index of tap 0 of node e = 0 in a z window
  float d[3][4];
  // component 0 (Hx / Ex): +dy C, -dz B  (times sg)
  {
    float4 rC[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) rC[q] = lds4(sC + (y + YL + o0 + q) * L::CW + z);
    float wB[12];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const float4 v = lds4(sB + y * L::AW + z + 4 * q);
      wB[4 * q] = v.x; wB[4 * q + 1] = v.y; wB[4 * q + 2] = v.z; wB[4 * q + 3] = v.w;
    }
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float dyC = dtap<ORDER>(f4(rC[0], e), f4(rC[I1], e), f4(rC[I2], e), f4(rC[I3], e));
      const float dzB = dtap<ORDER>(wB[zb + e], wB[zb + e + 1], wB[zb + e + 2], wB[zb + e + 3 < 12 ? zb + e + 3 : 11]);
      d[0][e] = 0.f;
      d[1][e] = __fmul_rn(cyp, dyC);
      d[2][e] = __fmul_rn(-czp, dzB);
    }
    torre_store<ORDER, ISH, TY>(p, stg, 0, d, x, j, y, z, z0, um, general, ms, off0);
  }
  // component 1 (Hy / Ey): -dx C, +dz A  (times sg)
  {
    float wA[12];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const float4 v = lds4(sA + (y + YL) * L::AW + z + 4 * q);
      wA[4 * q] = v.x; wA[4 * q + 1] = v.y; wA[4 * q + 2] = v.z; wA[4 * q + 3] = v.w;
    }
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float dxC = dtap<ORDER>(qc[0][e], qc[I1][e], qc[I2][e], qc[I3][e]);
      const float dzA = dtap<ORDER>(wA[zb + e], wA[zb + e + 1], wA[zb + e + 2], wA[zb + e + 3 < 12 ? zb + e + 3 : 11]);
      d[0][e] = __fmul_rn(-cxp, dxC);
      d[1][e] = 0.f;
      d[2][e] = __fmul_rn(czp, dzA);
    }
    torre_store<ORDER, ISH, TY>(p, stg, 1, d, x, j, y, z, z0, um, general, ms, off0);
  }
  // component 2 (Hz / Ez): +dx B, -dy A  (times sg)
  {
    float4 rA[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) rA[q] = lds4(sA + (y + YL + o0 + q) * L::AW + 4 + z);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float dxB = dtap<ORDER>(qb[0][e], qb[I1][e], qb[I2][e], qb[I3][e]);
      const float dyA = dtap<ORDER>(f4(rA[0], e), f4(rA[I1], e), f4(rA[I2], e), f4(rA[I3], e));
      d[0][e] = __fmul_rn(cxp, dxB);
      d[1][e] = __fmul_rn(-cyp, dyA);
      d[2][e] = 0.f;
    }
    torre_store<ORDER, ISH, TY>(p, stg, 2, d, x, j, y, z, z0, um, general, ms, off0);
  }
}

// Does the (plane x, tile) item need the general node path?
template <int TY>
__device__ __forceinline__ bool item_general(const Params& p, int x, int y0, int z0, bool isE, int um) {
  if (y0 + TY > p.g.n[1] || z0 + TT_Z > p.g.n[2]) return true;
  if (p.ab.kind != 0 && (in_slab(p, 0, x) || y0 < p.ab.L[1][0] || y0 + TY > p.g.n[1] - p.ab.L[1][1] ||
                         z0 < p.ab.L[2][0] || z0 + TT_Z > p.g.n[2] - p.ab.L[2][1]))
    return true;
  return isE && um < 0;
}

template <int ORDER, int NL, int TY>
__global__ void __launch_bounds__(TorreLayout<ORDER, TY>::NTHR, 1)
    torre_kernel(const __grid_constant__ Params p, const __grid_constant__ TorreMaps m, const TorreArgs ta) {
  using L = TorreLayout<ORDER, TY>;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* stages = smem;
  MatShared& ms = *reinterpret_cast<MatShared*>(smem + TT_NS * L::STAGE);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + TT_NS * L::STAGE + sizeof(MatShared));
  uint64_t* empty = full + TT_NS;
  uint64_t* done = empty + TT_NS;                          // step completion, ring of TT_NPUB
  int* stage_um = reinterpret_cast<int*>(done + TT_NPUB);  // material of each staged E item
  const int tz = blockIdx.x, ty = blockIdx.y;
  const int z0 = tz * TT_Z, y0 = ty * TY;
  const int nx = p.g.n[0];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Set when any wait of this CTA gave up.  From then on the producer issues
  // no copy (it never re-arms a stage whose copy may still be landing), every
  // warp leaves its loop, and the producer waits for its copies in flight
  // before it returns; the timeout is reported through p.err.
  __shared__ volatile int gave_up;
  if (threadIdx.x == 0) {
    for (int q = 0; q < TT_NS; q++) { mbar_init(&full[q], 1); mbar_init(&empty[q], L::NCW); }
    for (int q = 0; q < TT_NPUB; q++) mbar_init(&done[q], L::NCW);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    gave_up = 0;
  }
  for (int q = threadIdx.x; q < MAXMAT * 3; q += L::NTHR) (&ms.inv_eps[0][0])[q] = __ldg(&p.mt->inv_eps[0][0] + q);
  for (int q = threadIdx.x; q < MAXMAT; q += L::NTHR) ms.npoles[q] = __ldg(&p.mt->npoles[q]);
  __syncthreads();

  if (warp == L::NCW) {
    // ---------------- producer warp: neighbour waits (lanes 0-4), TMA issue (lane 0)
    int it = 0, seen = 0;
    for (int s = 0; s < ta.nsteps; s++) {
      // step s reads values produced up to step s - TT_K - 1 (own and neighbours)
      if (s - TT_K > 0 && !wait_tiles(p, ta, ty, tz, s - TT_K, seen)) gave_up = 1;
      if (lane == 0) {
        fence_proxy_async_global();
#pragma unroll 1
        for (int l = 0; l < NL && !gave_up; l++) {
          int x;
          if (!item_live<ORDER>(s, l, nx, x)) continue;
          const int st = it % TT_NS;
          if (it >= TT_NS && !mbar_wait(&empty[st], (unsigned)(((it / TT_NS) - 1) & 1), p.err, p.wait_limit)) {
            gave_up = 1;
            break;
          }
          const int um = ((l & 1) && x >= 0) ? torre_umat<TY>(p, x, ty, tz) : 0;
          stage_um[st] = um;
          const bool want_mat = (l & 1) && x >= 0 && um < 0;
          issue_item<ORDER, TY>(p, m, stages + st * L::STAGE, &full[st], l, x, y0, z0, want_mat);
          it++;
        }
      }
      if (__shfl_sync(0xffffffffu, gave_up, 0)) break;
      __syncwarp();
    }
    // no copy of this CTA may still be landing when it exits: after a wait
    // that gave up, the consumers may have moved past items still in flight
    if (lane == 0)
      for (int q = it - 1; q >= 0 && q >= it - TT_NS; q--)
        mbar_wait(&full[q % TT_NS], (unsigned)((q / TT_NS) & 1), nullptr, DRAIN_POLLS);
    return;
  }
  if (warp == L::NCW + 1) {
    // ---------------- publisher warp: release each completed wave step
    if (lane == 0) {
      int* mine = ta.ctr + ty * ta.ntz + tz;
      for (int s = 0; s < ta.nsteps && !gave_up; s++) {
        if (!mbar_wait(&done[s % TT_NPUB], (unsigned)((s / TT_NPUB) & 1), p.err, p.wait_limit)) {
          gave_up = 1;
          break;
        }
        __threadfence();
        st_release(mine, s + 1);
      }
    }
    return;
  }

  // ---------------- consumer warps
  float qb[NL][ORDER][4], qc[NL][ORDER][4];
#pragma unroll
  for (int l = 0; l < NL; l++)
#pragma unroll
    for (int q = 0; q < ORDER; q++)
#pragma unroll
      for (int e = 0; e < 4; e++) { qb[l][q][e] = 0.f; qc[l][q][e] = 0.f; }
  int it = 0;
  for (int s = 0; s < ta.nsteps; s++) {
    if (gave_up) break;
#pragma unroll
    for (int l = 0; l < NL; l++) {
      int x;
      if (!item_live<ORDER>(s, l, nx, x)) continue;
      const int st = it % TT_NS;
      // (all lanes poll; warp-uniform outcome, the stage completes for all of them at once)
      if (!mbar_wait(&full[st], (unsigned)((it / TT_NS) & 1), p.err, p.wait_limit)) gave_up = 1;
      if (__any_sync(0xffffffffu, gave_up != 0)) return;
      const unsigned char* stg = stages + st * L::STAGE;
      const bool isE = l & 1;
      const int um = stage_um[st];
      const bool gen = x >= 0 && item_general<TY>(p, x, y0, z0, isE, um);
      if (isE) torre_item<ORDER, false, TY>(p, stg, qb[l], qc[l], x, y0, z0, um, gen, ms);
      else torre_item<ORDER, true, TY>(p, stg, qb[l], qc[l], x, y0, z0, um, gen, ms);
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
      it++;
    }
    // this warp's stores of step s precede its arrival (release) on the step barrier
    __syncwarp();
    if (lane == 0) mbar_arrive(&done[s % TT_NPUB]);
  }
}

}  // namespace dtmx
