// dtmx_stream.cuh -- TMA-fed streaming kernels (one launch per half step).
//
// A CTA owns one (z,y) tile column and an x chunk, which the H step walks
// upwards and the E step downwards.  For every plane it needs the three
// source-field tiles (with y/z halo), the own values of the three updated
// components and, for the E step on mixed planes, their material indices.  One
// elected thread fetches all of them with cp.async.bulk.tensor (TMA, no
// multicast) into a ring of NST shared-memory stages, LEAD planes ahead of
// the ones the update reads; completion is tracked per stage by an mbarrier
// with a transaction count.  Out-of-array boxes are zero-filled by the TMA
// unit, which is exactly the zero-outside boundary; planes whose taps reach a
// mirror boundary are staged element-wise with the boundary rules instead.
#pragma once
#include "dtmx_device.cuh"

namespace dtmx {

__device__ __forceinline__ unsigned smem_u32(const void* q) { return (unsigned)__cvta_generic_to_shared(q); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred pp;\n mbarrier.try_wait.parity.shared::cta.b64 pp, [%1], %2;\n selp.u32 %0, 1, 0, pp;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `limit` polls (2^26 unless a test lowers it),
// records the failure in *err and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err, long long limit = 1LL << 26) {
  for (long long it = 0; !mbar_test(bar, parity); it++) {
    if (it > limit) {
      if (err) atomicExch(err, 1);
      return false;
    }
  }
  return true;
}
// Polls allowed while draining the copies of a CTA that gave up: TMA copies
// that were issued always complete, so this bound only guards a broken
// transaction count.
constexpr long long DRAIN_POLLS = 1LL << 20;
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

template <int ORDER, bool ISH>
struct Pipe {
  using S = Stage<ORDER, ISH>;
  static constexpr int OFF_A = 0;
  static constexpr int OFF_B = S::TA::N;
  static constexpr int OFF_C = OFF_B + S::TB::N;
  static constexpr int OFF_OWN = OFF_C + S::TC::N;
  static constexpr int OFF_MAT = OFF_OWN + 3 * OWN_N;
  static constexpr int STAGE = OFF_MAT + (ISH ? 0 : 3 * OWN_N / 4);   // floats, multiple of 32
  static constexpr unsigned BYTES = (S::TA::NV + S::TB::NV + S::TC::NV + 3 * OWN_N) * 4 + (ISH ? 0 : 3 * OWN_N);
  // The H step walks a chunk upwards in x, the E step downwards (the E update
  // reads only H, so the order of its planes is free).  Plane i needs its own
  // stage, AHEAD further planes along the walk (x taps not reached yet) and
  // BEHIND planes already passed (kept in the register queue): H taps -R..R-1
  // and E taps -(R-1)..R both give AHEAD = R-1 and BEHIND = R along their walk,
  // so each keeps LEAD planes in flight beyond the resident ones.
  static constexpr int DIR = ISH ? 1 : -1;             // direction of the walk along x
  static constexpr int AHEAD = ORDER == 4 ? 1 : 0;
  static constexpr int BEHIND = ORDER == 4 ? 2 : 1;
  // planes in flight beyond the resident ones: order 4 keeps one, so that its
  // 3-stage ring leaves room for 4 CTAs per SM (measured faster with absorbers)
  static constexpr int LEAD = ORDER == 4 ? 1 : 2;
  static constexpr int NST = AHEAD + 1 + LEAD;
  static constexpr int BASE = ISH ? 2 : 1;             // queue slot of x offset 0 (dstencil taps v0..v3)
  static constexpr size_t SMEM_BYTES = (size_t)NST * STAGE * 4 + sizeof(MatShared) + NST * 8 + 128;
};

// Stage plane ip into stage buffer st (all threads call; uniform fast flag);
// um: the plane tile's uniform material (< 0: mixed, the material tile is staged too).
template <int ORDER, bool ISH, int LD>
__device__ __forceinline__ void stage_plane(const Params& p, const TmaMaps& m, float* st, uint64_t* bar, int ip, int j0,
                                            int k0, bool fast, int um) {
  using P = Pipe<ORDER, ISH>;
  using S = typename P::S;
  const int c0 = ISH ? 0 : 3;       // source components
  const int cf = ISH ? 3 : 0;       // updated components
  const int tid = threadIdx.y * TZ + threadIdx.x;
  if (fast) {
    if (tid == 0) {
      // the material tile is needed only when this plane is updated with mixed materials
      const bool want_mat = !ISH && ip >= 0 && ip < p.g.n[0] && um < 0;
      mbar_arrive_expect_tx(bar, P::BYTES - (ISH || want_mat ? 0u : 3u * OWN_N));
      tma_load_3d(st + P::OFF_A, &m.src[c0], k0 - ZO, j0 - S::YL, ip, bar);
      tma_load_3d(st + P::OFF_B, &m.src[c0 + 1], k0 - ZO, j0, ip, bar);
      tma_load_3d(st + P::OFF_C, &m.src[c0 + 2], k0 - ZO, j0 - S::YL, ip, bar);
#pragma unroll
      for (int c = 0; c < 3; c++) tma_load_3d(st + P::OFF_OWN + c * OWN_N, &m.own[cf + c], k0, j0, ip, bar);
      if (want_mat)
#pragma unroll
        for (int c = 0; c < 3; c++)
          tma_load_3d(reinterpret_cast<uint8_t*>(st + P::OFF_MAT) + c * OWN_N, &m.mat[c], k0, j0, ip, bar);
    }
    return;
  }
  S::TA::template load_slow<LD>(st + P::OFF_A, p, c0, ip, j0, k0);
  S::TB::template load_slow<LD>(st + P::OFF_B, p, c0 + 1, ip, j0, k0);
  S::TC::template load_slow<LD>(st + P::OFF_C, p, c0 + 2, ip, j0, k0);
  const int tz = threadIdx.x, w = threadIdx.y;
#pragma unroll
  for (int r = 0; r < RY; r++) {
    const int y = w + TW * r, j = j0 + y, k = k0 + tz;
    const bool ok = ip >= 0 && ip < p.g.n[0] && j < p.g.n[1] && k < p.g.n[2];
    const long long off = (long long)ip * p.g.sx + (long long)j * p.g.sy + k;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      st[P::OFF_OWN + c * OWN_N + y * TZ + tz] = ok ? (LD ? __ldcg(p.f[cf + c] + off) : p.f[cf + c][off]) : 0.f;
      if (!ISH)
        reinterpret_cast<uint8_t*>(st + P::OFF_MAT)[c * OWN_N + y * TZ + tz] =
            (ok && p.mat[c]) ? __ldg(p.mat[c] + off) : (uint8_t)0;
    }
  }
  if (tid == 0) mbar_arrive(bar);
}

__device__ __forceinline__ bool tile_safe_yz(const Grid& g, int j0, int k0) {
  return j0 - 2 >= g.safe_lo[1] && j0 + TYT + 1 <= g.safe_hi[1] && k0 - 4 >= g.safe_lo[2] && k0 + TZ + 3 <= g.safe_hi[2];
}
__device__ __forceinline__ bool plane_safe_x(const Grid& g, int i) { return i - 2 >= g.safe_lo[0] && i + 2 <= g.safe_hi[0]; }

template <int ORDER, bool ISH>
__device__ __forceinline__ void stream_body(const Params& p, const TmaMaps& m, float* dsm) {
  using P = Pipe<ORDER, ISH>;
  using S = typename P::S;
  constexpr int NST = P::NST, AHEAD = P::AHEAD, BEHIND = P::BEHIND, BASE = P::BASE, LEAD = P::LEAD, DIR = P::DIR;
  MatShared& ms = *reinterpret_cast<MatShared*>(dsm + NST * P::STAGE);
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(&ms) + sizeof(MatShared));
  const int tz = threadIdx.x, w = threadIdx.y, tid = w * TZ + tz;
  const int k0 = blockIdx.x * TZ, j0 = blockIdx.y * TYT;
  const int xa = p.x0 + blockIdx.z * p.xchunk;
  const int xb = min(xa + p.xchunk, p.x1);
  const int len = xb - xa;
  const int i0 = DIR > 0 ? xa : xb - 1;      // first plane of the walk; step t works on plane i0 + DIR t
  // the uniform-material entries of the planes this CTA stages (stage number s),
  // read once so that the elected thread issues each stage without a dependent load
  constexpr int UMC = 128;
  __shared__ signed char umc[UMC];
  // set by the thread that waits for the stages when a wait gave up: the CTA
  // then stops issuing and computing, drains its copies in flight and returns
  __shared__ int gave_up;
  const int slast = len - 1 + AHEAD;         // last stage number that has to be staged
  if (tid == 0) {
    for (int q = 0; q < NST; q++) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    gave_up = 0;
  }
  if (!ISH) {
    load_matshared(ms, p);
    for (int sq = tid; sq <= slast && sq < UMC; sq += NTHR) {
      const int ip = i0 + DIR * sq;
      umc[sq] = (ip >= 0 && ip < p.g.n[0]) ? __ldg(p.umat + ((long long)ip * p.nty + blockIdx.y) * p.ntz + blockIdx.x)
                                          : (signed char)0;
    }
  }
  __syncthreads();
  // uniform material of stage number sq (0 for planes outside the array)
  auto um_of = [&](int sq) -> int {
    if (ISH) return 0;
    if (sq < UMC) return umc[sq];
    const int ip = i0 + DIR * sq;
    return (ip >= 0 && ip < p.g.n[0]) ? (int)__ldg(p.umat + ((long long)ip * p.nty + blockIdx.y) * p.ntz + blockIdx.x) : 0;
  };
  const bool yz_safe = tile_safe_yz(p.g, j0, k0);
  // (fast path of the per-node update additionally needs every node and tap live)
  const bool yz_in = j0 - 2 >= p.g.all_lo[1] && j0 + TYT + 1 <= p.g.all_hi[1] && k0 - 2 >= p.g.all_lo[2] &&
                     k0 + TZ + 1 <= p.g.all_hi[2];
  const int cb = ISH ? 1 : 4, cc = ISH ? 2 : 5;
  float qb[RY][4], qc[RY][4];
#pragma unroll
  for (int r = 0; r < RY; r++)
#pragma unroll
    for (int q = 0; q < 4; q++) { qb[r][q] = 0.f; qc[r][q] = 0.f; }
  // the BEHIND planes before the first one of the walk, from global memory
  for (int b = 1; b <= BEHIND; b++) {
    float tb[RY], tcv[RY];
    const int ip = i0 - DIR * b;
    const bool f = yz_in && ip >= p.g.all_lo[0] && ip <= p.g.all_hi[0];
    load_xtaps<0>(p, cb, ip, j0, k0, f, tb);
    load_xtaps<0>(p, cc, ip, j0, k0, f, tcv);
#pragma unroll
    for (int r = 0; r < RY; r++) { qb[r][BASE - DIR * b] = tb[r]; qc[r][BASE - DIR * b] = tcv[r]; }
  }
  // stage number s holds plane i0 + DIR s in slot s % NST (its (s / NST)-th use)
  for (int sq = 0; sq < AHEAD + LEAD && sq <= slast; sq++) {
    const int ip = i0 + DIR * sq;
    stage_plane<ORDER, ISH, 0>(p, m, dsm + (sq % NST) * P::STAGE, &bars[sq % NST], ip, j0, k0,
                               yz_safe && plane_safe_x(p.g, ip), um_of(sq));
  }
  for (int t = 0; t < len; t++) {
    const int i = i0 + DIR * t;
    const int spre = t + AHEAD + LEAD;
    if (spre <= slast) {
      const int ipre = i0 + DIR * spre;
      stage_plane<ORDER, ISH, 0>(p, m, dsm + (spre % NST) * P::STAGE, &bars[spre % NST], ipre, j0, k0,
                                 yz_safe && plane_safe_x(p.g, ipre), um_of(spre));
    }
    // values that do not depend on the staged tiles are loaded before the stage
    // wait, so their latency overlaps it: the plane's uniform material and the
    // absorber auxiliaries of the thread's nodes
    const int um = um_of(t);
    float old[RY][3][3];
    const bool tab = tile_absorber(p, i, j0, k0);
    if (tab) absorb_prefetch<ISH>(p, i, j0, k0, old);
    // stages t..t+AHEAD-1 were waited for in earlier steps (all of them at the
    // start); one thread polls the stage barriers and the CTA barrier then releases
    // everybody (and orders the staged data for them) without spinning issue slots
    if (tid == 0)
      for (int a = (t == 0 ? 0 : AHEAD); a <= AHEAD; a++)
        if (!mbar_wait(&bars[(t + a) % NST], (unsigned)(((t + a) / NST) & 1), p.err, p.wait_limit)) gave_up = 1;
    __syncthreads();
    if (gave_up) {
      // stages t .. the last one issued may still be landing: wait for them (bounded) before leaving
      if (tid == 0)
        for (int sq = t; sq <= min(slast, t + AHEAD + LEAD); sq++)
          mbar_wait(&bars[sq % NST], (unsigned)((sq / NST) & 1), nullptr, DRAIN_POLLS);
      return;
    }
    // every node of the tile in the array and live, every tap in range or zero: in the box
    // geometry a full tile (taps outside the array read the TMA zero fill)
    const bool fast = p.g.box ? (j0 + TYT <= p.g.n[1] && k0 + TZ <= p.g.n[2])
                              : (yz_in && i - 2 >= p.g.all_lo[0] && i + 2 <= p.g.all_hi[0]);
#pragma unroll
    for (int r = 0; r < RY; r++) {
      const int y = w + TW * r;
#pragma unroll
      for (int a = 0; a <= AHEAD; a++) {
        const float* st = dsm + ((t + a) % NST) * P::STAGE;
        qb[r][BASE + DIR * a] = S::TB::at(st + P::OFF_B, y, tz, 0, 0);
        qc[r][BASE + DIR * a] = S::TC::at(st + P::OFF_C, y, tz, 0, 0);
      }
    }
    const float* cur = dsm + (t % NST) * P::STAGE;
    const uint8_t* cmat = reinterpret_cast<const uint8_t*>(cur + P::OFF_MAT);
    if (fast && um >= 0 && !tab)
      plane_update<ORDER, ISH, 1>(p, i, j0, k0, cur, qb, qc, cur + P::OFF_OWN, cmat, ms, fast, um, old);
    else if (fast && um >= 0)
      plane_update<ORDER, ISH, 2>(p, i, j0, k0, cur, qb, qc, cur + P::OFF_OWN, cmat, ms, fast, um, old);
    else
      plane_update<ORDER, ISH, 0>(p, i, j0, k0, cur, qb, qc, cur + P::OFF_OWN, cmat, ms, fast, um, old);
    // the queue moves one plane along the walk
#pragma unroll
    for (int r = 0; r < RY; r++) {
      if (DIR > 0) {
#pragma unroll
        for (int q = 0; q < 3; q++) { qb[r][q] = qb[r][q + 1]; qc[r][q] = qc[r][q + 1]; }
      } else {
#pragma unroll
        for (int q = 3; q > 0; q--) { qb[r][q] = qb[r][q - 1]; qc[r][q] = qc[r][q - 1]; }
      }
    }
    __syncthreads();
  }
}

// 4 CTAs per SM: what shared memory allows for the 3-stage rings (64 registers)
template <int ORDER>
__global__ void __launch_bounds__(NTHR, 4) h_kernel(const __grid_constant__ Params p, const __grid_constant__ TmaMaps m) {
  extern __shared__ __align__(128) float dsm[];
  stream_body<ORDER, true>(p, m, dsm);
}

template <int ORDER>
__global__ void __launch_bounds__(NTHR, 4) e_kernel(const __grid_constant__ Params p, const __grid_constant__ TmaMaps m) {
  extern __shared__ __align__(128) float dsm[];
  stream_body<ORDER, false>(p, m, dsm);
}

}  // namespace dtmx
