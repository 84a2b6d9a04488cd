// dtmx_api.cu -- host runtime behind the C ABI declared in include/dtmx.h.
//
// Owns every device allocation of a simulation context, validates the
// configuration (the reference's printf+exit checks in GeoParamsHost::set,
// DTmxw.cu:278-487, become status codes), builds the coefficient tables and
// launches the per-step kernel sequence on the context's stream.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include <cudaTypedefs.h>

#include "dtmx.h"
#include "dtmx_device.cuh"
#include "dtmx_aux.cuh"
#include "dtmx_torre.cuh"
#include "dtmx_adjoint.cuh"
#include "dtmx_fused.cuh"

using namespace dtmx;

struct DftHost {
  DftDev d;
  int ncomp;
  double* omega = nullptr;
  double2* acc = nullptr;
  float* stage = nullptr;
  long long* sstep = nullptr;
  int nstaged = 0;          // samples staged since the last flush
};

// Six DFT patches of the tangential E and H components on the faces of a box
// and the device buffer their flux reduction writes to.
struct FluxHost {
  int face[6];              // DFT ids: x lo, x hi, y lo, y hi, z lo, z hi
  // far field: tangential E and H of each face plane and H of the next plane,
  // on windows [lo, hi] of the in-plane axes (one more point than the flux windows)
  int ffe[6], ffh[6];
  double sgn_area[6];       // outward sign times the cell face area
  int nfreq;
  double* d_out = nullptr;  // [6][nfreq]
};

// A device array of a parkable context: a CUDA virtual-address reservation
// with its own physical allocation, so that dtmx_park can release the physical
// memory while the address (held in Params, TMA descriptors and graphs) stays
// reserved, and dtmx_unpark can map new memory at the same address.
struct VmmBlock {
  CUdeviceptr va = 0;
  size_t size = 0;
  CUmemGenericAllocationHandle h = 0;
  void* host = nullptr;       // pinned copy while parked
  bool dead = false;          // parked without a copy: refilled with zeros on unpark
  bool fixed = false;         // constant once the context has stepped (materials, tables)
  bool saved_prepared = false;  // the host copy was taken after the context first stepped
};

struct dtmx_ctx {
  dtmx_config cfg{};
  int dev = 0;
  cudaStream_t stream = nullptr;
  Params P{};
  int nzp = 0;
  size_t nstore = 0;            // elements per component array (padded)
  size_t ncell = 0;             // nx*ny*nz
  std::vector<void*> allocs;
  std::vector<VmmBlock> vmm;    // the arrays of a parkable context (instead of allocs)
  bool parked = false;
  // coefficient tables
  float* ctab[3][3] = {};
  // materials
  MatTable* d_mt = nullptr;
  MatTable h_mt{};
  dtmx_material mats[DTMX_MAX_MATERIALS]{};
  int nmat = 1;
  uint8_t* d_mat[3] = {};
  std::vector<uint8_t> h_mat[3];
  // sources
  std::vector<PointSrcDev> psrc;
  PointSrcDev* d_psrc = nullptr;
  int has_tfsf = 0;
  dtmx_tfsf tfsf{};
  TfsfDev T{};
  int line_cap = 0;              // cells of line_e / line_h
  double* line_e = nullptr;
  double* line_h = nullptr;
  int line_src = 0;
  // monitors
  std::vector<ProbeDev> probes;
  ProbeDev* d_probes = nullptr;
  float* d_traces = nullptr;
  int probe_cap = 0;
  std::vector<DftHost> dfts;
  std::vector<FluxHost> fluxes;
  // state
  long long* d_step = nullptr;
  int* d_flag = nullptr;
  long long step = 0;
  long long launches = 0;
  bool prepared = false;
  bool profiling = false;
  cudaEvent_t ev[4] = {};
  double prof_ms_h = 0, prof_ms_e = 0;
  long long prof_count = 0;
  bool prof_pending = false;
  int engine = 0, tblock = 0;
  int xchunk = 0;               // planes per CTA of the per-step kernels (0: automatic)
  // 16 captured per-step launch sequences, one per field buffer holding the
  // current state (the single-sweep engine alternates them)
  cudaGraphExec_t graph16[2] = {};
  long long graph_launches[2] = {};
  TmaMaps maps{};
  // single-sweep engine (engine 3): the second field buffer and second set of
  // H auxiliaries (allocated on first use) and the maps reading each buffer
  // (its tiles are the per-step kernels' tiles and share their uniform-material
  // table).  P.f / P.ab.aux always point at the current state; the other set
  // is swapped in after every step.
  float* f_alt[6] = {};
  float* hax_alt[3][2] = {};
  TmaMaps maps_alt{};
  FusedMaps fmaps[2]{};               // 16-row tiles: [0] reads P.f, [1] reads f_alt (swapped with the buffers)
  FusedMaps fmaps8[2]{};              // the same for 8-row tiles
  int frows = 16;                     // tile rows of the single sweep (16 or 8; dtmx_set_tile_rows, dtmx_autotune)
  bool fused_ready = false;
  int parity = 0;                     // 0: state in the buffers allocated first
  int* d_err = nullptr;
  bool has_gyro = false;
  // design region and the objective of dtmx_forward_adjoint
  float* d_des_ie[3] = {};
  std::vector<float> h_des_ie[3];
  bool monitors_off = false;  // probes and DFT planes paused (recomputed segments)
  bool obj_on = false;        // capture the objective's flux DFT each step
  long long adj_budget = -1;  // bytes of design-region history the adjoint may keep (-1: a quarter of free memory)
  DftHost obj{};
  int gcur = 0;              // gyrotropic current buffer holding J^{n-1/2}
  // wavefront engine
  TorreMaps tmaps{};
  bool tmaps_ok = false;
  int* d_ctr = nullptr;
  signed char* d_umat = nullptr;
  std::string err;
};

// polls of one bounded device wait (mbarrier stages, wavefront neighbours / 16)
constexpr long long kWaitPolls = 1LL << 26;


static void drop_graphs(dtmx_ctx* ctx) {
  for (auto& g : ctx->graph16)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

static const char* kErrStr[] = {"ok", "invalid argument", "CUDA error", "out of device memory", "non-finite value",
                                "device wait timed out", "invalid state", "unsupported", "no CUDA device",
                                "input exceeds the fixed scratch size of the no-allocation entry point"};

#define CK(call)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      if (ctx) ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);              \
      return e_ == cudaErrorMemoryAllocation ? DTMX_ERR_OOM : DTMX_ERR_CUDA;               \
    }                                                                                      \
  } while (0)

static int fail(dtmx_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

// ---- parkable device memory (no reference counterpart) -----------------------
struct VmmApi {
  PFN_cuMemGetAllocationGranularity_v10020 gran = nullptr;
  PFN_cuMemAddressReserve_v10020 reserve = nullptr;
  PFN_cuMemAddressFree_v10020 vfree = nullptr;
  PFN_cuMemCreate_v10020 create = nullptr;
  PFN_cuMemRelease_v10020 release = nullptr;
  PFN_cuMemMap_v10020 map = nullptr;
  PFN_cuMemUnmap_v10020 unmap = nullptr;
  PFN_cuMemSetAccess_v10020 access = nullptr;
  bool ok = false;
};
static const VmmApi& vmm_api() {
  static const VmmApi api = [] {
    VmmApi v;
    auto get = [](const char* name, void** q) {
      cudaDriverEntryPointQueryResult qr;
      return cudaGetDriverEntryPoint(name, q, cudaEnableDefault, &qr) == cudaSuccess && qr == cudaDriverEntryPointSuccess;
    };
    v.ok = get("cuMemGetAllocationGranularity", (void**)&v.gran) && get("cuMemAddressReserve", (void**)&v.reserve) &&
           get("cuMemAddressFree", (void**)&v.vfree) && get("cuMemCreate", (void**)&v.create) &&
           get("cuMemRelease", (void**)&v.release) && get("cuMemMap", (void**)&v.map) &&
           get("cuMemUnmap", (void**)&v.unmap) && get("cuMemSetAccess", (void**)&v.access);
    return v;
  }();
  return api;
}
static CUmemAllocationProp vmm_prop(int dev) {
  CUmemAllocationProp prop{};
  prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  prop.location.id = dev;
  return prop;
}
// Physical allocations released by dtmx_park, kept per device for the next
// dtmx_unpark of a block of the same size (up to a byte limit, 0 by default:
// released at once).  Creating and releasing physical memory costs more than
// mapping it, so contexts that take turns on a device reuse each other's.
struct HandlePool {
  std::mutex mu;
  std::multimap<size_t, CUmemGenericAllocationHandle> free;
  size_t bytes = 0;
  long long limit = 0;          // < 0: unlimited
};
constexpr int kPoolDevices = 64;
static HandlePool& handle_pool(int dev) {
  static HandlePool pools[kPoolDevices];
  return pools[dev >= 0 && dev < kPoolDevices ? dev : 0];
}
static bool pool_take(int dev, size_t size, CUmemGenericAllocationHandle* h) {
  HandlePool& P = handle_pool(dev);
  std::lock_guard<std::mutex> lk(P.mu);
  auto it = P.free.find(size);
  if (it == P.free.end()) return false;
  *h = it->second;
  P.free.erase(it);
  P.bytes -= size;
  return true;
}
// keeps the handle (true) or leaves it to the caller to release (false)
static bool pool_put(int dev, size_t size, CUmemGenericAllocationHandle h) {
  HandlePool& P = handle_pool(dev);
  std::lock_guard<std::mutex> lk(P.mu);
  if (P.limit >= 0 && P.bytes + size > (size_t)P.limit) return false;
  P.free.insert({size, h});
  P.bytes += size;
  return true;
}
// physical memory for block b, mapped read-write at its reserved address
static CUresult vmm_back(int dev, VmmBlock& b) {
  const VmmApi& A = vmm_api();
  const CUmemAllocationProp prop = vmm_prop(dev);
  CUresult r = CUDA_SUCCESS;
  if (!pool_take(dev, b.size, &b.h) && (r = A.create(&b.h, b.size, &prop, 0)) != CUDA_SUCCESS) return r;
  if ((r = A.map(b.va, b.size, 0, b.h, 0)) != CUDA_SUCCESS) { A.release(b.h); return r; }
  CUmemAccessDesc acc{};
  acc.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  acc.location.id = dev;
  acc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
  if ((r = A.access(b.va, b.size, &acc, 1)) != CUDA_SUCCESS) { A.unmap(b.va, b.size); A.release(b.h); }
  return r;
}

template <class T>
static int dalloc(dtmx_ctx* ctx, T** p, size_t count, bool fixed = false) {
  if (ctx->cfg.parkable) {
    const VmmApi& A = vmm_api();
    if (!A.ok) return fail(ctx, DTMX_ERR_CUDA, "CUDA virtual memory management is unavailable");
    const CUmemAllocationProp prop = vmm_prop(ctx->dev);
    size_t g = 0;
    if (A.gran(&g, &prop, CU_MEM_ALLOC_GRANULARITY_MINIMUM) != CUDA_SUCCESS || g == 0)
      return fail(ctx, DTMX_ERR_CUDA, "allocation granularity");
    VmmBlock b;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    b.size = (bytes + g - 1) / g * g;
    if (A.reserve(&b.va, b.size, 0, 0, 0) != CUDA_SUCCESS) return fail(ctx, DTMX_ERR_OOM, "address reservation");
    if (vmm_back(ctx->dev, b) != CUDA_SUCCESS) { A.vfree(b.va, b.size); return fail(ctx, DTMX_ERR_OOM, "device memory"); }
    b.fixed = fixed;
    ctx->vmm.push_back(b);
    CK(cudaMemsetAsync((void*)b.va, 0, b.size, ctx->stream));
    *p = (T*)b.va;
    return DTMX_OK;
  }
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    ctx->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? DTMX_ERR_OOM : DTMX_ERR_CUDA;
  }
  e = cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(T), ctx->stream);
  if (e != cudaSuccess) { ctx->err = cudaGetErrorString(e); return DTMX_ERR_CUDA; }
  ctx->allocs.push_back(q);
  *p = (T*)q;
  return DTMX_OK;
}

extern "C" int dtmx_version(void) { return DTMX_ABI_VERSION; }
extern "C" const char* dtmx_error_string(int code) {
  if (code < 0 || code > 9) return "unknown";
  return kErrStr[code];
}
extern "C" const char* dtmx_last_error(const dtmx_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// ---------------------------------------------------------------- boundaries
static void setup_grid(dtmx_ctx* ctx) {
  Grid& g = ctx->P.g;
  const dtmx_config& c = ctx->cfg;
  int n[3] = {c.nx, c.ny, c.nz};
  for (int a = 0; a < 3; a++) g.n[a] = n[a];
  g.sy = ctx->nzp;
  g.sx = (long long)c.ny * ctx->nzp;
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) { g.btype[a][s] = 0; g.bsE[a][s] = 1; g.bsH[a][s] = 1; }
  g.box = c.geometry == DTMX_GEOM_BOX;
  if (c.geometry == DTMX_GEOM_BOX) {
    for (int a = 0; a < 3; a++) { g.bplane[a][0] = -1; g.bplane[a][1] = 2 * n[a]; }
  } else {
    // x: isOutS zero planes (defs.h:40); y: I-kernel free reflection at 0 with H odd
    // (genAlg.py:166-168) and X-kernel even mirror at 6*Na-3 (genAlg.py:9,36);
    // z: Vrefl even mirrors at 0 and 2*Nv-1 (defs.h:76-81).
    g.bplane[0][0] = 3; g.bplane[0][1] = 2 * n[0] - 3;
    g.btype[1][0] = 1; g.bplane[1][0] = 0; g.bsH[1][0] = -1;
    g.btype[1][1] = 1; g.bplane[1][1] = 2 * n[1] - 3;
    g.btype[2][0] = 1; g.bplane[2][0] = 0;
    g.btype[2][1] = 1; g.bplane[2][1] = 2 * n[2] - 1;
  }
  for (int comp = 0; comp < 6; comp++)
    for (int a = 0; a < 3; a++) {
      int lo = 0, hi = n[a] - 1;
      for (; lo <= hi; lo++) {
        int H = 2 * lo + comp_off(comp, a);
        if (g.btype[a][0] == 0 ? H > g.bplane[a][0] : H >= g.bplane[a][0]) break;
      }
      for (; hi >= lo; hi--) {
        int H = 2 * hi + comp_off(comp, a);
        if (g.btype[a][1] == 0 ? H < g.bplane[a][1] : H <= g.bplane[a][1]) break;
      }
      g.live_lo[comp][a] = lo;
      g.live_hi[comp][a] = hi;
    }
  for (int a = 0; a < 3; a++) {
    g.all_lo[a] = 0; g.all_hi[a] = n[a] - 1;
    for (int comp = 0; comp < 6; comp++) {
      g.all_lo[a] = std::max(g.all_lo[a], g.live_lo[comp][a]);
      g.all_hi[a] = std::min(g.all_hi[a], g.live_hi[comp][a]);
    }
    // a zero side never needs the boundary mapping: in-array non-live cells
    // hold zero and out-of-array boxes are zero-filled by the TMA unit
    g.safe_lo[a] = g.btype[a][0] == 0 ? -(1 << 28) : g.all_lo[a];
    g.safe_hi[a] = g.btype[a][1] == 0 ? (1 << 28) : g.all_hi[a];
  }
}

// Does the (plane i, y tile ty, z tile tz) streaming tile intersect the design region?
static bool design_touches(const dtmx_ctx* ctx, int i, int ty, int tz) {
  const Params& P = ctx->P;
  if (!P.des_on) return false;
  return i >= P.des_lo[0] && i < P.des_lo[0] + P.des_n[0] && ty * TYT < P.des_lo[1] + P.des_n[1] &&
         ty * TYT + TYT > P.des_lo[1] && tz * TZ < P.des_lo[2] + P.des_n[2] && tz * TZ + TZ > P.des_lo[2];
}

// ---------------------------------------------------------------- TMA descriptors
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* q = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &q, cudaEnableDefault, &qr) == cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)q;
  }
  return fn;
}

// 3-D map over a padded field (or material) array: dims (nz, ny, nx), box (bz, by, 1)
static int make_map(dtmx_ctx* ctx, CUtensorMap* map, void* base, bool bytes, int bz, int by) {
  auto fn = encode_fn();
  if (!fn) return fail(ctx, DTMX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const dtmx_config& c = ctx->cfg;
  const size_t es = bytes ? 1 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)c.nz, (cuuint64_t)c.ny, (cuuint64_t)c.nx};
  cuuint64_t strides[2] = {(cuuint64_t)ctx->nzp * es, (cuuint64_t)ctx->nzp * c.ny * es};
  cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, bytes ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box,
                  estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ctx, DTMX_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return DTMX_OK;
}

static int build_maps(dtmx_ctx* ctx) {
  const int R = ctx->cfg.order / 2;
  // source tiles: A and C components carry R (below) + R-1 (above) halo rows for
  // the H step and R-1 + R for the E step; B components no halo rows
  const int rows_h = TYT + 2 * R - 1, rows_e = TYT + 2 * R - 1;
  const int rows[6] = {rows_h, TYT, rows_h, rows_e, TYT, rows_e};
  int rc;
  for (int comp = 0; comp < 6; comp++) {
    if ((rc = make_map(ctx, &ctx->maps.src[comp], ctx->P.f[comp], false, TW_ROW, rows[comp]))) return rc;
    if ((rc = make_map(ctx, &ctx->maps.own[comp], ctx->P.f[comp], false, TZ, TYT))) return rc;
  }
  for (int comp = 0; comp < 3; comp++)
    if ((rc = make_map(ctx, &ctx->maps.mat[comp], ctx->d_mat[comp], true, TZ, TYT))) return rc;
  return DTMX_OK;
}

// Reference PMLgamma_func (DTmxw.cu:220-229).
static double ref_gamma(int i, int N, double dstep, double vmax) {
  if (i >= N - 3) return 0.0;
  if (i < 0) i = 0;
  N -= 3;
  const double att = 4.0;
  const double smax = vmax * std::log(10000.0) * ((att + 1.0) / (2.0 * (N * dstep * 0.5)));
  const double xmax = std::pow(smax, 1.0 / att);
  const double x = xmax - i * (xmax / N);
  return std::pow(x, att);
}

static int setup_absorber(dtmx_ctx* ctx) {
  const dtmx_config& c = ctx->cfg;
  Absorb& ab = ctx->P.ab;
  ab.kind = c.absorber;
  const int n[3] = {c.nx, c.ny, c.nz};
  const double d[3] = {c.dx, c.dy, c.dz};
  std::vector<float> t0[3], t1[3], t2[3];
  for (int a = 0; a < 3; a++) {
    const int H = 2 * n[a] + 2;
    t0[a].assign(H, 1.f); t1[a].assign(H, 0.f); t2[a].assign(H, 1.f);
    ab.L[a][0] = ab.L[a][1] = 0;
  }
  if (c.absorber == DTMX_ABS_CPML) {
    const double m = c.cpml_m > 0 ? c.cpml_m : 3.0;
    const double fac = c.cpml_sigma_factor > 0 ? c.cpml_sigma_factor : 1.0;
    const double kmax = c.cpml_kappa_max >= 1 ? c.cpml_kappa_max : 1.0;
    const double amax = c.cpml_alpha_max;
    for (int a = 0; a < 3; a++)
      for (int s = 0; s < 2; s++) {
        const int L = c.pml[a][s];
        ab.L[a][s] = L;
        if (L <= 0) continue;
        const double smax = fac * 0.8 * (m + 1.0) / d[a];
        for (int h = 0; h < 2 * n[a]; h++) {
          double dep = s == 0 ? (2.0 * L - 1.0 - h) * 0.5 : (h - (2.0 * n[a] - 2.0 * L)) * 0.5;
          if (dep <= 0) continue;
          dep = std::min<double>(dep, L);
          const double r = dep / L;
          const double sg = smax * std::pow(r, m);
          const double kp = 1.0 + (kmax - 1.0) * std::pow(r, m);
          const double al = amax * (1.0 - r);
          const double b = std::exp(-(sg / kp + al) * c.dt);
          const double aa = sg > 0 ? sg / (sg * kp + kp * kp * al) * (b - 1.0) : 0.0;
          t0[a][h] = (float)b; t1[a][h] = (float)aa; t2[a][h] = (float)(1.0 / kp);
        }
      }
  } else if (c.absorber == DTMX_ABS_SPLIT_PML) {
    // setPMLcoeffs (DTmxw.cu:250-265): K2 = 1/(1+dt/2*gamma), K1 = 2*K2-1;
    // K1 = K2 = 1 where gamma = 0
    for (int a = 0; a < 3; a++) t1[a].assign(2 * n[a] + 2, 1.f);
    const double V = c.spml_vmax;
    // table lengths KNpmlx = 2 Npmlx NDT, KNpmly = 2 Npmly NDT, KNpmlz = 2 Npmlz (params.h:106-108);
    // the slabs are Npmlx/2 and Npmly/2 rags of NDT cells and the Npmlz/2 top layers
    const int KX = 4 * c.pml[0][0], KY = 4 * c.pml[1][0], KZ = 4 * c.pml[2][1];
    const int XS = 2 * c.pml[0][0] - 3;                // inPMLsync (defs.h:45): Npmlx/2*2*NDT - NDT
    ab.L[0][0] = c.pml[0][0]; ab.L[0][1] = c.pml[0][1];
    ab.L[1][0] = c.pml[1][0]; ab.L[1][1] = c.pml[1][1];
    ab.L[2][0] = 0;           ab.L[2][1] = c.pml[2][1];
    for (int h = 0; h < 2 * n[0] + 2; h++) {
      int i = -1;
      if (h < XS) i = h;
      else if (h >= 2 * n[0] - XS) i = h - 2 * n[0] + KX;
      if (i < 0 || i >= KX) continue;
      const double k2 = 1.0 / (1.0 + 0.5 * c.dt * ref_gamma(KX / 2 - std::abs(i - KX / 2) - 3, KX / 2 - 3, c.dx, V));
      t1[0][h] = (float)k2; t0[0][h] = (float)(2.0 * k2 - 1.0);
    }
    for (int h = 0; h < 2 * n[1] + 2; h++) {
      int i = -1;
      if (h < KY / 2) i = h;
      else if (h >= 2 * n[1] - KY / 2) i = h - 2 * n[1] + KY;
      if (i < 0 || i >= KY) continue;
      const double k2 = 1.0 / (1.0 + 0.5 * c.dt * ref_gamma(i < KY / 2 ? i : KY - i - 3, KY / 2, c.dy, V));
      t1[1][h] = (float)k2; t0[1][h] = (float)(2.0 * k2 - 1.0);
    }
    for (int h = 0; h < 2 * n[2] + 2; h++) {
      const int i = h - 2 * n[2] + KZ;                 // top face only (DTmxw.cu:262)
      if (i < KZ / 2 || i >= KZ) continue;
      const double k2 = 1.0 / (1.0 + 0.5 * c.dt * ref_gamma(KZ - i - 1, KZ / 2, c.dz, V));
      t1[2][h] = (float)k2; t0[2][h] = (float)(2.0 * k2 - 1.0);
    }
  }
  for (int a = 0; a < 3; a++) {
    const int H = 2 * n[a] + 2;
    float* q[3];
    for (int t = 0; t < 3; t++) {
      int rc = dalloc(ctx, &q[t], H, true);
      if (rc) return rc;
    }
    CK(cudaMemcpyAsync(q[0], t0[a].data(), H * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(q[1], t1[a].data(), H * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(q[2], t2[a].data(), H * 4, cudaMemcpyHostToDevice, ctx->stream));
    ab.c0[a] = q[0]; ab.c1[a] = q[1]; ab.c2[a] = q[2];
    const size_t th = (size_t)(ab.L[a][0] + ab.L[a][1]);
    for (int s = 0; s < 4; s++) ab.aux[a][s] = nullptr;
    if (!th || c.absorber == DTMX_ABS_NONE) continue;
    const size_t cnt = th * (ctx->ncell / (size_t)n[a]);
    if (cnt >= (size_t)INT32_MAX) return fail(ctx, DTMX_ERR_UNSUPPORTED, "absorber slab of more than 2^31 values");
    for (int s = 0; s < 4; s++) {
      int rc = dalloc(ctx, &ab.aux[a][s], cnt);
      if (rc) return rc;
    }
    // sync the coefficient vectors (host memory) before they go out of scope
    CK(cudaStreamSynchronize(ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return DTMX_OK;
}

static int upload_mattable(dtmx_ctx* ctx) {
  dtmx_ctx* c = ctx;
  CK(cudaMemcpyAsync(c->d_mt, &c->h_mt, sizeof(MatTable), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DTMX_OK;
}

extern "C" int dtmx_create(const dtmx_config* cfg, dtmx_ctx** out) {
  if (!cfg || !out) return DTMX_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DTMX_ERR_NODEVICE;
  const dtmx_config& c = *cfg;
  if (c.nx < 8 || c.ny < 8 || c.nz < 8) return DTMX_ERR_INVALID;
  if (c.order != 2 && c.order != 4) return DTMX_ERR_INVALID;
  if (!(c.dx > 0 && c.dy > 0 && c.dz > 0 && c.dt > 0)) return DTMX_ERR_INVALID;
  // Courant limits: 1 for the Yee stencil, 6/7 for the (27,-1)/24 stencil (DTmxw.cu:332)
  const double cn = c.dt * std::sqrt(1 / (c.dx * c.dx) + 1 / (c.dy * c.dy) + 1 / (c.dz * c.dz));
  if (cn > (c.order == 4 ? 6.0 / 7.0 : 1.0)) return DTMX_ERR_INVALID;
  if (c.geometry != DTMX_GEOM_BOX && c.geometry != DTMX_GEOM_REFERENCE) return DTMX_ERR_INVALID;
  if (c.absorber == DTMX_ABS_CPML && c.geometry != DTMX_GEOM_BOX) return DTMX_ERR_UNSUPPORTED;
  if (c.absorber == DTMX_ABS_SPLIT_PML && c.geometry != DTMX_GEOM_REFERENCE) return DTMX_ERR_UNSUPPORTED;
  if (c.geometry == DTMX_GEOM_REFERENCE && (c.nx % 3 || c.ny % 3)) return DTMX_ERR_INVALID;  // DTmxw.cu:330-331
  // split PML: whole rags along x and y on both faces, the top z face only (Npmlx/2, Npmly/2 rags, Npmlz/2 layers)
  if (c.absorber == DTMX_ABS_SPLIT_PML &&
      (c.pml[0][0] != c.pml[0][1] || c.pml[1][0] != c.pml[1][1] || c.pml[0][0] % 3 || c.pml[1][0] % 3 ||
       c.pml[0][0] < 3 || c.pml[1][0] < 3 || c.pml[2][0] != 0 || c.pml[2][1] < 2))
    return DTMX_ERR_INVALID;
  const int n[3] = {c.nx, c.ny, c.nz};
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++)
      if (c.pml[a][s] < 0 || c.pml[a][0] + c.pml[a][1] > n[a] - 4) return DTMX_ERR_INVALID;

  dtmx_ctx* ctx = new dtmx_ctx();
  ctx->cfg = c;
  if (cudaGetDevice(&ctx->dev) != cudaSuccess) { delete ctx; return DTMX_ERR_CUDA; }
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return DTMX_ERR_CUDA; }
  ctx->nzp = (c.nz + 31) / 32 * 32;
  ctx->ncell = (size_t)c.nx * c.ny * c.nz;
  ctx->nstore = (size_t)c.nx * c.ny * ctx->nzp;
  setup_grid(ctx);
  int rc = DTMX_OK;
  // 64 floats of slack: aligned 16-byte tile rows may read up to 3 floats past the last node
  for (int comp = 0; comp < 6 && !rc; comp++) rc = dalloc(ctx, &ctx->P.f[comp], ctx->nstore + 64);
  if (!rc) rc = setup_absorber(ctx);
  if (!rc) rc = dalloc(ctx, &ctx->d_mt, 1, true);
  if (!rc) rc = dalloc(ctx, &ctx->d_step, 1);
  if (!rc) rc = dalloc(ctx, &ctx->d_flag, 1);
  if (!rc) rc = dalloc(ctx, &ctx->d_err, 1);
  for (int comp = 0; comp < 3 && !rc; comp++) rc = dalloc(ctx, &ctx->d_mat[comp], ctx->nstore + 64, true);
  if (!rc) rc = build_maps(ctx);
  ctx->P.ntz = (c.nz + TZ - 1) / TZ;
  ctx->P.nty = (c.ny + TYT - 1) / TYT;
  if (!rc) rc = dalloc(ctx, &ctx->d_umat, (size_t)c.nx * ctx->P.nty * ctx->P.ntz, true);   // zeros: material 0 everywhere
  if (rc) { *out = ctx; return rc; }
  ctx->P.umat = ctx->d_umat;
  ctx->P.err = ctx->d_err;
  ctx->P.wait_limit = kWaitPolls;
  for (int comp = 0; comp < 3; comp++) ctx->P.mat[comp] = ctx->d_mat[comp];
  ctx->P.cdt[0] = (float)(c.dt / c.dx); ctx->P.cdt[1] = (float)(c.dt / c.dy); ctx->P.cdt[2] = (float)(c.dt / c.dz);
  // default material 0: vacuum
  dtmx_material vac{};
  vac.eps[0] = vac.eps[1] = vac.eps[2] = 1.0;
  ctx->mats[0] = vac;
  for (int comp = 0; comp < 3; comp++) ctx->h_mt.inv_eps[0][comp] = 1.f;
  ctx->P.mt = ctx->d_mt;
  rc = upload_mattable(ctx);
  if (rc) { *out = ctx; return rc; }
  ctx->probe_cap = c.probe_capacity > 0 ? c.probe_capacity : 4096;
  *out = ctx;
  return DTMX_OK;
}

extern "C" void dtmx_destroy(dtmx_ctx* ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& g : ctx->graph16)
    if (g) cudaGraphExecDestroy(g);
  for (void* p : ctx->allocs) cudaFree(p);
  for (auto& b : ctx->vmm) {
    const VmmApi& A = vmm_api();
    if (!ctx->parked) { A.unmap(b.va, b.size); A.release(b.h); }
    A.vfree(b.va, b.size);
    if (b.host) cudaFreeHost(b.host);
  }
  for (auto& d : ctx->dfts) { cudaFree(d.omega); cudaFree(d.acc); cudaFree(d.stage); cudaFree(d.sstep); }
  for (auto& fx : ctx->fluxes) cudaFree(fx.d_out);
  cudaFree(ctx->obj.omega); cudaFree(ctx->obj.acc); cudaFree(ctx->obj.stage); cudaFree(ctx->obj.sstep);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

// ---------------------------------------------------------------- materials
// DispStruct::set (dispersion.cpp:41-82), coefficients in double then stored in float.
static void disp_coeffs(const dtmx_material& M, double dt, MatTable& t, int mi) {
  double alpha[MAXPOLE], ksi[MAXPOLE], zetp[MAXPOLE], zetm[MAXPOLE], zet[MAXPOLE];
  double zms = 0, zps = 0, zs = 0;
  for (int i = 0; i < M.npoles; i++) {
    const double Deps = M.pole[i][0], wp = M.pole[i][1], gp = M.pole[i][2], gp_ = M.pole[i][3];
    const double a0 = Deps * wp * wp, a1 = Deps * gp_;
    const double b0 = M.pole_kind[i] == DTMX_POLE_DRUDE ? 0.0 : wp * wp, b1 = 2 * gp;
    alpha[i] = (4 - 2 * b0 * dt * dt) / (b1 * dt + 2);
    ksi[i] = (b1 * dt - 2) / (b1 * dt + 2);
    zetp[i] = (a0 * dt * dt + 2 * a1 * dt) / (b1 * dt + 2);
    zetm[i] = (-a0 * dt * dt + 2 * a1 * dt) / (b1 * dt + 2);
    zet[i] = -(4 * a1 * dt) / (b1 * dt + 2);
    zms += zetm[i]; zps += zetp[i]; zs += zet[i];
  }
  const double den = 2 * M.eps_inf + M.sigma * dt + zps;
  const double C1 = -zms / den, C2 = (2 * M.eps_inf - M.sigma * dt - zs) / den, C3 = 2 * dt / den;
  for (int xc = 0; xc < 3; xc++) {
    for (int i = 0; i < M.npoles; i++) {
      t.kJ[mi][xc][i][0] = (float)alpha[i]; t.kJ[mi][xc][i][1] = (float)ksi[i];
      t.kJ[mi][xc][i][2] = (float)(zetp[i] / dt); t.kJ[mi][xc][i][3] = (float)(zetm[i] / dt);
      t.kJ[mi][xc][i][4] = (float)(zet[i] / dt);
      t.kEJ[mi][xc][i][0] = (float)(C3 * 0.5 * (1 + alpha[i])); t.kEJ[mi][xc][i][1] = (float)(C3 * 0.5 * ksi[i]);
    }
    t.kE[mi][xc][0] = (float)C1; t.kE[mi][xc][1] = (float)C2; t.kE[mi][xc][2] = (float)(C3 / dt);
  }
}

static inline size_t store_index(const dtmx_ctx* ctx, int i, int j, int k) {
  return ((size_t)i * ctx->cfg.ny + j) * ctx->nzp + k;
}

// Per (plane, y tile, z tile): the common non-dispersive material of all
// three E components, -1 if mixed, dispersive, gyrotropic or in the design
// region (selects the simple path of the field kernels).
static int upload_umat(dtmx_ctx* ctx) {
  const dtmx_config& c = ctx->cfg;
  const int nty = ctx->P.nty, ntz = ctx->P.ntz;
  const bool have = !ctx->h_mat[0].empty();
  std::vector<signed char> um((size_t)c.nx * nty * ntz);
  for (int i = 0; i < c.nx; i++)
    for (int ty = 0; ty < nty; ty++)
      for (int tz = 0; tz < ntz; tz++) {
        int m0 = have ? -2 : 0;
        for (int j = ty * TYT; have && j < std::min(c.ny, ty * TYT + TYT) && m0 != -1; j++)
          for (int comp = 0; comp < 3 && m0 != -1; comp++) {
            const uint8_t* row = ctx->h_mat[comp].data() + store_index(ctx, i, j, 0);
            for (int k = tz * TZ; k < std::min(c.nz, tz * TZ + TZ); k++) {
              const int m = row[k];
              if (m0 == -2) m0 = m;
              // (a gyrotropic node takes the plain update with 1/eps_inf; its current is
              // subtracted by the post-pass, so a uniform gyrotropic tile stays uniform)
              if (m != m0 || ctx->mats[m].npoles > 0) { m0 = -1; break; }
            }
          }
        um[((size_t)i * nty + ty) * ntz + tz] = (signed char)(m0 < 0 || design_touches(ctx, i, ty, tz) ? -1 : m0);
      }
  CK(cudaMemcpyAsync(ctx->d_umat, um.data(), um.size(), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return DTMX_OK;
}

extern "C" int dtmx_set_materials(dtmx_ctx* ctx, const dtmx_material* table, int nmat, const uint8_t* idx_x,
                                  const uint8_t* idx_y, const uint8_t* idx_z) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || !table || nmat < 1 || nmat > DTMX_MAX_MATERIALS || !idx_x) return fail(ctx, DTMX_ERR_INVALID, "bad material arguments");
  if (ctx->prepared) return fail(ctx, DTMX_ERR_STATE, "materials must be set before the first step");
  const uint8_t* src[3] = {idx_x, idx_y ? idx_y : idx_x, idx_z ? idx_z : idx_x};
  for (int m = 0; m < nmat; m++) {
    const dtmx_material& M = table[m];
    if (M.npoles < 0 || M.npoles > DTMX_MAX_POLES) return fail(ctx, DTMX_ERR_INVALID, "npoles out of range");
    if (M.npoles > 0 && !(M.eps_inf > 0)) return fail(ctx, DTMX_ERR_INVALID, "dispersive material needs eps_inf > 0");
    if (M.npoles == 0 && !(M.eps[0] > 0 && M.eps[1] > 0 && M.eps[2] > 0)) return fail(ctx, DTMX_ERR_INVALID, "eps must be > 0");
    if (M.gyro_wp < 0) return fail(ctx, DTMX_ERR_INVALID, "gyro_wp must be >= 0");
    if (M.gyro_wp > 0 && (M.npoles > 0 || !(M.eps_inf > 0)))
      return fail(ctx, DTMX_ERR_INVALID, "a gyrotropic material needs npoles = 0 and eps_inf > 0");
  }
  MatTable& t = ctx->h_mt;
  memset(&t, 0, sizeof(t));
  for (int m = 0; m < nmat; m++) {
    ctx->mats[m] = table[m];
    t.npoles[m] = table[m].npoles;
    for (int c = 0; c < 3; c++) t.inv_eps[m][c] = table[m].npoles > 0 ? 0.f : (float)(1.0 / table[m].eps[c]);
    if (table[m].npoles > 0) disp_coeffs(table[m], ctx->cfg.dt, t, m);
    if (table[m].gyro_wp > 0) {
      const double dt = ctx->cfg.dt;
      for (int c = 0; c < 3; c++) t.inv_eps[m][c] = (float)(1.0 / table[m].eps_inf);
      t.gA[m] = (float)std::exp(-table[m].gyro_gamma * dt);
      t.gC[m] = (float)std::cos(table[m].gyro_wc * dt);
      t.gS[m] = (float)std::sin(table[m].gyro_wc * dt);
      t.gB[m] = (float)(table[m].gyro_wp * table[m].gyro_wp * dt);
      t.gjc[m] = (float)(dt / table[m].eps_inf);
    }
  }
  ctx->nmat = nmat;
  const dtmx_config& c = ctx->cfg;
  int lo[3] = {c.nx, c.ny, c.nz}, hi[3] = {-1, -1, -1};
  for (int comp = 0; comp < 3; comp++) {
    ctx->h_mat[comp].assign(ctx->nstore, 0);
    for (int i = 0; i < c.nx; i++)
      for (int j = 0; j < c.ny; j++) {
        const uint8_t* row = src[comp] + ((size_t)i * c.ny + j) * c.nz;
        uint8_t* dst = ctx->h_mat[comp].data() + store_index(ctx, i, j, 0);
        for (int k = 0; k < c.nz; k++) {
          const uint8_t m = row[k];
          if (m >= nmat) return fail(ctx, DTMX_ERR_INVALID, "material index out of range");
          dst[k] = m;
          if (table[m].npoles > 0 || table[m].gyro_wp > 0) {
            const int v[3] = {i, j, k};
            for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], v[a]); hi[a] = std::max(hi[a], v[a]); }
          }
        }
      }
    CK(cudaMemcpyAsync(ctx->d_mat[comp], ctx->h_mat[comp].data(), ctx->nstore, cudaMemcpyHostToDevice, ctx->stream));
    ctx->P.mat[comp] = ctx->d_mat[comp];
  }
  int rc = upload_mattable(ctx);
  if (rc) return rc;
  if ((rc = upload_umat(ctx))) return rc;
  Ade& A = ctx->P.ade;
  if (hi[0] >= 0) {
    size_t na = 1;
    for (int a = 0; a < 3; a++) { A.lo[a] = lo[a]; A.n[a] = hi[a] - lo[a] + 1; na *= A.n[a]; }
    int maxp = 0;
    bool gyro = false;
    for (int m = 0; m < nmat; m++) { maxp = std::max(maxp, table[m].npoles); gyro = gyro || table[m].gyro_wp > 0; }
    ctx->has_gyro = gyro;
    ctx->gcur = 0;
    for (int comp = 0; comp < 3 && gyro; comp++)
      for (int b = 0; b < 2; b++)
        if ((rc = dalloc(ctx, &A.Jg[b][comp], na))) return rc;
    for (int comp = 0; comp < 3; comp++) {
      if ((rc = dalloc(ctx, &A.Em[comp], na))) return rc;
      for (int q = 0; q < maxp; q++) {
        if ((rc = dalloc(ctx, &A.Jp[comp][q], na))) return rc;
        if ((rc = dalloc(ctx, &A.Jm[comp][q], na))) return rc;
      }
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return DTMX_OK;
}

static bool node_live(const dtmx_ctx* ctx, int comp, int i, int j, int k) {
  const Grid& g = ctx->P.g;
  return i >= g.live_lo[comp][0] && i <= g.live_hi[comp][0] && j >= g.live_lo[comp][1] && j <= g.live_hi[comp][1] &&
         k >= g.live_lo[comp][2] && k <= g.live_hi[comp][2];
}

extern "C" int dtmx_add_point_source(dtmx_ctx* ctx, const dtmx_point_source* s) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || !s || s->comp < 0 || s->comp > 2) return fail(ctx, DTMX_ERR_INVALID, "bad point source");
  if (!node_live(ctx, s->comp, s->i, s->j, s->k)) return fail(ctx, DTMX_ERR_INVALID, "point source outside the live domain");
  if (!(s->tau > 0)) return fail(ctx, DTMX_ERR_INVALID, "point source tau must be > 0");
  if (ctx->prepared) return fail(ctx, DTMX_ERR_STATE, "sources must be added before the first step");
  PointSrcDev d;
  d.comp = s->comp;
  d.id = (long long)store_index(ctx, s->i, s->j, s->k);
  d.amp = s->amp; d.f0 = s->f0; d.tau = s->tau; d.t0 = s->t0;
  ctx->psrc.push_back(d);
  return DTMX_OK;
}

// inSF along one axis with the reference's float arithmetic (signal.hpp:153-160)
static void sf_range(double dstep, double bm, double bp, int hmax, int* lo, int* hi) {
  const float bmf = (float)bm, bpf = (float)bp, df = (float)dstep;
  *lo = 1; *hi = 0;
  bool first = true;
  for (int h = -8; h <= hmax + 8; h++) {
    const float sv = (float)((double)h * 0.5 * (double)df);
    if (sv > bmf && sv < bpf) { if (first) { *lo = h; first = false; } *hi = h; }
  }
}

extern "C" int dtmx_set_tfsf(dtmx_ctx* ctx, const dtmx_tfsf* s) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || !s || (s->kind != DTMX_TFSF_DIPOLE && s->kind != DTMX_TFSF_PLANE_X)) return fail(ctx, DTMX_ERR_INVALID, "bad TF/SF source");
  if (ctx->prepared) return fail(ctx, DTMX_ERR_STATE, "TF/SF source must be set before the first step");
  const dtmx_config& c = ctx->cfg;
  // a slab of a larger grid: plane 0 is whole-grid cell xo of gnx
  const int xo = (int)s->x_origin;
  const int gnx = s->x_cells > 0 ? (int)s->x_cells : c.nx;
  if ((double)xo != s->x_origin || (s->x_cells > 0 && (double)gnx != s->x_cells) || xo < 0 || xo + c.nx > gnx ||
      (c.geometry != DTMX_GEOM_BOX && (xo != 0 || gnx != c.nx)))
    return fail(ctx, DTMX_ERR_INVALID, "TF/SF x_origin / x_cells do not place this grid inside a whole grid");
  TfsfDev& T = ctx->T;
  T = TfsfDev{};
  T.xo = xo;
  const double d[3] = {c.dx, c.dy, c.dz};
  const int n[3] = {c.nx, c.ny, c.nz};
  for (int a = 0; a < 3; a++) {
    sf_range(d[a], s->box_lo[a], s->box_hi[a], 2 * (a == 0 ? gnx : n[a]), &T.lo[a], &T.hi[a]);
    if (T.lo[a] > T.hi[a]) return fail(ctx, DTMX_ERR_INVALID, "TF/SF box contains no node");
    if (a == 0) { T.lo[0] -= 2 * xo; T.hi[0] -= 2 * xo; }
    // the correction shell (3 half cells around the surface) must stay inside the
    // live domain and clear of the absorber (along x: at the grid's uncut ends)
    const int clo = (T.lo[a] - 4) / 2 - 1, chi = (T.hi[a] + 4) / 2 + 1;
    const int alo = c.absorber == DTMX_ABS_NONE ? 0 : ctx->P.ab.L[a][0];
    const int ahi = c.absorber == DTMX_ABS_NONE ? 0 : ctx->P.ab.L[a][1];
    int llo = 0, lhi = n[a] - 1;
    for (int comp = 0; comp < 6; comp++) { llo = std::max(llo, ctx->P.g.live_lo[comp][a]); lhi = std::min(lhi, ctx->P.g.live_hi[comp][a]); }
    const bool lo_end = a != 0 || xo == 0, hi_end = a != 0 || xo + c.nx == gnx;
    if ((lo_end && clo < std::max(alo, llo) + 1) || (hi_end && chi > std::min(n[a] - 1 - ahi, lhi) - 1))
      return fail(ctx, DTMX_ERR_INVALID, "TF/SF box too close to the boundary or absorber");
  }
  T.active_cfg = 1;
  T.kind = s->kind;
  for (int a = 0; a < 3; a++) { T.ctr[a] = (s->box_lo[a] + s->box_hi[a]) * 0.5; T.hd[a] = d[a] * 0.5; }
  T.dt = c.dt; T.c = s->c; T.w = s->w; T.kenv = s->kenv; T.tstop = s->tstop;
  T.ntime = s->ntime > 0 ? s->ntime : 1;
  // correction jobs: per half step, component and curl term (axis a, source
  // component g), the nodes within 3 half cells of each face along a whose g
  // taps lie inside the box range on the other two axes
  for (int hs = 0; hs < 2; hs++) {
    T.njob[hs] = 0;
    for (int comp = hs * 3; comp < hs * 3 + 3; comp++) {
      int ax[2], gs[2];
      curl_terms(comp, ax[0], gs[0], ax[1], gs[1]);
      for (int term = 0; term < 2; term++) {
        const int a = ax[term], g = gs[term];
        if (s->kind == DTMX_TFSF_PLANE_X && g != 2 && g != 4) continue;
        for (int side = 0; side < 2; side++) {
          TfsfJob jb{};
          jb.c = comp;
          bool empty = false;
          for (int b = 0; b < 3; b++) {
            int X0, X1, o;
            if (b == a) { X0 = side ? T.hi[a] - 3 : T.lo[a] - 4; X1 = side ? T.hi[a] + 4 : T.lo[a] + 3; o = comp_off(comp, a); }
            else { X0 = T.lo[b]; X1 = T.hi[b]; o = comp_off(g, b); }
            // indices v with X0 <= 2v + o <= X1, clipped to the grid
            int v0 = (int)std::ceil((X0 - o) / 2.0), v1 = (int)std::floor((X1 - o) / 2.0);
            v0 = std::max(v0, 0); v1 = std::min(v1, n[b] - 1);
            if (b == a) {
              // along the curl axis keep only the indices where a tap of g actually
              // crosses the box surface (the other two axes agree for c and g)
              const int t0 = hs ? -2 : -1, qa = c.order == 4 ? 0 : 1, qb = c.order == 4 ? 3 : 2;
              auto crosses = [&](int v) {
                const int S = 2 * v + comp_off(comp, a);
                const bool sin_ = S >= T.lo[a] && S <= T.hi[a];
                for (int q = qa; q <= qb; q++) {
                  const int G = 2 * (v + t0 + q) + comp_off(g, a);
                  if ((G >= T.lo[a] && G <= T.hi[a]) != sin_) return true;
                }
                return false;
              };
              while (v0 <= v1 && !crosses(v0)) v0++;
              while (v1 >= v0 && !crosses(v1)) v1--;
            }
            if (v0 > v1) empty = true;
            jb.lo[b] = v0; jb.hi[b] = v1;
          }
          if (empty) continue;
          jb.cells = (long long)(jb.hi[0] - jb.lo[0] + 1) * (jb.hi[1] - jb.lo[1] + 1) * (jb.hi[2] - jb.lo[2] + 1);
          if (jb.cells >= (long long)INT32_MAX) return fail(ctx, DTMX_ERR_UNSUPPORTED, "TF/SF correction shell of more than 2^31 nodes");
          T.job[hs][T.njob[hs]++] = jb;
        }
      }
    }
  }
  if (s->kind == DTMX_TFSF_PLANE_X) {
    // the 1-D line spans the whole grid with 4096 cells beyond each end; plane 0
    // of this grid reads line cell xo + 4096, the source sits 10 cells before
    // the box's lower x face
    constexpr int kLinePad = 4096;
    T.line_M = kLinePad + xo;
    T.line_n = gnx + 2 * kLinePad;
    int rc;
    if (ctx->line_cap < T.line_n) {
      if ((rc = dalloc(ctx, &ctx->line_e, T.line_n))) return rc;
      if ((rc = dalloc(ctx, &ctx->line_h, T.line_n))) return rc;
      ctx->line_cap = T.line_n;
    }
    T.line_e = ctx->line_e; T.line_h = ctx->line_h;
    ctx->line_src = (T.lo[0] + 2 * xo - 1) / 2 - 10 + kLinePad;
  }
  ctx->tfsf = *s;
  ctx->has_tfsf = 1;
  CK(cudaStreamSynchronize(ctx->stream));
  return DTMX_OK;
}

extern "C" int dtmx_add_probe(dtmx_ctx* ctx, int comp, int i, int j, int k, int mode, int* id_out) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || comp < 0 || comp > 5 || (mode != DTMX_PROBE_NODE && mode != DTMX_PROBE_REFERENCE)) return fail(ctx, DTMX_ERR_INVALID, "bad probe");
  if (i < 0 || i >= ctx->cfg.nx || j < 0 || j >= ctx->cfg.ny || k < 0 || k >= ctx->cfg.nz) return fail(ctx, DTMX_ERR_INVALID, "probe outside the grid");
  if (ctx->prepared) return fail(ctx, DTMX_ERR_STATE, "probes must be added before the first step");
  ProbeDev p{comp, i, j, k, mode};
  ctx->probes.push_back(p);
  if (id_out) *id_out = (int)ctx->probes.size() - 1;
  return DTMX_OK;
}

extern "C" int dtmx_read_probes(dtmx_ctx* ctx, float* out, int max_samples, int* nsamples) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || !out || max_samples < 0) return fail(ctx, DTMX_ERR_INVALID, "bad arguments");
  const int every = ctx->cfg.probe_every > 0 ? ctx->cfg.probe_every : 1;
  const long long have = std::min<long long>(ctx->step / every, ctx->probe_cap);
  const int ns = (int)std::min<long long>(have, max_samples);
  CK(cudaStreamSynchronize(ctx->stream));
  if (ns > 0 && !ctx->probes.empty())
    CK(cudaMemcpy2D(out, (size_t)max_samples * 4, ctx->d_traces, (size_t)ctx->probe_cap * 4, (size_t)ns * 4,
                    ctx->probes.size(), cudaMemcpyDeviceToHost));
  if (nsamples) *nsamples = ns;
  return DTMX_OK;
}

extern "C" int dtmx_add_dft_patch(dtmx_ctx* ctx, int axis, int index, int lo1, int n1, int lo2, int n2, int comp_mask,
                                  int nfreq, const double* omegas, int* id_out) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || axis < 0 || axis > 2 || nfreq < 1 || nfreq > 64 || !omegas || (comp_mask & ~63) || !comp_mask)
    return fail(ctx, DTMX_ERR_INVALID, "bad DFT plane");
  const int n[3] = {ctx->cfg.nx, ctx->cfg.ny, ctx->cfg.nz};
  const int e1 = n[axis == 0 ? 1 : 0], e2 = n[axis == 2 ? 1 : 2];
  if (index < 0 || index >= n[axis]) return fail(ctx, DTMX_ERR_INVALID, "DFT plane index out of range");
  if (lo1 < 0 || n1 < 1 || lo1 + n1 > e1 || lo2 < 0 || n2 < 1 || lo2 + n2 > e2)
    return fail(ctx, DTMX_ERR_INVALID, "DFT patch outside the plane");
  if (ctx->prepared) return fail(ctx, DTMX_ERR_STATE, "DFT planes must be added before the first step");
  DftHost h{};
  h.d.axis = axis; h.d.index = index; h.d.comp_mask = comp_mask; h.d.nfreq = nfreq;
  h.d.lo1 = lo1; h.d.n1 = n1;
  h.d.lo2 = lo2; h.d.n2 = n2;
  h.ncomp = __builtin_popcount(comp_mask);
  const size_t nacc = (size_t)h.ncomp * nfreq * h.d.n1 * h.d.n2;
  if (cudaMalloc(&h.omega, nfreq * sizeof(double)) != cudaSuccess) return fail(ctx, DTMX_ERR_OOM, "DFT allocation");
  const size_t nstage = (size_t)DFT_STAGE * h.ncomp * h.d.n1 * h.d.n2;
  if (cudaMalloc(&h.acc, nacc * sizeof(double2)) != cudaSuccess || cudaMalloc(&h.stage, nstage * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h.sstep, DFT_STAGE * sizeof(long long)) != cudaSuccess) {
    cudaFree(h.omega); cudaFree(h.acc); cudaFree(h.stage); cudaFree(h.sstep);
    return fail(ctx, DTMX_ERR_OOM, "DFT allocation");
  }
  CK(cudaMemsetAsync(h.acc, 0, nacc * sizeof(double2), ctx->stream));
  CK(cudaMemcpyAsync(h.omega, omegas, nfreq * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  h.d.omega = h.omega; h.d.acc = h.acc; h.d.stage = h.stage; h.d.sstep = h.sstep;
  ctx->dfts.push_back(h);
  CK(cudaStreamSynchronize(ctx->stream));
  if (id_out) *id_out = (int)ctx->dfts.size() - 1;
  return DTMX_OK;
}

extern "C" int dtmx_add_dft_plane(dtmx_ctx* ctx, int axis, int index, int comp_mask, int nfreq, const double* omegas, int* id_out) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || axis < 0 || axis > 2) return fail(ctx, DTMX_ERR_INVALID, "bad DFT plane");
  const int n[3] = {ctx->cfg.nx, ctx->cfg.ny, ctx->cfg.nz};
  return dtmx_add_dft_patch(ctx, axis, index, 0, n[axis == 0 ? 1 : 0], 0, n[axis == 2 ? 1 : 2], comp_mask, nfreq, omegas,
                            id_out);
}

extern "C" int dtmx_add_flux_box(dtmx_ctx* ctx, const int lo[3], const int hi[3], int nfreq, const double* omegas,
                                 int* id_out) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || !lo || !hi) return fail(ctx, DTMX_ERR_INVALID, "bad flux box");
  const int n[3] = {ctx->cfg.nx, ctx->cfg.ny, ctx->cfg.nz};
  const double ds[3] = {ctx->cfg.dx, ctx->cfg.dy, ctx->cfg.dz};
  for (int a = 0; a < 3; a++)
    if (lo[a] < 0 || hi[a] <= lo[a] || hi[a] + 1 >= n[a]) return fail(ctx, DTMX_ERR_INVALID, "flux box outside the grid");
  FluxHost fx{};
  fx.nfreq = nfreq;
  for (int a = 0; a < 3; a++) {
    // in-plane axes in (slow, fast) order and the tangential components
    const int s1 = a == 0 ? 1 : 0, s2 = a == 2 ? 1 : 2;
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    const int mask = (1 << b) | (1 << c) | (1 << (3 + b)) | (1 << (3 + c));
    for (int side = 0; side < 2; side++) {
      int id = -1;
      const int rc = dtmx_add_dft_patch(ctx, a, side ? hi[a] : lo[a], lo[s1], hi[s1] - lo[s1], lo[s2], hi[s2] - lo[s2],
                                        mask, nfreq, omegas, &id);
      if (rc) return rc;
      fx.face[2 * a + side] = id;
      fx.sgn_area[2 * a + side] = (side ? 1.0 : -1.0) * ds[s1] * ds[s2];
      const int w = side ? hi[a] : lo[a];
      const int n1 = hi[s1] - lo[s1] + 1, n2 = hi[s2] - lo[s2] + 1;
      int eid = -1, hid = -1;
      int rc2 = dtmx_add_dft_patch(ctx, a, w, lo[s1], n1, lo[s2], n2, mask, nfreq, omegas, &eid);
      if (!rc2)
        rc2 = dtmx_add_dft_patch(ctx, a, w + 1, lo[s1], n1, lo[s2], n2, (1 << (3 + b)) | (1 << (3 + c)), nfreq,
                                 omegas, &hid);
      if (rc2) return rc2;
      fx.ffe[2 * a + side] = eid;
      fx.ffh[2 * a + side] = hid;
    }
  }
  if (cudaMalloc(&fx.d_out, (size_t)6 * nfreq * sizeof(double)) != cudaSuccess)
    return fail(ctx, DTMX_ERR_OOM, "flux box allocation");
  ctx->fluxes.push_back(fx);
  if (id_out) *id_out = (int)ctx->fluxes.size() - 1;
  return DTMX_OK;
}

extern "C" int dtmx_flux_faces(dtmx_ctx* ctx, int id, int faces[6]) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || id < 0 || id >= (int)ctx->fluxes.size() || !faces) return fail(ctx, DTMX_ERR_INVALID, "bad flux box id");
  for (int q = 0; q < 6; q++) faces[q] = ctx->fluxes[id].face[q];
  return DTMX_OK;
}

// fold the staged samples of one DFT plane into its accumulators
static void dft_flush(dtmx_ctx* ctx, DftHost& h) {
  if (h.nstaged == 0) return;
  const long long npts = (long long)h.d.n1 * h.d.n2;
  dft_flush_kernel<<<(unsigned)((npts + 255) / 256), 256, 0, ctx->stream>>>(h.d, h.nstaged, ctx->cfg.dt);
  ctx->launches++;
  h.nstaged = 0;
}

extern "C" int dtmx_read_dft(dtmx_ctx* ctx, int id, double* out, size_t out_len) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || id < 0 || id >= (int)ctx->dfts.size() || !out) return fail(ctx, DTMX_ERR_INVALID, "bad DFT id");
  DftHost& h = ctx->dfts[id];
  const size_t n = (size_t)h.ncomp * h.d.nfreq * h.d.n1 * h.d.n2 * 2;
  if (out_len < n) return fail(ctx, DTMX_ERR_INVALID, "output buffer too small");
  dft_flush(ctx, h);
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(out, h.acc, n * sizeof(double), cudaMemcpyDeviceToHost));
  return DTMX_OK;
}

extern "C" int dtmx_read_flux(dtmx_ctx* ctx, int id, double* out, size_t out_len) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || id < 0 || id >= (int)ctx->fluxes.size() || !out) return fail(ctx, DTMX_ERR_INVALID, "bad flux box id");
  FluxHost& fx = ctx->fluxes[id];
  const int nf = fx.nfreq;
  if (out_len < (size_t)7 * nf) return fail(ctx, DTMX_ERR_INVALID, "output buffer too small");
  for (int q = 0; q < 6; q++) {
    DftHost& h = ctx->dfts[fx.face[q]];
    dft_flush(ctx, h);
    flux_face_kernel<<<nf, FLUX_THREADS, 0, ctx->stream>>>(h.d, fx.sgn_area[q], fx.d_out + (size_t)q * nf);
    ctx->launches++;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(out, fx.d_out, (size_t)6 * nf * sizeof(double), cudaMemcpyDeviceToHost));
  for (int f = 0; f < nf; f++) {
    double t = 0.0;
    for (int q = 0; q < 6; q++) t += out[(size_t)q * nf + f];
    out[(size_t)6 * nf + f] = t;
  }
  return DTMX_OK;
}

extern "C" int dtmx_ntff(dtmx_ctx* ctx, int id, int ndir, const double* theta, const double* phi, const double* origin,
                         double* out, size_t out_len) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || id < 0 || id >= (int)ctx->fluxes.size() || ndir < 1 || !theta || !phi || !out)
    return fail(ctx, DTMX_ERR_INVALID, "bad far-field arguments");
  FluxHost& fx = ctx->fluxes[id];
  const int nf = fx.nfreq;
  if (out_len < (size_t)ndir * nf * 5) return fail(ctx, DTMX_ERR_INVALID, "output buffer too small");
  NtffFaces F{};
  const double ds[3] = {ctx->cfg.dx, ctx->cfg.dy, ctx->cfg.dz};
  for (int q = 0; q < 6; q++) {
    DftHost& h = ctx->dfts[fx.ffe[q]];
    dft_flush(ctx, h);
    F.f[q] = h.d;
    DftHost& h2 = ctx->dfts[fx.ffh[q]];
    dft_flush(ctx, h2);
    F.h[q] = h2.d;
  }
  for (int a = 0; a < 3; a++) {
    F.ds[a] = ds[a];
    F.lo[a] = F.f[2 * a].index;
    F.hi[a] = F.f[2 * a + 1].index;
    // default origin: the centre of the E surface (box lo + 1/2 .. hi + 1/2)
    F.org[a] = origin ? origin[a] : (0.5 * (F.lo[a] + F.hi[a]) + 0.5) * ds[a];
  }
  double *dth = nullptr, *dph = nullptr, *dout = nullptr;
  const size_t nout = (size_t)ndir * nf * 5;
  if (cudaMalloc(&dth, ndir * 8) != cudaSuccess || cudaMalloc(&dph, ndir * 8) != cudaSuccess ||
      cudaMalloc(&dout, nout * 8) != cudaSuccess) {
    cudaFree(dth); cudaFree(dph); cudaFree(dout);
    return fail(ctx, DTMX_ERR_OOM, "far-field allocation");
  }
  CK(cudaMemcpyAsync(dth, theta, ndir * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dph, phi, ndir * 8, cudaMemcpyHostToDevice, ctx->stream));
  ntff_kernel<<<dim3(ndir, nf), FLUX_THREADS, 0, ctx->stream>>>(F, dth, dph, nf, dout);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, nout * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(dth); cudaFree(dph); cudaFree(dout);
  if (e != cudaSuccess) return fail(ctx, DTMX_ERR_CUDA, std::string("far field: ") + cudaGetErrorString(e));
  return DTMX_OK;
}

// ---------------------------------------------------------------- stepping
static int xchunk_for(const dtmx_ctx* ctx) {
  if (ctx->xchunk > 0) return ctx->xchunk;
  const dtmx_config& c = ctx->cfg;
  const long long tiles = (long long)((c.nz + TZ - 1) / TZ) * ((c.ny + TYT - 1) / TYT);
  const long long target = 148LL * 8 * 3;   // about three waves of 8 CTAs per SM
  long long chunks = std::max<long long>(1, (target + tiles - 1) / tiles);
  long long xc = (c.nx + chunks - 1) / chunks;
  // at most 10 planes per CTA: the autotuner picks 8-10 on 384^3 and
  // 1024x1024x1536 grids (longer chunks leave the tail of each CTA alone on its SM)
  return (int)std::min<long long>(10, std::max<long long>(4, xc));
}

static int set_kernel_attributes() {
  static bool done = false;
  if (done) return 0;
  cudaFuncSetAttribute(h_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Pipe<2, true>::SMEM_BYTES);
  cudaFuncSetAttribute(h_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Pipe<4, true>::SMEM_BYTES);
  cudaFuncSetAttribute(e_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Pipe<2, false>::SMEM_BYTES);
  cudaFuncSetAttribute(e_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Pipe<4, false>::SMEM_BYTES);
  done = true;
  return 0;
}

static int launch_step(dtmx_ctx* ctx) {
  set_kernel_attributes();
  const dtmx_config& c = ctx->cfg;
  Params P = ctx->P;
  P.x0 = 0; P.x1 = c.nx;
  P.xchunk = xchunk_for(ctx);
  const dim3 blk(TZ, TW);
  const dim3 grd((c.nz + TZ - 1) / TZ, (c.ny + TYT - 1) / TYT, (c.nx + P.xchunk - 1) / P.xchunk);
  const bool o4 = c.order == 4;
  cudaStream_t st = ctx->stream;
  const bool pw = ctx->has_tfsf && ctx->tfsf.kind == DTMX_TFSF_PLANE_X;
  long long nl = 0;
  if (ctx->profiling) cudaEventRecord(ctx->ev[0], st);
  if (o4) h_kernel<4><<<grd, blk, Pipe<4, true>::SMEM_BYTES, st>>>(P, ctx->maps);
  else h_kernel<2><<<grd, blk, Pipe<2, true>::SMEM_BYTES, st>>>(P, ctx->maps);
  if (ctx->profiling) cudaEventRecord(ctx->ev[1], st);
  nl++;
  dim3 tgrid[2];
  for (int hs = 0; hs < 2 && ctx->has_tfsf; hs++) {
    long long mx = 1;
    for (int r = 0; r < ctx->T.njob[hs]; r++) mx = std::max(mx, ctx->T.job[hs][r].cells);
    tgrid[hs] = dim3((unsigned)((mx + 255) / 256), std::max(1, ctx->T.njob[hs]));
  }
  if (ctx->has_tfsf) {
    if (o4) tfsf_kernel<4><<<tgrid[1], 256, 0, st>>>(P, ctx->T, ctx->d_step, 1);
    else tfsf_kernel<2><<<tgrid[1], 256, 0, st>>>(P, ctx->T, ctx->d_step, 1);
    nl++;
  }
  const double r1 = c.dt / c.dx;
  if (pw) {
    if (o4) line_h_kernel<4><<<8, 256, 0, st>>>(ctx->line_e, ctx->line_h, ctx->T.line_n, r1);
    else line_h_kernel<2><<<8, 256, 0, st>>>(ctx->line_e, ctx->line_h, ctx->T.line_n, r1);
    nl++;
  }
  const dim3 ablk(32, 8), agrd((P.ade.n[2] + 31) / 32, (P.ade.n[1] + 7) / 8, std::max(1, P.ade.n[0]));
  if (ctx->has_gyro) {
    gyro_current_kernel<<<agrd, ablk, 0, st>>>(P, ctx->gcur);
    P.ade.gnew = 1 - ctx->gcur;
    ctx->gcur = 1 - ctx->gcur;
    nl++;
  }
  if (ctx->profiling) cudaEventRecord(ctx->ev[2], st);
  if (o4) e_kernel<4><<<grd, blk, Pipe<4, false>::SMEM_BYTES, st>>>(P, ctx->maps);
  else e_kernel<2><<<grd, blk, Pipe<2, false>::SMEM_BYTES, st>>>(P, ctx->maps);
  if (P.ade.Em[0] || ctx->has_gyro) {
    // dispersive and gyrotropic nodes of the E half step (e_kernel skipped them)
    const bool box = c.geometry == DTMX_GEOM_BOX;
    if (o4) { if (box) ade_node_kernel<4, true><<<agrd, ablk, 0, st>>>(P); else ade_node_kernel<4, false><<<agrd, ablk, 0, st>>>(P); }
    else { if (box) ade_node_kernel<2, true><<<agrd, ablk, 0, st>>>(P); else ade_node_kernel<2, false><<<agrd, ablk, 0, st>>>(P); }
    nl++;
  }
  if (ctx->profiling) {
    cudaEventRecord(ctx->ev[3], st);
    // read back this step's two kernel durations (keeps the events reusable)
    cudaEventSynchronize(ctx->ev[3]);
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&b, ctx->ev[2], ctx->ev[3]);
    ctx->prof_ms_h += a; ctx->prof_ms_e += b; ctx->prof_count++;
  }
  nl++;
  if (!ctx->psrc.empty()) {
    point_source_kernel<<<((int)ctx->psrc.size() + 63) / 64, 64, 0, st>>>(P, ctx->d_psrc, (int)ctx->psrc.size(), ctx->d_step, c.dt);
    nl++;
  }
  if (ctx->has_tfsf) {
    if (o4) tfsf_kernel<4><<<tgrid[0], 256, 0, st>>>(P, ctx->T, ctx->d_step, 0);
    else tfsf_kernel<2><<<tgrid[0], 256, 0, st>>>(P, ctx->T, ctx->d_step, 0);
    nl++;
  }
  if (pw) {
    const dtmx_tfsf& s = ctx->tfsf;
    if (o4) line_e_kernel<4><<<8, 256, 0, st>>>(ctx->line_e, ctx->line_h, ctx->T.line_n, r1, ctx->line_src, ctx->d_step, c.dt, s.amp, s.f0, s.tau, s.t0);
    else line_e_kernel<2><<<8, 256, 0, st>>>(ctx->line_e, ctx->line_h, ctx->T.line_n, r1, ctx->line_src, ctx->d_step, c.dt, s.amp, s.f0, s.tau, s.t0);
    nl++;
  }
  if (!ctx->probes.empty() && !ctx->monitors_off) {
    const int every = c.probe_every > 0 ? c.probe_every : 1;
    probe_kernel<<<((int)ctx->probes.size() + 127) / 128, 128, 0, st>>>(P, ctx->d_probes, (int)ctx->probes.size(), ctx->d_traces,
                                                                       ctx->probe_cap, ctx->d_step, every);
    nl++;
  }
  for (auto& d : ctx->dfts) {
    if (ctx->monitors_off) break;
    const long long npts = (long long)d.d.n1 * d.d.n2;
    dft_capture_kernel<<<(unsigned)((npts + 255) / 256), 256, 0, st>>>(P, d.d, ctx->d_step, d.nstaged);
    nl++;
    if (++d.nstaged == DFT_STAGE) dft_flush(ctx, d);
  }
  if (ctx->obj_on) {
    DftHost& d = ctx->obj;
    const long long npts = (long long)d.d.n1 * d.d.n2;
    dft_capture_kernel<<<(unsigned)((npts + 255) / 256), 256, 0, st>>>(P, d.d, ctx->d_step, d.nstaged);
    nl++;
    if (++d.nstaged == DFT_STAGE) dft_flush(ctx, d);
  }
  advance_step_kernel<<<1, 1, 0, st>>>(ctx->d_step);
  nl++;
  ctx->launches += nl;
  return DTMX_OK;
}

// First-step preparation: upload the source and probe lists, allocate the
// probe traces and check the TF/SF shell against the materials.
static int prepare(dtmx_ctx* ctx) {
  if (ctx->prepared) return DTMX_OK;
  int rc;
  if (!ctx->psrc.empty()) {
    if ((rc = dalloc(ctx, &ctx->d_psrc, ctx->psrc.size(), true))) return rc;
    CK(cudaMemcpyAsync(ctx->d_psrc, ctx->psrc.data(), ctx->psrc.size() * sizeof(PointSrcDev), cudaMemcpyHostToDevice, ctx->stream));
  }
  if (!ctx->probes.empty()) {
    if ((rc = dalloc(ctx, &ctx->d_probes, ctx->probes.size(), true))) return rc;
    CK(cudaMemcpyAsync(ctx->d_probes, ctx->probes.data(), ctx->probes.size() * sizeof(ProbeDev), cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = dalloc(ctx, &ctx->d_traces, ctx->probes.size() * (size_t)ctx->probe_cap))) return rc;
  }
  if (ctx->has_tfsf && ctx->h_mat[0].size()) {
    // every E node that gets a correction, and the E nodes next to them, must be non-dispersive
    const TfsfDev& T = ctx->T;
    for (int r = 0; r < T.njob[0]; r++) {
      const TfsfJob& jb = T.job[0][r];
      for (int i = std::max(0, jb.lo[0] - 1); i <= std::min(ctx->cfg.nx - 1, jb.hi[0] + 1); i++)
        for (int j = std::max(0, jb.lo[1] - 1); j <= std::min(ctx->cfg.ny - 1, jb.hi[1] + 1); j++)
          for (int k = std::max(0, jb.lo[2] - 1); k <= std::min(ctx->cfg.nz - 1, jb.hi[2] + 1); k++)
            for (int comp = 0; comp < 3; comp++)
              if (ctx->mats[ctx->h_mat[comp][store_index(ctx, i, j, k)]].npoles > 0 ||
                  ctx->mats[ctx->h_mat[comp][store_index(ctx, i, j, k)]].gyro_wp > 0)
                return fail(ctx, DTMX_ERR_UNSUPPORTED, "dispersive or gyrotropic material on the TF/SF surface");
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->prepared = true;
  return DTMX_OK;
}

// ---------------------------------------------------------------- wavefront engine
constexpr int TORRE_TY = 32;

static int build_torre_maps(dtmx_ctx* ctx) {
  if (ctx->tmaps_ok) return DTMX_OK;
  const int R2 = ctx->cfg.order - 1, TY = TORRE_TY;
  TorreMaps& m = ctx->tmaps;
  int rc;
  for (int h = 0; h < 2; h++) {
    const int c0 = 3 * h;
    if ((rc = make_map(ctx, &m.A[h], ctx->P.f[c0], false, 40, TY + R2))) return rc;
    if ((rc = make_map(ctx, &m.B[h], ctx->P.f[c0 + 1], false, 40, TY))) return rc;
    if ((rc = make_map(ctx, &m.C[h], ctx->P.f[c0 + 2], false, 32, TY + R2))) return rc;
  }
  for (int c = 0; c < 6; c++)
    if ((rc = make_map(ctx, &m.core[c], ctx->P.f[c], false, 32, TY))) return rc;
  for (int c = 0; c < 3; c++)
    if ((rc = make_map(ctx, &m.mat[c], ctx->d_mat[c], true, 32, TY))) return rc;
  ctx->tmaps_ok = true;
  return DTMX_OK;
}

using TorreFn = void (*)(const Params, const TorreMaps, const TorreArgs);

static TorreFn torre_fn(int order, int T, size_t* smem, int* nthr) {
  constexpr int TY = TORRE_TY;
#define DTMX_TORRE_CASE(O, TT)                                                         \
  if (order == O && T == TT) {                                                          \
    *smem = TorreLayout<O, TY>::SMEM; *nthr = TorreLayout<O, TY>::NTHR;                 \
    return torre_kernel<O, 2 * TT, TY>;                                                 \
  }
  DTMX_TORRE_CASE(2, 1) DTMX_TORRE_CASE(2, 2) DTMX_TORRE_CASE(2, 3) DTMX_TORRE_CASE(2, 4)
  DTMX_TORRE_CASE(4, 1) DTMX_TORRE_CASE(4, 2)
#undef DTMX_TORRE_CASE
  return nullptr;
}

// Can the wavefront engine run this context with T steps per launch?
static bool torre_usable(dtmx_ctx* ctx, int T, std::string* why) {
  const dtmx_config& c = ctx->cfg;
  size_t smem = 0;
  int nthr = 0;
  TorreFn fn = torre_fn(c.order, T, &smem, &nthr);
  if (!fn) { *why = "no kernel for order " + std::to_string(c.order) + " with " + std::to_string(T) + " steps per launch"; return false; }
  if (c.geometry != DTMX_GEOM_BOX) { *why = "needs the box geometry"; return false; }
  if (c.absorber == DTMX_ABS_SPLIT_PML) { *why = "split PML is not supported"; return false; }
  if (ctx->has_gyro) { *why = "gyrotropic materials need a current pass between half steps"; return false; }
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    *why = "shared memory attribute refused";
    return false;
  }
  int per_sm = 0, nsm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, nthr, smem) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->dev) != cudaSuccess) {
    cudaGetLastError();
    *why = "occupancy query failed";
    return false;
  }
  const long long tiles = (long long)((c.nz + TT_Z - 1) / TT_Z) * ((c.ny + TORRE_TY - 1) / TORRE_TY);
  if (tiles > (long long)per_sm * nsm) {
    *why = std::to_string(tiles) + " tiles exceed the " + std::to_string(per_sm * nsm) + " co-resident CTAs";
    return false;
  }
  return true;
}

// features the wavefront engine does not carry inside its launch
static bool torre_features_ok(const dtmx_ctx* ctx, std::string* why) {
  if (ctx->has_gyro) { *why = "gyrotropic materials"; return false; }
  if (ctx->has_tfsf) { *why = "TF/SF source"; return false; }
  if (!ctx->psrc.empty()) { *why = "point sources"; return false; }
  if (!ctx->probes.empty()) { *why = "probes"; return false; }
  if (!ctx->dfts.empty()) { *why = "DFT planes"; return false; }
  return true;
}

__global__ void advance_step_by_kernel(long long* d_step, int n) { *d_step += n; }

static int launch_torre(dtmx_ctx* ctx, int T) {
  const dtmx_config& c = ctx->cfg;
  int rc = build_torre_maps(ctx);
  if (rc) return rc;
  size_t smem = 0;
  int nthr = 0;
  TorreFn fn = torre_fn(c.order, T, &smem, &nthr);
  const int ntz = (c.nz + TT_Z - 1) / TT_Z, nty = (c.ny + TORRE_TY - 1) / TORRE_TY;
  if (!ctx->d_ctr && (rc = dalloc(ctx, &ctx->d_ctr, (size_t)ntz * nty))) return rc;
  CK(cudaMemsetAsync(ctx->d_ctr, 0, sizeof(int) * ntz * nty, ctx->stream));
  Params P = ctx->P;
  P.x0 = 0; P.x1 = c.nx;
  TorreArgs ta;
  ta.ctr = ctx->d_ctr; ta.ntz = ntz; ta.nty = nty;
  ta.nsteps = c.nx + (c.order == 4 ? TorreGeom<4>::off(2 * T - 1) : TorreGeom<2>::off(2 * T - 1));
  void* args[] = {(void*)&P, (void*)&ctx->tmaps, (void*)&ta};
  if (ctx->profiling) cudaEventRecord(ctx->ev[0], ctx->stream);
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)fn, dim3(ntz, nty), dim3(nthr), args, smem, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, DTMX_ERR_CUDA, std::string("wavefront launch: ") + cudaGetErrorString(e));
  if (ctx->profiling) {
    cudaEventRecord(ctx->ev[1], ctx->stream);
    cudaEventSynchronize(ctx->ev[1]);
    float a = 0;
    cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
    ctx->prof_ms_h += a; ctx->prof_count += T;
  }
  advance_step_by_kernel<<<1, 1, 0, ctx->stream>>>(ctx->d_step, T);
  ctx->launches += 2;
  ctx->step += T;
  return DTMX_OK;
}

// ---------------------------------------------------------------- single-sweep engine
// Applies to the box geometry with the Yee stencil and a CPML or no absorber;
// everything else the per-step engine covers.
static bool fused_usable(const dtmx_ctx* ctx, std::string* why) {
  const dtmx_config& c = ctx->cfg;
  if (c.geometry != DTMX_GEOM_BOX) { if (why) *why = "box geometry only"; return false; }
  if (c.order != 2) { if (why) *why = "order 2 only"; return false; }
  if (c.absorber == DTMX_ABS_SPLIT_PML) { if (why) *why = "no split PML"; return false; }
  return true;
}

template <int NR>
static int build_fused_maps(dtmx_ctx* ctx, FusedMaps& fm, float* const* f) {
  using L = FL<NR>;
  int rc;
  for (int c = 0; c < 3; c++) {
    if ((rc = make_map(ctx, &fm.e[c], f[c], false, FE_W, L::FE_R))) return rc;
    fm.mat[c] = ctx->maps.mat[c];
  }
  if ((rc = make_map(ctx, &fm.hx, f[3], false, FHX_W, L::FHX_R))) return rc;
  if ((rc = make_map(ctx, &fm.hy, f[4], false, FHY_W, L::FHY_R))) return rc;
  return make_map(ctx, &fm.hz, f[5], false, FHZ_W, L::FHZ_R);
}

// First use: the second buffer set, the maps reading each set, the tile table.
static int fused_prepare(dtmx_ctx* ctx) {
  if (ctx->fused_ready) return DTMX_OK;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(fused_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FL<2>::SMEM);
    cudaFuncSetAttribute(fused_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FL<1>::SMEM);
    attr = true;
  }
  const dtmx_config& c = ctx->cfg;
  int rc = DTMX_OK;
  for (int comp = 0; comp < 6 && !rc; comp++) rc = dalloc(ctx, &ctx->f_alt[comp], ctx->nstore + 64);
  for (int a = 0; a < 3 && !rc; a++) {
    const size_t th = (size_t)(ctx->P.ab.L[a][0] + ctx->P.ab.L[a][1]);
    if (!ctx->P.ab.aux[a][2] || !th) continue;
    const size_t cnt = th * (ctx->ncell / (size_t)(a == 0 ? c.nx : a == 1 ? c.ny : c.nz));
    for (int q = 0; q < 2 && !rc; q++) rc = dalloc(ctx, &ctx->hax_alt[a][q], cnt);
  }
  // maps of the per-step kernels over the second set, so either engine runs from either buffer
  if (!rc) {
    TmaMaps save = ctx->maps;
    float* fsave[6];
    for (int comp = 0; comp < 6; comp++) { fsave[comp] = ctx->P.f[comp]; ctx->P.f[comp] = ctx->f_alt[comp]; }
    rc = build_maps(ctx);
    ctx->maps_alt = ctx->maps;
    ctx->maps = save;
    for (int comp = 0; comp < 6; comp++) ctx->P.f[comp] = fsave[comp];
  }
  if (!rc) rc = build_fused_maps<2>(ctx, ctx->fmaps[0], ctx->P.f);
  if (!rc) rc = build_fused_maps<2>(ctx, ctx->fmaps[1], ctx->f_alt);
  if (!rc) rc = build_fused_maps<1>(ctx, ctx->fmaps8[0], ctx->P.f);
  if (!rc) rc = build_fused_maps<1>(ctx, ctx->fmaps8[1], ctx->f_alt);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->fused_ready = true;
  return DTMX_OK;
}

// The state now lives in the other buffer set: swap the pointers (fields, H
// auxiliaries, the maps reading them) so that P and every pass see it.
static void fused_swap(dtmx_ctx* ctx) {
  for (int comp = 0; comp < 6; comp++) std::swap(ctx->P.f[comp], ctx->f_alt[comp]);
  for (int a = 0; a < 3; a++)
    for (int q = 0; q < 2; q++) std::swap(ctx->P.ab.aux[a][2 + q], ctx->hax_alt[a][q]);
  std::swap(ctx->maps, ctx->maps_alt);
  std::swap(ctx->fmaps[0], ctx->fmaps[1]);
  std::swap(ctx->fmaps8[0], ctx->fmaps8[1]);
  ctx->parity ^= 1;
  ctx->tmaps_ok = false;          // the wavefront engine's maps are rebuilt for the current buffer
}

// planes per CTA (at most FX_MAX): about eight waves of 3 CTAs per SM, and
// at least 8 planes (each chunk stages one plane and updates one H plane more)
static int fused_xchunk_for(const dtmx_ctx* ctx) {
  if (ctx->xchunk > 0) return std::min(ctx->xchunk, FX_MAX);
  const dtmx_config& c = ctx->cfg;
  const long long tiles = (long long)((c.nz + TZ - 1) / TZ) * ((c.ny + ctx->frows - 1) / ctx->frows);
  const long long target = 148LL * 3 * 8;
  const long long chunks = std::max<long long>(1, (target + tiles - 1) / tiles);
  const long long xc = (c.nx + chunks - 1) / chunks;
  return (int)std::min<long long>(32, std::max<long long>(8, xc));
}

// One time step of the single-sweep engine: the side passes that act on the
// old state (TF/SF H correction, gyrotropic current), the sweep A -> B, the
// passes on the new state (dispersive nodes, sources, TF/SF E correction,
// monitors), then the buffer swap.
static int launch_fused_step(dtmx_ctx* ctx) {
  int rc = fused_prepare(ctx);
  if (rc) return rc;
  const dtmx_config& c = ctx->cfg;
  Params PA = ctx->P;
  PA.x0 = 0; PA.x1 = c.nx;
  PA.xchunk = fused_xchunk_for(ctx);
  Params PB = PA;
  FusedArgs fa{};
  for (int comp = 0; comp < 6; comp++) { PB.f[comp] = ctx->f_alt[comp]; fa.dst[comp] = ctx->f_alt[comp]; }
  for (int a = 0; a < 3; a++)
    for (int q = 0; q < 2; q++) {
      fa.hsrc[a][q] = PA.ab.aux[a][2 + q];
      fa.hdst[a][q] = ctx->hax_alt[a][q];
      PB.ab.aux[a][2 + q] = ctx->hax_alt[a][q];
    }
  cudaStream_t st = ctx->stream;
  const bool pw = ctx->has_tfsf && ctx->tfsf.kind == DTMX_TFSF_PLANE_X;
  long long nl = 0;
  dim3 tgrid[2];
  for (int hs = 0; hs < 2 && ctx->has_tfsf; hs++) {
    long long mx = 1;
    for (int r = 0; r < ctx->T.njob[hs]; r++) mx = std::max(mx, ctx->T.job[hs][r].cells);
    tgrid[hs] = dim3((unsigned)((mx + 255) / 256), std::max(1, ctx->T.njob[hs]));
  }
  // TF/SF correction of H, added to the old H (the H update is linear in it)
  if (ctx->has_tfsf) { tfsf_kernel<2><<<tgrid[1], 256, 0, st>>>(PA, ctx->T, ctx->d_step, 1); nl++; }
  const double r1 = c.dt / c.dx;
  if (pw) { line_h_kernel<2><<<8, 256, 0, st>>>(ctx->line_e, ctx->line_h, ctx->T.line_n, r1); nl++; }
  const dim3 ablk(32, 8), agrd((PA.ade.n[2] + 31) / 32, (PA.ade.n[1] + 7) / 8, std::max(1, PA.ade.n[0]));
  if (ctx->has_gyro) {
    gyro_current_kernel<<<agrd, ablk, 0, st>>>(PA, ctx->gcur);
    PA.ade.gnew = PB.ade.gnew = 1 - ctx->gcur;
    ctx->gcur = 1 - ctx->gcur;
    nl++;
  }
  const dim3 blk(TZ, TW), grd((c.nz + TZ - 1) / TZ, (c.ny + ctx->frows - 1) / ctx->frows, (c.nx + PA.xchunk - 1) / PA.xchunk);
  if (ctx->profiling) cudaEventRecord(ctx->ev[0], st);
  if (ctx->frows == 8) fused_kernel<1><<<grd, blk, FL<1>::SMEM, st>>>(PA, fa, ctx->fmaps8[0]);
  else fused_kernel<2><<<grd, blk, FL<2>::SMEM, st>>>(PA, fa, ctx->fmaps[0]);
  if (ctx->profiling) cudaEventRecord(ctx->ev[1], st);
  nl++;
  if (PA.ade.Em[0] || ctx->has_gyro) {
    // dispersive nodes (left by the sweep) from the old E in A; E -= dt/eps_inf J on gyrotropic nodes
    for (int comp = 0; comp < 3; comp++) PB.fe_old[comp] = PA.f[comp];
    ade_node_kernel<2, true><<<agrd, ablk, 0, st>>>(PB);
    nl++;
  }
  if (ctx->profiling) {
    cudaEventSynchronize(ctx->ev[1]);
    float a = 0;
    cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
    ctx->prof_ms_h += a; ctx->prof_count++;
  }
  if (!ctx->psrc.empty()) {
    point_source_kernel<<<((int)ctx->psrc.size() + 63) / 64, 64, 0, st>>>(PB, ctx->d_psrc, (int)ctx->psrc.size(), ctx->d_step, c.dt);
    nl++;
  }
  if (ctx->has_tfsf) { tfsf_kernel<2><<<tgrid[0], 256, 0, st>>>(PB, ctx->T, ctx->d_step, 0); nl++; }
  if (pw) {
    const dtmx_tfsf& s = ctx->tfsf;
    line_e_kernel<2><<<8, 256, 0, st>>>(ctx->line_e, ctx->line_h, ctx->T.line_n, r1, ctx->line_src, ctx->d_step, c.dt, s.amp, s.f0, s.tau, s.t0);
    nl++;
  }
  if (!ctx->probes.empty() && !ctx->monitors_off) {
    const int every = c.probe_every > 0 ? c.probe_every : 1;
    probe_kernel<<<((int)ctx->probes.size() + 127) / 128, 128, 0, st>>>(PB, ctx->d_probes, (int)ctx->probes.size(), ctx->d_traces,
                                                                       ctx->probe_cap, ctx->d_step, every);
    nl++;
  }
  for (auto& d : ctx->dfts) {
    if (ctx->monitors_off) break;
    const long long npts = (long long)d.d.n1 * d.d.n2;
    dft_capture_kernel<<<(unsigned)((npts + 255) / 256), 256, 0, st>>>(PB, d.d, ctx->d_step, d.nstaged);
    nl++;
    if (++d.nstaged == DFT_STAGE) dft_flush(ctx, d);
  }
  if (ctx->obj_on) {
    DftHost& d = ctx->obj;
    const long long npts = (long long)d.d.n1 * d.d.n2;
    dft_capture_kernel<<<(unsigned)((npts + 255) / 256), 256, 0, st>>>(PB, d.d, ctx->d_step, d.nstaged);
    nl++;
    if (++d.nstaged == DFT_STAGE) dft_flush(ctx, d);
  }
  advance_step_kernel<<<1, 1, 0, st>>>(ctx->d_step);
  nl++;
  ctx->launches += nl;
  fused_swap(ctx);
  return DTMX_OK;
}

// one time step of the selected per-step engine (per-step or single sweep)
static int launch_one(dtmx_ctx* ctx) { return ctx->engine == 3 ? launch_fused_step(ctx) : launch_step(ctx); }

// Capture (once per field buffer) and launch 16 per-step launch sequences as
// one graph.  The host-side bookkeeping of the 16 steps (staging slots,
// flushes, buffer parities) is done during the capture; the captured kernels
// read the step number from the device counter, so the graph is valid at
// every 16-step boundary of an aligned run that starts from the same buffer
// (16 single-sweep steps come back to it).
static int graph_steps16(dtmx_ctx* ctx) {
  const int par = ctx->parity;
  if (!ctx->graph16[par]) {
    set_kernel_attributes();
    if (ctx->engine == 3) { int rc = fused_prepare(ctx); if (rc) return rc; }
    const long long launches0 = ctx->launches;
    const int gcur0 = ctx->gcur;
    std::vector<int> staged0;
    for (auto& d : ctx->dfts) staged0.push_back(d.nstaged);
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return fail(ctx, DTMX_ERR_CUDA, "graph capture could not start");
    int rc = DTMX_OK;
    for (int q = 0; q < 16 && !rc; q++) rc = launch_one(ctx);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc || e != cudaSuccess) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return rc ? rc : fail(ctx, DTMX_ERR_CUDA, "graph capture failed"); }
    e = cudaGraphInstantiate(&ctx->graph16[par], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { ctx->graph16[par] = nullptr; cudaGetLastError(); return fail(ctx, DTMX_ERR_CUDA, "graph instantiation failed"); }
    // the capture ran the bookkeeping of 16 steps; the graph below executes them
    if (ctx->gcur != gcur0 || ctx->parity != par) return fail(ctx, DTMX_ERR_STATE, "graph capture: unexpected buffer parity");
    for (size_t q = 0; q < ctx->dfts.size(); q++)
      if (ctx->dfts[q].nstaged != staged0[q]) return fail(ctx, DTMX_ERR_STATE, "graph capture: staging not aligned");
    ctx->graph_launches[par] = ctx->launches - launches0;
  } else {
    ctx->launches += ctx->graph_launches[par];
  }
  CK(cudaGraphLaunch(ctx->graph16[par], ctx->stream));
  ctx->step += 16;
  return DTMX_OK;
}

extern "C" int dtmx_step(dtmx_ctx* ctx, int nsteps) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || nsteps < 0) return fail(ctx, DTMX_ERR_INVALID, "bad step count");
  int rc0 = prepare(ctx);
  if (rc0) return rc0;
  int left = nsteps;
  if (ctx->engine == 2) {
    std::string why;
    if (!torre_features_ok(ctx, &why)) return fail(ctx, DTMX_ERR_UNSUPPORTED, "wavefront engine: " + why);
    while (left >= ctx->tblock) {
      int rc = launch_torre(ctx, ctx->tblock);
      if (rc) return rc;
      left -= ctx->tblock;
    }
  }
  if (ctx->engine == 3) {
    std::string why;
    if (!fused_usable(ctx, &why)) return fail(ctx, DTMX_ERR_UNSUPPORTED, "single-sweep engine: " + why);
  }
  while (left > 0) {
    // 16 steps as one CUDA graph when every DFT staging cycle is at its start
    // (the captured sequence then repeats exactly: staging slots, the flush
    // every 16 steps and the gyrotropic buffer parity)
    bool aligned = left >= 16 && !ctx->profiling && !ctx->monitors_off && ctx->engine != 2;
    for (auto& d : ctx->dfts) aligned = aligned && d.nstaged == 0;
    if (ctx->obj_on) aligned = aligned && ctx->obj.nstaged == 0;
    if (aligned && !ctx->obj_on) {
      int rc = graph_steps16(ctx);
      if (rc) return rc;
      left -= 16;
      continue;
    }
    int rc = ctx->engine == 2 ? launch_step(ctx) : launch_one(ctx);
    if (rc) return rc;
    ctx->step++;
    left--;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ctx, DTMX_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return DTMX_OK;
}

// ---------------------------------------------------------------- design region and adjoint
extern "C" int dtmx_set_design(dtmx_ctx* ctx, const int* lo, const int* n, const float* eps) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || !lo || !n || !eps) return fail(ctx, DTMX_ERR_INVALID, "bad design region");
  const dtmx_config& c = ctx->cfg;
  const int dim[3] = {c.nx, c.ny, c.nz};
  for (int a = 0; a < 3; a++)
    if (n[a] < 1 || lo[a] < 0 || lo[a] + n[a] > dim[a]) return fail(ctx, DTMX_ERR_INVALID, "design region outside the grid");
  if (ctx->prepared) return fail(ctx, DTMX_ERR_STATE, "the design region must be set before the first step");
  const size_t nd = (size_t)n[0] * n[1] * n[2];
  for (int comp = 0; comp < 3; comp++) {
    ctx->h_des_ie[comp].resize(nd);
    for (size_t q = 0; q < nd; q++) {
      const float e = eps[comp * nd + q];
      if (!(e > 0)) return fail(ctx, DTMX_ERR_INVALID, "design permittivity must be > 0");
      ctx->h_des_ie[comp][q] = (float)(1.0 / (double)e);
    }
  }
  for (int comp = 0; comp < 3; comp++) {
    if (ctx->d_des_ie[comp] && (size_t)ctx->P.des_n[0] * ctx->P.des_n[1] * ctx->P.des_n[2] != nd) ctx->d_des_ie[comp] = nullptr;
    int rc;
    if (!ctx->d_des_ie[comp] && (rc = dalloc(ctx, &ctx->d_des_ie[comp], nd))) return rc;
    CK(cudaMemcpyAsync(ctx->d_des_ie[comp], ctx->h_des_ie[comp].data(), nd * 4, cudaMemcpyHostToDevice, ctx->stream));
    ctx->P.des_ie[comp] = ctx->d_des_ie[comp];
  }
  for (int a = 0; a < 3; a++) { ctx->P.des_lo[a] = lo[a]; ctx->P.des_n[a] = n[a]; }
  ctx->P.des_on = 1;
  return upload_umat(ctx);
}

// device buffers that make up the restartable state of a context
static void state_parts(dtmx_ctx* ctx, std::vector<std::pair<void*, size_t>>& parts) {
  parts.clear();
  for (int comp = 0; comp < 6; comp++) parts.push_back({ctx->P.f[comp], ctx->nstore * 4});
  for (int a = 0; a < 3; a++) {
    const size_t cnt = (size_t)(ctx->P.ab.L[a][0] + ctx->P.ab.L[a][1]) * (ctx->ncell / (size_t)ctx->P.g.n[a]);
    for (int q = 0; q < 4; q++)
      if (ctx->P.ab.aux[a][q]) parts.push_back({ctx->P.ab.aux[a][q], cnt * 4});
  }
  const Ade& A = ctx->P.ade;
  const size_t na = (size_t)A.n[0] * A.n[1] * A.n[2];
  for (int comp = 0; comp < 3 && na; comp++) {
    if (A.Em[comp]) parts.push_back({A.Em[comp], na * 4});
    for (int q = 0; q < MAXPOLE; q++) {
      if (A.Jp[comp][q]) parts.push_back({A.Jp[comp][q], na * 4});
      if (A.Jm[comp][q]) parts.push_back({A.Jm[comp][q], na * 4});
    }
    for (int b = 0; b < 2; b++)
      if (A.Jg[b][comp]) parts.push_back({A.Jg[b][comp], na * 4});
  }
  parts.push_back({ctx->d_step, sizeof(long long)});
  if (ctx->line_e) {
    parts.push_back({ctx->line_e, (size_t)ctx->T.line_n * 8});
    parts.push_back({ctx->line_h, (size_t)ctx->T.line_n * 8});
  }
}

static int state_copy(dtmx_ctx* ctx, char* ck, bool save) {
  std::vector<std::pair<void*, size_t>> parts;
  state_parts(ctx, parts);
  size_t off = 0;
  for (auto& pr : parts) {
    if (save) CK(cudaMemcpyAsync(ck + off, pr.first, pr.second, cudaMemcpyDeviceToDevice, ctx->stream));
    else CK(cudaMemcpyAsync(pr.first, ck + off, pr.second, cudaMemcpyDeviceToDevice, ctx->stream));
    off += (pr.second + 255) / 256 * 256;
  }
  return DTMX_OK;
}

static size_t state_bytes(dtmx_ctx* ctx) {
  std::vector<std::pair<void*, size_t>> parts;
  state_parts(ctx, parts);
  size_t off = 0;
  for (auto& pr : parts) off += (pr.second + 255) / 256 * 256;
  return off;
}

// Forward + adjoint run of one context, split into phases so that a batch of
// contexts can interleave them step by step (each context on its own stream).
struct FaRun {
  int N = 0, K = 0, nseg = 0, nd = 0, npl = 0, plane_x = 0;
  double omega = 0, J = 0;
  long long s0 = 0;
  int gcur0 = 0;              // gyrotropic current buffer at the start (it alternates every step)
  std::vector<char*> ck;
  AdjDev A{};
  float* hist = nullptr;
  double* dF = nullptr;
  int seg = -1, len = 0;
  bool full = false;          // the forward pass records the whole design history: no checkpoints, no recompute
  cudaStream_t st = nullptr;
  std::vector<void*> bufs;
  // Device buffers of the run come from the device's stream-ordered pool:
  // released blocks stay in the pool (release threshold raised once per
  // process), so later runs -- on this context or a fresh one -- reuse them
  // without a device-wide synchronisation.
  void* take(dtmx_ctx* ctx, size_t bytes) {
    static const bool pool_kept = [] {
      int dev = 0;
      cudaMemPool_t pool;
      if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return false;
      uint64_t keep = ~0ull;
      return cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess;
    }();
    (void)pool_kept;
    st = ctx->stream;
    void* q = nullptr;
    if (cudaMallocAsync(&q, bytes, ctx->stream) != cudaSuccess) return nullptr;
    bufs.push_back(q);
    return q;
  }
  void release() {
    for (void* q : bufs) cudaFreeAsync(q, st);
    bufs.clear();
    ck.clear();
  }
};

// Does the design-region E history of a whole run fit the context's budget?
// Then the forward pass records it and the adjoint needs no recomputation.
static double fa_history_bytes(const dtmx_ctx* ctx, int nsteps) {
  const Params& P = ctx->P;
  return (double)(nsteps + 1) * 3.0 * P.des_n[0] * P.des_n[1] * P.des_n[2] * 4.0;
}
static double free_device_bytes() {
  size_t fr = 0, tot = 0;
  return cudaMemGetInfo(&fr, &tot) == cudaSuccess ? (double)fr : 0.0;
}
static bool fa_history_fits(dtmx_ctx* ctx, int nsteps) {
  const double bytes = fa_history_bytes(ctx, nsteps);
  if (ctx->adj_budget >= 0) return bytes <= (double)ctx->adj_budget;
  return bytes <= 0.25 * free_device_bytes();
}

static int fa_begin(dtmx_ctx* ctx, FaRun& R, int nsteps, int checkpoint_every, int plane_x, double omega, bool full) {
  const dtmx_config& c = ctx->cfg;
  Params& P = ctx->P;
  if (nsteps < 1 || checkpoint_every < 1) return fail(ctx, DTMX_ERR_INVALID, "bad arguments");
  if (!P.des_on) return fail(ctx, DTMX_ERR_STATE, "no design region");
  if (plane_x < 0 || plane_x >= c.nx) return fail(ctx, DTMX_ERR_INVALID, "objective plane outside the grid");
  if (c.geometry != DTMX_GEOM_BOX || c.absorber == DTMX_ABS_SPLIT_PML)
    return fail(ctx, DTMX_ERR_UNSUPPORTED, "the adjoint needs the box geometry with CPML or no absorber");
  if (ctx->has_gyro && !ctx->h_mat[0].empty()) {
    // the design permittivity of a gyrotropic node would enter next to its current: not carried
    for (int comp = 0; comp < 3; comp++)
      for (int i = P.des_lo[0]; i < P.des_lo[0] + P.des_n[0]; i++)
        for (int j = P.des_lo[1]; j < P.des_lo[1] + P.des_n[1]; j++)
          for (int k = P.des_lo[2]; k < P.des_lo[2] + P.des_n[2]; k++)
            if (ctx->mats[ctx->h_mat[comp][store_index(ctx, i, j, k)]].gyro_wp > 0)
              return fail(ctx, DTMX_ERR_UNSUPPORTED, "the design region holds a gyrotropic node");
  }
  for (const auto& q : ctx->psrc) {
    const long long sz = ctx->nzp, sy = (long long)c.ny * sz;
    const int i = (int)(q.id / sy), j = (int)((q.id % sy) / sz), k = (int)(q.id % sz);
    if (design_index(P, i, j, k) >= 0) return fail(ctx, DTMX_ERR_INVALID, "a point source lies in the design region");
  }
  int rc = prepare(ctx);
  if (rc) return rc;
  R.full = full;
  R.N = nsteps; R.K = full ? nsteps : std::min(checkpoint_every, nsteps);
  R.nseg = (R.N + R.K - 1) / R.K;
  R.nd = P.des_n[0] * P.des_n[1] * P.des_n[2];
  R.npl = c.ny * c.nz;
  R.plane_x = plane_x; R.omega = omega;
  // objective flux DFT on the plane x = plane_x: Ey, Ez, Hy, Hz at omega
  DftHost& O = ctx->obj;
  if (!O.acc || O.d.index != plane_x) {
    cudaFree(O.omega); cudaFree(O.acc); cudaFree(O.stage); cudaFree(O.sstep);
    O = DftHost{};
    O.d.axis = 0; O.d.index = plane_x; O.d.comp_mask = (1 << 1) | (1 << 2) | (1 << 4) | (1 << 5); O.d.nfreq = 1;
    O.d.n1 = c.ny; O.d.n2 = c.nz; O.ncomp = 4;
    if (cudaMalloc(&O.omega, 8) != cudaSuccess || cudaMalloc(&O.acc, (size_t)4 * R.npl * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&O.stage, (size_t)DFT_STAGE * 4 * R.npl * 4) != cudaSuccess || cudaMalloc(&O.sstep, DFT_STAGE * 8) != cudaSuccess)
      return fail(ctx, DTMX_ERR_OOM, "objective DFT allocation");
    O.d.omega = O.omega; O.d.acc = O.acc; O.d.stage = O.stage; O.d.sstep = O.sstep;
  }
  CK(cudaMemcpyAsync(O.omega, &omega, 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(O.acc, 0, (size_t)4 * R.npl * sizeof(double2), ctx->stream));
  O.nstaged = 0;
  if (full) {
    // design-region history of every step: slot s holds E after s steps of the run
    void* h = R.take(ctx, (size_t)(R.N + 1) * 3 * R.nd * 4);
    if (!h) return fail(ctx, DTMX_ERR_OOM, "design history allocation");
    R.hist = (float*)h;
  } else {
    // checkpoints of the state every K steps plus the final state
    const size_t sb = state_bytes(ctx);
    R.ck.assign(R.nseg + 1, nullptr);
    for (auto& q : R.ck)
      if (!(q = (char*)R.take(ctx, sb))) { R.release(); return fail(ctx, DTMX_ERR_OOM, "checkpoint allocation"); }
  }
  R.s0 = ctx->step;
  R.gcur0 = ctx->gcur;
  ctx->obj_on = true;
  return DTMX_OK;
}

static unsigned design_blocks(const FaRun& R) { return (unsigned)((3 * R.nd + 255) / 256); }

// forward step st (0-based) of the run
static int fa_forward(dtmx_ctx* ctx, FaRun& R, int st) {
  if (R.full) {
    if (st == 0) {
      design_capture_kernel<<<design_blocks(R), 256, 0, ctx->stream>>>(ctx->P, R.hist, 0, R.nd);
      ctx->launches++;
    }
  } else if (st % R.K == 0) {
    state_copy(ctx, R.ck[st / R.K], true);
  }
  int rc = launch_one(ctx);
  if (rc) return rc;
  ctx->step++;
  if (R.full) {
    design_capture_kernel<<<design_blocks(R), 256, 0, ctx->stream>>>(ctx->P, R.hist, st + 1, R.nd);
    ctx->launches++;
  }
  return DTMX_OK;
}

// end of the forward pass: objective, adjoint buffers (waits for the stream)
static int fa_forward_done(dtmx_ctx* ctx, FaRun& R) {
  Params& P = ctx->P;
  ctx->obj_on = false;
  if (!R.full) state_copy(ctx, R.ck[R.nseg], true);
  DftHost& O = ctx->obj;
  dft_flush(ctx, O);
  std::vector<double> F((size_t)8 * R.npl);
  CK(cudaMemcpyAsync(F.data(), O.acc, F.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  double J = 0;
  for (int u = 0; u < R.npl; u++) {
    const double *ey = &F[(0 * (size_t)R.npl + u) * 2], *ez = &F[(1 * (size_t)R.npl + u) * 2];
    const double *hy = &F[(2 * (size_t)R.npl + u) * 2], *hz = &F[(3 * (size_t)R.npl + u) * 2];
    J += ey[0] * hz[0] + ey[1] * hz[1] - (ez[0] * hy[0] + ez[1] * hy[1]);
  }
  R.J = J;
  AdjDev& A = R.A;
  A = AdjDev{};
  A.nd = R.nd;
  auto talloc = [&](void** q, size_t bytes) {
    if (!(*q = R.take(ctx, bytes))) return false;
    return cudaMemsetAsync(*q, 0, bytes, ctx->stream) == cudaSuccess;
  };
  bool ok = true;
  for (int comp = 0; comp < 6; comp++) ok = ok && talloc((void**)&A.lam[comp], (ctx->nstore + 64) * 4);
  for (int a = 0; a < 3; a++) {
    const size_t cnt = (size_t)(P.ab.L[a][0] + P.ab.L[a][1]) * (ctx->ncell / (size_t)P.g.n[a]);
    if (!P.ab.aux[a][0]) continue;
    for (int q = 0; q < 4; q++) ok = ok && talloc((void**)&A.lpsi[a][q], cnt * 4);
  }
  for (int c3 = 0; c3 < 3; c3++)
    for (int t = 0; t < 2; t++) ok = ok && talloc((void**)&A.w[c3][t], (ctx->nstore + 64) * 4);
  if (ctx->has_gyro) {
    const size_t na = (size_t)P.ade.n[0] * P.ade.n[1] * P.ade.n[2];
    for (int c3 = 0; c3 < 3; c3++) ok = ok && talloc((void**)&A.lJg[c3], na * 4) && talloc((void**)&A.lT[c3], na * 4);
  }
  if (P.ade.Em[0]) {
    // adjoint of the ADE state, over the ADE box
    const size_t na = (size_t)P.ade.n[0] * P.ade.n[1] * P.ade.n[2];
    for (int c3 = 0; c3 < 3; c3++) {
      ok = ok && talloc((void**)&A.lEm[c3], na * 4);
      for (int r = 0; r < MAXPOLE; r++)
        if (P.ade.Jp[c3][r]) ok = ok && talloc((void**)&A.lJp[c3][r], na * 4) && talloc((void**)&A.lJm[c3][r], na * 4);
    }
  }
  ok = ok && talloc((void**)&A.grad, (size_t)3 * R.nd * 8) && talloc((void**)&R.dF, F.size() * 8);
  if (!R.full) ok = ok && talloc((void**)&R.hist, (size_t)(R.K + 1) * 3 * R.nd * 4);
  if (!ok) { R.release(); return fail(ctx, DTMX_ERR_OOM, "adjoint allocation"); }
  A.hist = R.hist;
  CK(cudaMemcpyAsync(R.dF, F.data(), F.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->monitors_off = true;
  return DTMX_OK;
}

// restore checkpoint seg and record the design region of its first state
// (with the whole history recorded: the one segment is the run, nothing to restore)
static int fa_segment_begin(dtmx_ctx* ctx, FaRun& R, int seg) {
  R.seg = seg;
  const int start = seg * R.K;
  R.len = std::min(R.N, start + R.K) - start;
  if (R.full) return DTMX_OK;
  state_copy(ctx, R.ck[seg], false);
  ctx->step = R.s0 + start;
  ctx->gcur = R.gcur0 ^ (start & 1);
  design_capture_kernel<<<design_blocks(R), 256, 0, ctx->stream>>>(ctx->P, R.hist, 0, R.nd);
  return DTMX_OK;
}

// recompute step q (1..len) of the current segment
static int fa_recompute(dtmx_ctx* ctx, FaRun& R, int q) {
  if (R.full) return DTMX_OK;
  int rc = launch_one(ctx);
  if (rc) return rc;
  ctx->step++;
  design_capture_kernel<<<design_blocks(R), 256, 0, ctx->stream>>>(ctx->P, R.hist, q, R.nd);
  return DTMX_OK;
}

// adjoint of step q (len..1) of the current segment
static int fa_adjoint(dtmx_ctx* ctx, FaRun& R, int q) {
  const Params& P = ctx->P;
  const dtmx_config& c = ctx->cfg;
  AdjDev& A = R.A;
  cudaStream_t st = ctx->stream;
  adj_source_kernel<<<(R.npl + 255) / 256, 256, 0, st>>>(P, A, R.dF, R.s0 + (long long)R.seg * R.K + q, R.plane_x, R.omega, c.dt);
  adj_grad_kernel<<<design_blocks(R), 256, 0, st>>>(P, A, q);
  const dim3 blk(32, 8), grd((c.nz + 31) / 32, (c.ny + 7) / 8, c.nx);
  const dim3 wgrd((c.nz + 31) / 32, (c.ny + 7) / 8, (c.nx + ADJ_XP - 1) / ADJ_XP);   // adj_w: ADJ_XP planes per thread
  // the dispersive nodes' transposed ADE recursion replaces their w (after adj_w, before adj_curl);
  // the gyrotropic current's transposition reads lam_E' (after adj_w) and gathers over the box
  const bool ade = P.ade.Em[0] != nullptr;
  const bool gyro = ctx->has_gyro;
  const dim3 ablk(32, 8), agrd((P.ade.n[2] + 31) / 32, (P.ade.n[1] + 7) / 8, std::max(1, P.ade.n[0]));
  if (c.order == 4) {
    adj_w_kernel<4, 0><<<wgrd, blk, 0, st>>>(P, A);
    if (ade) adj_ade_kernel<<<agrd, ablk, 0, st>>>(P, A);
    if (gyro) { adj_gyro_mu_kernel<<<agrd, ablk, 0, st>>>(P, A); adj_gyro_j_kernel<<<agrd, ablk, 0, st>>>(P, A); }
    adj_curl_kernel<4, 0><<<grd, blk, 0, st>>>(P, A);
    adj_w_kernel<4, 1><<<wgrd, blk, 0, st>>>(P, A);
    adj_curl_kernel<4, 1><<<grd, blk, 0, st>>>(P, A);
    ctx->launches += 6 + (ade ? 1 : 0) + (gyro ? 2 : 0);
  } else {
    adj_w_kernel<2, 0><<<wgrd, blk, 0, st>>>(P, A);
    if (ade) adj_ade_kernel<<<agrd, ablk, 0, st>>>(P, A);
    if (gyro) { adj_gyro_mu_kernel<<<agrd, ablk, 0, st>>>(P, A); adj_gyro_j_kernel<<<agrd, ablk, 0, st>>>(P, A); }
    adj_curl_kernel<2, 0><<<grd, blk, 0, st>>>(P, A);
    adj_w_kernel<2, 1><<<wgrd, blk, 0, st>>>(P, A);
    adj_curl_kernel<2, 1><<<grd, blk, 0, st>>>(P, A);
    ctx->launches += 6 + (ade ? 1 : 0) + (gyro ? 2 : 0);
  }
  return DTMX_OK;
}

// final state back in place, gradient to the caller (waits for the stream)
static int fa_finish(dtmx_ctx* ctx, FaRun& R, double* objective, float* grad_eps) {
  ctx->monitors_off = false;
  if (!R.full) state_copy(ctx, R.ck[R.nseg], false);
  ctx->step = R.s0 + R.N;
  ctx->gcur = R.gcur0 ^ (R.N & 1);
  std::vector<double> g((size_t)3 * R.nd);
  CK(cudaMemcpyAsync(g.data(), R.A.grad, g.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  R.release();
  if (e != cudaSuccess) return fail(ctx, DTMX_ERR_CUDA, std::string("adjoint: ") + cudaGetErrorString(e));
  for (int comp = 0; comp < 3; comp++)
    for (int q = 0; q < R.nd; q++) {
      const double ie = ctx->h_des_ie[comp][q];
      grad_eps[(size_t)comp * R.nd + q] = (float)(-ie * ie * g[(size_t)comp * R.nd + q]);
    }
  *objective = R.J;
  return DTMX_OK;
}

static void fa_abort(dtmx_ctx* ctx, FaRun& R) {
  cudaStreamSynchronize(ctx->stream);
  ctx->obj_on = false;
  ctx->monitors_off = false;
  R.release();
}

extern "C" int dtmx_forward_adjoint(dtmx_ctx* ctx, int nsteps, int checkpoint_every, int plane_x, double omega,
                                    double* objective, float* grad_eps) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || !objective || !grad_eps) return fail(ctx, DTMX_ERR_INVALID, "bad arguments");
  FaRun R;
  if (nsteps < 1 || checkpoint_every < 1) return fail(ctx, DTMX_ERR_INVALID, "bad arguments");
  int rc = fa_begin(ctx, R, nsteps, checkpoint_every, plane_x, omega, fa_history_fits(ctx, nsteps));
  if (rc) return rc;
  for (int st = 0; st < R.N && !rc; st++) rc = fa_forward(ctx, R, st);
  if (!rc) rc = fa_forward_done(ctx, R);
  for (int seg = R.nseg - 1; seg >= 0 && !rc; seg--) {
    fa_segment_begin(ctx, R, seg);
    for (int q = 1; q <= R.len && !rc; q++) rc = fa_recompute(ctx, R, q);
    for (int q = R.len; q >= 1 && !rc; q--) rc = fa_adjoint(ctx, R, q);
  }
  if (rc) { fa_abort(ctx, R); return rc; }
  return fa_finish(ctx, R, objective, grad_eps);
}

extern "C" int dtmx_set_adjoint_memory(dtmx_ctx* ctx, int64_t bytes) {
  if (!ctx) return DTMX_ERR_INVALID;
  ctx->adj_budget = bytes < 0 ? -1 : (long long)bytes;
  return DTMX_OK;
}

// Batch of independent forward + adjoint runs: every phase is issued for all
// contexts step by step, each context on its own stream, so that the GPU runs
// the instances' kernels concurrently (instances of uneven sizes fill each
// other's gaps) and no instance waits on the host between its steps.
extern "C" int dtmx_batch_forward_adjoint(dtmx_ctx* const* ctxs, int n, int nsteps, int checkpoint_every,
                                          const int* plane_x, const double* omega, double* objectives,
                                          float* const* grads) {
  if (!ctxs || n < 1 || !plane_x || !omega || !objectives || !grads) return DTMX_ERR_INVALID;
  for (int b = 0; b < n; b++)
    if (ctxs[b] && ctxs[b]->parked) return fail(ctxs[b], DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  std::vector<FaRun> R(n);
  int rc = DTMX_OK;
  auto abort_all = [&](int upto) {
    for (int b = 0; b < upto; b++) fa_abort(ctxs[b], R[b]);
  };
  // one mode for the whole batch (the segments advance in lock step)
  bool full = nsteps >= 1;
  double total = 0.0;
  bool automatic = true;
  for (int b = 0; b < n; b++) {
    full = full && ctxs[b] && fa_history_fits(ctxs[b], nsteps);
    if (!full) break;
    total += fa_history_bytes(ctxs[b], nsteps);
    automatic = automatic && ctxs[b]->adj_budget < 0;
  }
  if (full && automatic) full = total <= 0.25 * free_device_bytes();
  for (int b = 0; b < n; b++)
    if ((rc = fa_begin(ctxs[b], R[b], nsteps, checkpoint_every, plane_x[b], omega[b], full))) { abort_all(b); return rc; }
  for (int st = 0; st < nsteps && !rc; st++)
    for (int b = 0; b < n && !rc; b++) rc = fa_forward(ctxs[b], R[b], st);
  for (int b = 0; b < n && !rc; b++) rc = fa_forward_done(ctxs[b], R[b]);
  const int nseg = R[0].nseg;
  for (int seg = nseg - 1; seg >= 0 && !rc; seg--) {
    for (int b = 0; b < n; b++) fa_segment_begin(ctxs[b], R[b], seg);
    const int len = R[0].len;
    for (int q = 1; q <= len && !rc; q++)
      for (int b = 0; b < n && !rc; b++) rc = fa_recompute(ctxs[b], R[b], q);
    for (int q = len; q >= 1 && !rc; q--)
      for (int b = 0; b < n && !rc; b++) rc = fa_adjoint(ctxs[b], R[b], q);
  }
  if (rc) { abort_all(n); return rc; }
  for (int b = 0; b < n; b++) {
    int r = fa_finish(ctxs[b], R[b], &objectives[b], grads[b]);
    if (r && !rc) rc = r;
  }
  return rc;
}

// ---------------------------------------------------------------- autotuner
// Times every applicable engine configuration for trial_steps steps from the
// current state (monitors paused, state restored after each trial) and keeps
// the fastest: the per-step engine with x chunks of {auto, 4, 8, 16, 32, 64}
// planes per CTA, and the wavefront engine with 1, 2 and 4 steps per launch.
// Results are cached per grid shape and feature set for the process.
struct TuneKey {
  int nx, ny, nz, order, absorber, geometry, feats;
  bool operator<(const TuneKey& o) const {
    return std::tie(nx, ny, nz, order, absorber, geometry, feats) < std::tie(o.nx, o.ny, o.nz, o.order, o.absorber, o.geometry, o.feats);
  }
};
struct TuneVal { int engine, tblock, xchunk; double ms; int rows = 16; };
static std::map<TuneKey, TuneVal>& tune_cache() {
  static std::map<TuneKey, TuneVal> m;
  return m;
}

extern "C" int dtmx_autotune(dtmx_ctx* ctx, int trial_steps, int* engine_out, int* tblock_out, int* xchunk_out,
                             double* ms_per_step_out) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || trial_steps < 1) return fail(ctx, DTMX_ERR_INVALID, "bad arguments");
  int rc = prepare(ctx);
  if (rc) return rc;
  const dtmx_config& c = ctx->cfg;
  const int feats = (ctx->has_tfsf ? 1 : 0) | (ctx->psrc.empty() ? 0 : 2) | (ctx->probes.empty() ? 0 : 4) |
                    (ctx->dfts.empty() ? 0 : 8) | (ctx->P.ade.Em[0] ? 16 : 0) | (ctx->has_gyro ? 32 : 0) |
                    (ctx->P.des_on ? 64 : 0);
  const TuneKey key{c.nx, c.ny, c.nz, c.order, c.absorber, c.geometry, feats};
  TuneVal best{1, 0, 0, 1e30};
  auto it = tune_cache().find(key);
  if (it != tune_cache().end()) {
    best = it->second;
  } else {
    char* ck = nullptr;
    if (cudaMalloc(&ck, state_bytes(ctx)) != cudaSuccess) return fail(ctx, DTMX_ERR_OOM, "autotune state copy");
    state_copy(ctx, ck, true);
    const long long step0 = ctx->step;
    const int gcur0 = ctx->gcur, eng0 = ctx->engine, tb0 = ctx->tblock, xc0 = ctx->xchunk, fr0 = ctx->frows;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<TuneVal> cand;
    for (int xc : {0, 4, 6, 8, 10, 12, 16, 24, 32, 64})
      if (xc <= c.nx) cand.push_back({1, 0, xc, 0});
    if (fused_usable(ctx, nullptr) && fused_prepare(ctx) == DTMX_OK)
      for (int rows : {16, 8})
        for (int xc : {0, 2, 4, 6, 8, 12, 16, 24, 32, 48, 64})
          if (xc <= c.nx) cand.push_back({3, 0, xc, 0, rows});
    std::string why;
    if (torre_features_ok(ctx, &why))
      for (int T : {1, 2, 4})
        if (trial_steps >= T && torre_usable(ctx, T, &why)) cand.push_back({2, T, 0, 0});
    ctx->monitors_off = true;
    for (auto& cd : cand) {
      ctx->xchunk = cd.xchunk;
      ctx->engine = cd.engine;
      ctx->frows = cd.rows;
      int r = DTMX_OK;
      const int n = cd.engine == 2 ? (trial_steps / cd.tblock) * cd.tblock : trial_steps;
      cudaEventRecord(e0, ctx->stream);
      if (cd.engine == 2) {
        for (int q = 0; q < n && !r; q += cd.tblock) r = launch_torre(ctx, cd.tblock);
      } else {
        for (int q = 0; q < n && !r; q++) { r = launch_one(ctx); ctx->step++; }
      }
      cudaEventRecord(e1, ctx->stream);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      cd.ms = r ? 1e30 : ms / n;
      if (r) cudaGetLastError();
      state_copy(ctx, ck, false);
      ctx->step = step0;
      ctx->gcur = gcur0;
      if (cd.ms < best.ms) best = cd;
    }
    ctx->monitors_off = false;
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(ck);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->engine = eng0; ctx->tblock = tb0; ctx->xchunk = xc0; ctx->frows = fr0;
    tune_cache()[key] = best;
  }
  ctx->engine = best.engine;
  ctx->tblock = best.tblock;
  ctx->xchunk = best.xchunk;
  ctx->frows = best.rows;
  drop_graphs(ctx);
  if (engine_out) *engine_out = best.engine;
  if (tblock_out) *tblock_out = best.tblock;
  if (xchunk_out) *xchunk_out = best.xchunk;
  if (ms_per_step_out) *ms_per_step_out = best.ms;
  return DTMX_OK;
}

// ---------------------------------------------------------------- field and state files
// Field snapshot in the reference's .arr layout (drop.cu:84-107): int32 header
// {12, 0, 0, 0, 3, sizeof(float), nz, ny, nx} (a 12-byte comment of zeros, the
// rank, the element size and the extents, fastest first), then the values
// with z fastest and x slowest; dense cells instead of the reference's one
// value per rag.
extern "C" int dtmx_write_arr(dtmx_ctx* ctx, int comp, const char* path) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || comp < 0 || comp > 5 || !path) return fail(ctx, DTMX_ERR_INVALID, "bad arguments");
  const dtmx_config& c = ctx->cfg;
  std::vector<float> buf((size_t)c.nx * c.ny * c.nz);
  int rc = dtmx_get_field(ctx, comp, buf.data());
  if (rc) return rc;
  FILE* f = fopen(path, "wb");
  if (!f) return fail(ctx, DTMX_ERR_INVALID, std::string("cannot open ") + path);
  const int32_t hdr[9] = {12, 0, 0, 0, 3, (int32_t)sizeof(float), c.nz, c.ny, c.nx};
  const bool ok = fwrite(hdr, sizeof(hdr), 1, f) == 1 && fwrite(buf.data(), 4, buf.size(), f) == buf.size();
  if (fclose(f) != 0 || !ok) return fail(ctx, DTMX_ERR_INVALID, std::string("write failed: ") + path);
  return DTMX_OK;
}

// Restartable state file: a header (magic, version, grid, order, geometry,
// absorber, step, byte count) and the device state of the context (fields,
// absorber and ADE state, step counter, plane-wave line), so that loading it
// into a context set up the same way and stepping on reproduces the saved run
// bit for bit.  Probe traces and DFT accumulators are not part of it.
struct StateHeader {
  char magic[8];
  int32_t version, nx, ny, nz, order, geometry, absorber, pad;
  int64_t step, bytes;
};

extern "C" int dtmx_save_state(dtmx_ctx* ctx, const char* path) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || !path) return fail(ctx, DTMX_ERR_INVALID, "bad arguments");
  int rc = prepare(ctx);
  if (rc) return rc;
  const size_t sb = state_bytes(ctx);
  char* dev = nullptr;
  if (cudaMalloc(&dev, sb) != cudaSuccess) return fail(ctx, DTMX_ERR_OOM, "state buffer");
  state_copy(ctx, dev, true);
  std::vector<char> host(sb);
  cudaError_t e = cudaMemcpyAsync(host.data(), dev, sb, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(dev);
  if (e != cudaSuccess) return fail(ctx, DTMX_ERR_CUDA, std::string("state copy: ") + cudaGetErrorString(e));
  const dtmx_config& c = ctx->cfg;
  StateHeader h{};
  memcpy(h.magic, "DTMXSTAT", 8);
  h.version = 1; h.nx = c.nx; h.ny = c.ny; h.nz = c.nz; h.order = c.order; h.geometry = c.geometry;
  h.absorber = c.absorber; h.step = ctx->step; h.bytes = (int64_t)sb;
  FILE* f = fopen(path, "wb");
  if (!f) return fail(ctx, DTMX_ERR_INVALID, std::string("cannot open ") + path);
  const bool ok = fwrite(&h, sizeof(h), 1, f) == 1 && fwrite(host.data(), 1, sb, f) == sb;
  if (fclose(f) != 0 || !ok) return fail(ctx, DTMX_ERR_INVALID, std::string("write failed: ") + path);
  return DTMX_OK;
}

extern "C" int dtmx_load_state(dtmx_ctx* ctx, const char* path) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || !path) return fail(ctx, DTMX_ERR_INVALID, "bad arguments");
  int rc = prepare(ctx);
  if (rc) return rc;
  FILE* f = fopen(path, "rb");
  if (!f) return fail(ctx, DTMX_ERR_INVALID, std::string("cannot open ") + path);
  StateHeader h{};
  const size_t sb = state_bytes(ctx);
  const dtmx_config& c = ctx->cfg;
  if (fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, "DTMXSTAT", 8) != 0 || h.version != 1) {
    fclose(f);
    return fail(ctx, DTMX_ERR_INVALID, "not a state file");
  }
  if (h.nx != c.nx || h.ny != c.ny || h.nz != c.nz || h.order != c.order || h.geometry != c.geometry ||
      h.absorber != c.absorber || h.bytes != (int64_t)sb) {
    fclose(f);
    return fail(ctx, DTMX_ERR_INVALID, "state file does not match this context (grid, scheme or state layout)");
  }
  std::vector<char> host(sb);
  const bool ok = fread(host.data(), 1, sb, f) == sb;
  fclose(f);
  if (!ok) return fail(ctx, DTMX_ERR_INVALID, "truncated state file");
  char* dev = nullptr;
  if (cudaMalloc(&dev, sb) != cudaSuccess) return fail(ctx, DTMX_ERR_OOM, "state buffer");
  cudaError_t e = cudaMemcpyAsync(dev, host.data(), sb, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) { state_copy(ctx, dev, false); e = cudaStreamSynchronize(ctx->stream); }
  cudaFree(dev);
  if (e != cudaSuccess) return fail(ctx, DTMX_ERR_CUDA, std::string("state copy: ") + cudaGetErrorString(e));
  ctx->step = h.step;
  // the host-side parity of the gyrotropic current buffers follows the step count
  if (ctx->has_gyro) ctx->gcur = (int)(h.step & 1);
  return DTMX_OK;
}

extern "C" int dtmx_sync(dtmx_ctx* ctx) {
  if (!ctx) return DTMX_ERR_INVALID;
  CK(cudaStreamSynchronize(ctx->stream));
  int err = 0;
  CK(cudaMemcpy(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    CK(cudaMemset(ctx->d_err, 0, sizeof(int)));
    return fail(ctx, DTMX_ERR_TIMEOUT, err == 2 ? "a wavefront tile waited too long for its neighbours"
                                                : "a staged load did not arrive in time");
  }
  return DTMX_OK;
}

extern "C" int dtmx_get_step(const dtmx_ctx* ctx, int64_t* n) {
  if (!ctx || !n) return DTMX_ERR_INVALID;
  *n = ctx->step;
  return DTMX_OK;
}

extern "C" int dtmx_get_field(dtmx_ctx* ctx, int comp, float* host_out) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || comp < 0 || comp > 5 || !host_out) return fail(ctx, DTMX_ERR_INVALID, "bad field request");
  const dtmx_config& c = ctx->cfg;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy2D(host_out, (size_t)c.nz * 4, ctx->P.f[comp], (size_t)ctx->nzp * 4, (size_t)c.nz * 4,
                  (size_t)c.nx * c.ny, cudaMemcpyDeviceToHost));
  return DTMX_OK;
}

extern "C" int dtmx_set_field(dtmx_ctx* ctx, int comp, const float* host_in) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || comp < 0 || comp > 5 || !host_in) return fail(ctx, DTMX_ERR_INVALID, "bad field request");
  const dtmx_config& c = ctx->cfg;
  CK(cudaMemcpy2DAsync(ctx->P.f[comp], (size_t)ctx->nzp * 4, host_in, (size_t)c.nz * 4, (size_t)c.nz * 4,
                       (size_t)c.nx * c.ny, cudaMemcpyHostToDevice, ctx->stream));
  // non-live nodes are held at zero
  mask_nonlive_kernel<<<148 * 4, 256, 0, ctx->stream>>>(ctx->P, comp, (long long)ctx->ncell);
  ctx->launches++;
  CK(cudaStreamSynchronize(ctx->stream));
  return DTMX_OK;
}

extern "C" int dtmx_field_device_ptr(dtmx_ctx* ctx, int comp, void** dptr, int64_t strides[3]) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx || comp < 0 || comp > 5 || !dptr) return fail(ctx, DTMX_ERR_INVALID, "bad field request");
  *dptr = ctx->P.f[comp];
  if (strides) { strides[0] = ctx->P.g.sx; strides[1] = ctx->P.g.sy; strides[2] = 1; }
  return DTMX_OK;
}

extern "C" int dtmx_check_finite(dtmx_ctx* ctx) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx) return DTMX_ERR_INVALID;
  CK(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  for (int comp = 0; comp < 6; comp++) {
    nonfinite_kernel<<<148 * 4, 256, 0, ctx->stream>>>(ctx->P, comp, (long long)ctx->ncell, ctx->d_flag);
    ctx->launches++;
  }
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return flag ? fail(ctx, DTMX_ERR_NONFINITE, "non-finite field value") : DTMX_OK;
}

extern "C" int dtmx_kernel_launches(const dtmx_ctx* ctx, int64_t* n) {
  if (!ctx || !n) return DTMX_ERR_INVALID;
  *n = ctx->launches;
  return DTMX_OK;
}

extern "C" int dtmx_set_engine(dtmx_ctx* ctx, int engine, int time_block) {
  if (!ctx || engine < 0 || engine > 3 || time_block < 0) return fail(ctx, DTMX_ERR_INVALID, "bad engine");
  if (engine == 3) {
    std::string why;
    if (!fused_usable(ctx, &why)) return fail(ctx, DTMX_ERR_UNSUPPORTED, "single-sweep engine: " + why);
    ctx->tblock = 0;
  } else if (engine == 2) {
    const int T = time_block > 0 ? time_block : 2;
    std::string why;
    if (!torre_usable(ctx, T, &why)) return fail(ctx, DTMX_ERR_UNSUPPORTED, "wavefront engine: " + why);
    ctx->tblock = T;
  } else {
    ctx->tblock = time_block;
  }
  ctx->engine = engine;
  drop_graphs(ctx);
  return DTMX_OK;
}

extern "C" int dtmx_park(dtmx_ctx* ctx) {
  if (!ctx) return DTMX_ERR_INVALID;
  if (!ctx->cfg.parkable) return fail(ctx, DTMX_ERR_STATE, "the context was not created parkable");
  if (ctx->parked) return DTMX_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  const VmmApi& A = vmm_api();
  for (auto& b : ctx->vmm) {
    // the single sweep's output buffers hold nothing between steps: every
    // node they carry is written by the next step (zero where no step writes)
    b.dead = false;
    for (int comp = 0; comp < 6; comp++) b.dead = b.dead || b.va == (CUdeviceptr)ctx->f_alt[comp];
    for (int a = 0; a < 3; a++)
      for (int q = 0; q < 2; q++) b.dead = b.dead || b.va == (CUdeviceptr)ctx->hax_alt[a][q];
    if (b.dead) continue;
    // arrays fixed once the context has stepped keep the host copy of an earlier park
    if (b.fixed && b.host && ctx->prepared && b.saved_prepared) continue;
    if (!b.host) CK(cudaMallocHost(&b.host, b.size));
    CK(cudaMemcpyAsync(b.host, (void*)b.va, b.size, cudaMemcpyDeviceToHost, ctx->stream));
    b.saved_prepared = ctx->prepared;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  for (auto& b : ctx->vmm) {
    if (A.unmap(b.va, b.size) != CUDA_SUCCESS || (!pool_put(ctx->dev, b.size, b.h) && A.release(b.h) != CUDA_SUCCESS))
      return fail(ctx, DTMX_ERR_CUDA, "releasing the device memory of a parked context");
    b.h = 0;
  }
  ctx->parked = true;
  return DTMX_OK;
}

extern "C" int dtmx_set_park_pool(int device, int64_t bytes) {
  if (device < 0 || device >= kPoolDevices) return DTMX_ERR_INVALID;
  const VmmApi& A = vmm_api();
  HandlePool& P = handle_pool(device);
  std::lock_guard<std::mutex> lk(P.mu);
  P.limit = bytes < 0 ? -1 : bytes;
  // release what the new limit does not hold, largest first
  while (P.limit >= 0 && P.bytes > (size_t)P.limit && !P.free.empty()) {
    auto it = std::prev(P.free.end());
    if (A.ok) A.release(it->second);
    P.bytes -= it->first;
    P.free.erase(it);
  }
  return DTMX_OK;
}

extern "C" int dtmx_unpark(dtmx_ctx* ctx) {
  if (!ctx) return DTMX_ERR_INVALID;
  if (!ctx->parked) return DTMX_OK;
  CK(cudaSetDevice(ctx->dev));
  for (size_t q = 0; q < ctx->vmm.size(); q++) {
    VmmBlock& b = ctx->vmm[q];
    if (vmm_back(ctx->dev, b) != CUDA_SUCCESS) {
      // keep the context consistent: release what was mapped again and stay parked
      const VmmApi& A = vmm_api();
      for (size_t r = 0; r < q; r++) { A.unmap(ctx->vmm[r].va, ctx->vmm[r].size); A.release(ctx->vmm[r].h); }
      return fail(ctx, DTMX_ERR_OOM, "device memory for an unparked context");
    }
  }
  for (auto& b : ctx->vmm) {
    if (b.dead) CK(cudaMemsetAsync((void*)b.va, 0, b.size, ctx->stream));
    else CK(cudaMemcpyAsync((void*)b.va, b.host, b.size, cudaMemcpyHostToDevice, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->parked = false;
  return DTMX_OK;
}

// ---- plane state: fields, y/z CPML auxiliaries and ADE state of x planes,
// section-major in a dense host layout (the same for every context with the
// same y/z configuration and material table, whatever its ADE box).
static int plane_poles(const dtmx_ctx* ctx) {
  int p = 0;
  for (int m = 0; m < ctx->nmat; m++) p = std::max(p, ctx->mats[m].npoles);
  return p;
}

static size_t plane_floats(const dtmx_ctx* ctx) {
  const dtmx_config& c = ctx->cfg;
  const size_t nyz = (size_t)c.ny * c.nz;
  size_t n = 6 * nyz;
  if (ctx->P.ab.aux[1][0]) n += 4 * (size_t)(ctx->P.ab.L[1][0] + ctx->P.ab.L[1][1]) * c.nz;
  if (ctx->P.ab.aux[2][0]) n += 4 * (size_t)c.ny * (ctx->P.ab.L[2][0] + ctx->P.ab.L[2][1]);
  return n + (size_t)3 * (1 + 2 * plane_poles(ctx)) * nyz;
}

static int plane_refusal(dtmx_ctx* ctx) {
  if (ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (ctx->cfg.geometry != DTMX_GEOM_BOX || ctx->cfg.absorber == DTMX_ABS_SPLIT_PML)
    return fail(ctx, DTMX_ERR_UNSUPPORTED, "plane state: box geometry with a CPML or no absorber only");
  // (a TF/SF line is not per plane either, but every slab integrates the same one)
  if (ctx->has_gyro || ctx->P.des_on)
    return fail(ctx, DTMX_ERR_UNSUPPORTED, "plane state: gyrotropic materials and design regions are not per plane");
  return DTMX_OK;
}

static int plane_copy(dtmx_ctx* ctx, int x0, int np, float* host, bool read) {
  if (!ctx) return DTMX_ERR_INVALID;
  if (int rc = plane_refusal(ctx)) return rc;
  const dtmx_config& c = ctx->cfg;
  if (!host || np < 0 || x0 < 0 || x0 + np > c.nx) return fail(ctx, DTMX_ERR_INVALID, "planes outside the grid");
  const int xl = ctx->P.ab.aux[0][0] ? ctx->P.ab.L[0][0] : 0, xh = ctx->P.ab.aux[0][0] ? ctx->P.ab.L[0][1] : 0;
  if (np > 0 && (x0 < xl || x0 + np > c.nx - xh))
    return fail(ctx, DTMX_ERR_UNSUPPORTED, "planes inside an x absorber slab");
  if (np == 0) return DTMX_OK;
  const cudaMemcpyKind kind = read ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice;
  const size_t nyz = (size_t)c.ny * c.nz;
  float* h = host;
  for (int comp = 0; comp < 6; comp++) {
    float* d = ctx->P.f[comp] + (size_t)x0 * ctx->P.g.sx;
    if (read) CK(cudaMemcpy2DAsync(h, (size_t)c.nz * 4, d, (size_t)ctx->nzp * 4, (size_t)c.nz * 4, (size_t)np * c.ny, kind, ctx->stream));
    else CK(cudaMemcpy2DAsync(d, (size_t)ctx->nzp * 4, h, (size_t)c.nz * 4, (size_t)c.nz * 4, (size_t)np * c.ny, kind, ctx->stream));
    h += (size_t)np * nyz;
  }
  for (int a = 1; a < 3; a++) {
    if (!ctx->P.ab.aux[a][0]) continue;
    const size_t th = (size_t)(ctx->P.ab.L[a][0] + ctx->P.ab.L[a][1]);
    const size_t pp = a == 1 ? th * c.nz : (size_t)c.ny * th;     // slab_index: x-major in both
    for (int q = 0; q < 4; q++) {
      float* d = ctx->P.ab.aux[a][q] + (size_t)x0 * pp;
      CK(cudaMemcpyAsync(read ? (void*)h : (void*)d, read ? (const void*)d : (const void*)h, (size_t)np * pp * 4, kind, ctx->stream));
      h += (size_t)np * pp;
    }
  }
  const Ade& A = ctx->P.ade;
  const int P = plane_poles(ctx);
  const int b0 = std::max(x0, A.lo[0]), b1 = std::min(x0 + np, A.lo[0] + A.n[0]);
  for (int comp = 0; comp < 3; comp++)
    for (int s = 0; s < 1 + 2 * P; s++) {
      float* arr = s == 0 ? A.Em[comp] : s <= P ? A.Jp[comp][s - 1] : A.Jm[comp][s - 1 - P];
      if (read) memset(h, 0, (size_t)np * nyz * 4);      // zero off the dispersive box
      if (arr && b0 < b1) {
        cudaMemcpy3DParms m = {};
        const cudaPitchedPtr dev = make_cudaPitchedPtr(arr, (size_t)A.n[2] * 4, A.n[2], A.n[1]);
        const cudaPitchedPtr hst = make_cudaPitchedPtr(h, (size_t)c.nz * 4, c.nz, c.ny);
        const cudaPos pd = make_cudaPos(0, 0, b0 - A.lo[0]), ph = make_cudaPos((size_t)A.lo[2] * 4, A.lo[1], b0 - x0);
        if (read) { m.srcPtr = dev; m.srcPos = pd; m.dstPtr = hst; m.dstPos = ph; }
        else { m.srcPtr = hst; m.srcPos = ph; m.dstPtr = dev; m.dstPos = pd; }
        m.extent = make_cudaExtent((size_t)A.n[2] * 4, A.n[1], b1 - b0);
        m.kind = kind;
        CK(cudaMemcpy3DAsync(&m, ctx->stream));
      }
      h += (size_t)np * nyz;
    }
  CK(cudaStreamSynchronize(ctx->stream));
  return DTMX_OK;
}

// Where array arr of ctx lives now: its device address, or while the context is
// parked, the same offset in its block's pinned host copy (nullptr if that block
// has no copy).  `bytes` from arr must lie inside the block.
static char* array_home(dtmx_ctx* ctx, const void* arr, size_t bytes) {
  if (!ctx->parked) return (char*)arr;
  const CUdeviceptr a = (CUdeviceptr)arr;
  for (const VmmBlock& b : ctx->vmm)
    if (a >= b.va && a + bytes <= b.va + b.size) return (b.host && !b.dead) ? (char*)b.host + (a - b.va) : nullptr;
  return nullptr;
}

// Plane state of planes [src_x0, src_x0 + n) of src into planes [dst_x0, ...)
// of dst, either of them parked (then its pinned host copy is read or written).
extern "C" int dtmx_copy_planes(dtmx_ctx* dst, int dst_x0, dtmx_ctx* src, int src_x0, int nplanes) {
  if (!dst || !src || dst == src) return fail(dst, DTMX_ERR_INVALID, "copy_planes needs two contexts");
  for (dtmx_ctx* x : {dst, src}) {
    if (x->cfg.geometry != DTMX_GEOM_BOX || x->cfg.absorber == DTMX_ABS_SPLIT_PML)
      return fail(dst, DTMX_ERR_UNSUPPORTED, "plane state: box geometry with a CPML or no absorber only");
    if (x->has_gyro || x->P.des_on)
      return fail(dst, DTMX_ERR_UNSUPPORTED, "plane state: gyrotropic materials and design regions are not per plane");
  }
  const dtmx_config &cd = dst->cfg, &cs = src->cfg;
  if (cd.ny != cs.ny || cd.nz != cs.nz || dst->nzp != src->nzp || plane_poles(dst) != plane_poles(src) ||
      plane_floats(dst) != plane_floats(src))
    return fail(dst, DTMX_ERR_INVALID, "copy_planes: contexts of different y/z configurations or material tables");
  for (int a = 1; a < 3; a++)
    if ((dst->P.ab.aux[a][0] != nullptr) != (src->P.ab.aux[a][0] != nullptr) || dst->P.ab.L[a][0] != src->P.ab.L[a][0] ||
        dst->P.ab.L[a][1] != src->P.ab.L[a][1])
      return fail(dst, DTMX_ERR_INVALID, "copy_planes: different y/z absorber slabs");
  const int np = nplanes;
  if (np < 0 || dst_x0 < 0 || src_x0 < 0 || dst_x0 + np > cd.nx || src_x0 + np > cs.nx)
    return fail(dst, DTMX_ERR_INVALID, "planes outside the grid");
  for (dtmx_ctx* x : {dst, src}) {
    const int x0 = x == dst ? dst_x0 : src_x0;
    const int xl = x->P.ab.aux[0][0] ? x->P.ab.L[0][0] : 0, xh = x->P.ab.aux[0][0] ? x->P.ab.L[0][1] : 0;
    if (np > 0 && (x0 < xl || x0 + np > x->cfg.nx - xh)) return fail(dst, DTMX_ERR_UNSUPPORTED, "planes inside an x absorber slab");
  }
  if (np == 0) return DTMX_OK;
  dtmx_ctx* ctx = dst;                          // errors of the copies are reported on dst
  CK(cudaStreamSynchronize(src->stream));
  cudaStream_t st = dst->stream;
  auto span = [&](dtmx_ctx* x, const float* arr, size_t off, size_t cnt) -> char* {
    // cnt floats from arr + off, inside the array's block
    return array_home(x, arr + off, cnt * 4);
  };
  // fields and y/z auxiliaries: the same per-plane layout in both contexts
  const size_t sx = (size_t)src->P.g.sx;
  for (int comp = 0; comp < 6; comp++) {
    char* d = span(dst, dst->P.f[comp], (size_t)dst_x0 * sx, (size_t)np * sx);
    char* h = span(src, src->P.f[comp], (size_t)src_x0 * sx, (size_t)np * sx);
    if (!d || !h) return fail(dst, DTMX_ERR_STATE, "copy_planes: a parked array has no host copy");
    CK(cudaMemcpyAsync(d, h, (size_t)np * sx * 4, cudaMemcpyDefault, st));
  }
  for (int a = 1; a < 3; a++) {
    if (!src->P.ab.aux[a][0]) continue;
    const size_t th = (size_t)(src->P.ab.L[a][0] + src->P.ab.L[a][1]);
    const size_t pp = a == 1 ? th * cs.nz : (size_t)cs.ny * th;
    for (int q = 0; q < 4; q++) {
      char* d = span(dst, dst->P.ab.aux[a][q], (size_t)dst_x0 * pp, (size_t)np * pp);
      char* h = span(src, src->P.ab.aux[a][q], (size_t)src_x0 * pp, (size_t)np * pp);
      if (!d || !h) return fail(dst, DTMX_ERR_STATE, "copy_planes: a parked array has no host copy");
      CK(cudaMemcpyAsync(d, h, (size_t)np * pp * 4, cudaMemcpyDefault, st));
    }
  }
  // ADE state over the intersection of the two boxes (a dispersive node of
  // the copied planes lies in both; the rest of either box holds zeros there)
  const Ade &As = src->P.ade, &Ad = dst->P.ade;
  const int P = plane_poles(src);
  const int p0 = std::max(std::max(0, As.lo[0] - src_x0), Ad.lo[0] - dst_x0);
  const int p1 = std::min(std::min(np, As.lo[0] + As.n[0] - src_x0), Ad.lo[0] + Ad.n[0] - dst_x0);
  const int y0 = std::max(As.lo[1], Ad.lo[1]), y1 = std::min(As.lo[1] + As.n[1], Ad.lo[1] + Ad.n[1]);
  const int z0 = std::max(As.lo[2], Ad.lo[2]), z1 = std::min(As.lo[2] + As.n[2], Ad.lo[2] + Ad.n[2]);
  for (int comp = 0; comp < 3; comp++)
    for (int q = 0; q < 1 + 2 * P; q++) {
      float* as = q == 0 ? As.Em[comp] : q <= P ? As.Jp[comp][q - 1] : As.Jm[comp][q - 1 - P];
      float* ad = q == 0 ? Ad.Em[comp] : q <= P ? Ad.Jp[comp][q - 1] : Ad.Jm[comp][q - 1 - P];
      if (!as || p0 >= p1 || y0 >= y1 || z0 >= z1) continue;       // nothing dispersive in the copied planes
      if (!ad) return fail(dst, DTMX_ERR_INVALID, "copy_planes: dispersive nodes the destination does not hold");
      const size_t ns = (size_t)As.n[0] * As.n[1] * As.n[2], nd = (size_t)Ad.n[0] * Ad.n[1] * Ad.n[2];
      char* hs = array_home(src, as, ns * 4);
      char* hd = array_home(dst, ad, nd * 4);
      if (!hs || !hd) return fail(dst, DTMX_ERR_STATE, "copy_planes: a parked array has no host copy");
      cudaMemcpy3DParms m = {};
      m.srcPtr = make_cudaPitchedPtr(hs, (size_t)As.n[2] * 4, As.n[2], As.n[1]);
      m.srcPos = make_cudaPos((size_t)(z0 - As.lo[2]) * 4, y0 - As.lo[1], src_x0 + p0 - As.lo[0]);
      m.dstPtr = make_cudaPitchedPtr(hd, (size_t)Ad.n[2] * 4, Ad.n[2], Ad.n[1]);
      m.dstPos = make_cudaPos((size_t)(z0 - Ad.lo[2]) * 4, y0 - Ad.lo[1], dst_x0 + p0 - Ad.lo[0]);
      m.extent = make_cudaExtent((size_t)(z1 - z0) * 4, y1 - y0, p1 - p0);
      m.kind = cudaMemcpyDefault;
      CK(cudaMemcpy3DAsync(&m, st));
    }
  CK(cudaStreamSynchronize(st));
  return DTMX_OK;
}

extern "C" int dtmx_plane_state_floats(dtmx_ctx* ctx, size_t* floats_per_plane) {
  if (!ctx || !floats_per_plane) return fail(ctx, DTMX_ERR_INVALID, "bad plane state request");
  if (int rc = plane_refusal(ctx)) return rc;
  *floats_per_plane = plane_floats(ctx);
  return DTMX_OK;
}

extern "C" int dtmx_read_planes(dtmx_ctx* ctx, int x0, int nplanes, float* host) {
  return plane_copy(ctx, x0, nplanes, host, true);
}

extern "C" int dtmx_write_planes(dtmx_ctx* ctx, int x0, int nplanes, const float* host) {
  return plane_copy(ctx, x0, nplanes, const_cast<float*>(host), false);
}

extern "C" int dtmx_set_tile_rows(dtmx_ctx* ctx, int rows) {
  if (!ctx || (rows != 0 && rows != 8 && rows != 16)) return fail(ctx, DTMX_ERR_INVALID, "tile rows must be 8 or 16");
  ctx->frows = rows ? rows : 16;
  drop_graphs(ctx);
  return DTMX_OK;
}

extern "C" int dtmx_get_engine(dtmx_ctx* ctx, int* engine, int* time_block, int* xchunk, int* tile_rows) {
  if (!ctx) return DTMX_ERR_INVALID;
  if (engine) *engine = ctx->engine;
  if (time_block) *time_block = ctx->tblock;
  if (xchunk) *xchunk = ctx->xchunk;
  if (tile_rows) *tile_rows = ctx->frows;
  return DTMX_OK;
}

extern "C" int dtmx_set_xchunk(dtmx_ctx* ctx, int planes) {
  if (!ctx || planes < 0) return fail(ctx, DTMX_ERR_INVALID, "bad x chunk");
  ctx->xchunk = planes;
  drop_graphs(ctx);
  return DTMX_OK;
}

extern "C" int dtmx_set_wait_limit(dtmx_ctx* ctx, int64_t polls) {
  if (!ctx) return DTMX_ERR_INVALID;
  ctx->P.wait_limit = polls > 0 ? (long long)polls : kWaitPolls;
  return DTMX_OK;
}

extern "C" int dtmx_get_stream(dtmx_ctx* ctx, void** stream) {
  if (!ctx || !stream) return DTMX_ERR_INVALID;
  *stream = (void*)ctx->stream;
  return DTMX_OK;
}

extern "C" int dtmx_set_profiling(dtmx_ctx* ctx, int enable) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx) return DTMX_ERR_INVALID;
  if (enable && !ctx->ev[0])
    for (int q = 0; q < 4; q++) CK(cudaEventCreate(&ctx->ev[q]));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->profiling = enable != 0;
  ctx->prof_ms_h = ctx->prof_ms_e = 0;
  ctx->prof_count = 0;
  ctx->prof_pending = false;
  return DTMX_OK;
}

extern "C" int dtmx_read_profile(dtmx_ctx* ctx, double* ms_h, double* ms_e, int64_t* count) {
  if (ctx && ctx->parked) return fail(ctx, DTMX_ERR_STATE, "the context is parked (dtmx_unpark first)");
  if (!ctx) return DTMX_ERR_INVALID;
  CK(cudaStreamSynchronize(ctx->stream));
  if (ms_h) *ms_h = ctx->prof_ms_h;
  if (ms_e) *ms_e = ctx->prof_ms_e;
  if (count) *count = ctx->prof_count;
  return DTMX_OK;
}

extern "C" int dtmx_abi_sizes(int64_t out[6]) {
  if (!out) return DTMX_ERR_INVALID;
  out[0] = sizeof(dtmx_config); out[1] = sizeof(dtmx_material);
  out[2] = sizeof(dtmx_point_source); out[3] = sizeof(dtmx_tfsf);
  out[4] = sizeof(dtmx_tfsfsrc); out[5] = sizeof(dtmx_ref_globals);
  return DTMX_OK;
}
