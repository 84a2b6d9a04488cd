// dtmx_ref_driver.cpp -- the reference's headless driver (_main with --test)
// rebuilt on top of the C ABI: grid constants, the analytic layered Ag-film
// geometry, the material table, the TF/SF dipole from TFSFsrc, the default
// sensor line and the per-calcStep sensor files.
//
// Reference: _main (DTmxw.cu:731-834), GeoParamsHost::set checks
// (DTmxw.cu:278-487), init_index sensors (DTmxw.cu:502-553), init_material
// (DTmxw.cu:604-706), get_mat_indev (defs.h:128-148), TFSFsrc::set
// (signal.hpp:99-115), Sensor (sensor.h:6-84), calcStep's rate line
// (diamond.cu:477-485).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <chrono>
#include <sys/stat.h>

#include "dtmx.h"

namespace {

// Material indices of the reference enum that get_mat_indev can return.
enum { kOrg = 0, kAg = 1, kITO = 2, kGlass = 3, kNumMat = 4 };

// get_mat_indev (defs.h:128-148) with the reference's mixed precision: the
// coordinates are products computed in double and stored in float
// (`float x=ix*0.5*dx` with dx a float constant), the layer tests in float;
// (ix, iy, iz) are half-cell coordinates.
int ref_material(int ix, int iy, int iz, const dtmx_ref_globals* g) {
  const int NDT = 3;
  const float dx = (float)g->ds, dy = (float)g->da, dz = (float)g->dv;
  float x = (float)(ix * 0.5 * (double)dx), y = (float)(iy * 0.5 * (double)dy), z = (float)(iz * 0.5 * (double)dz);
  const float Xc = (float)(0.5 * g->Np * NDT * (double)dx), Yc = (float)(0.5 * g->Na * NDT * (double)dy);
  const int Npmlx = g->Npmlx > 0 ? g->Npmlx : 10, Npmly = g->Npmly > 0 ? g->Npmly : 10;
  if (x < (Npmlx * NDT + 100) * dx / 2 || x > g->Np * NDT * dx - (Npmlx * NDT + 100) * dx / 2 ||
      y < (Npmly * NDT + 100) * dy / 2 || y > g->Na * NDT * dy - (Npmly * NDT + 100) * dy / 2)
    return kOrg;
  const float period = 0.4f, rad = 0.1f, height = 0.1f;
  const float xr = x - Xc - std::round((x - Xc) / period) * period;
  const float yr = y - Yc - std::round((y - Yc) / period) * period;
  const float shift = 1e-5f;
  z -= 0.150f - shift;
  if (z < 0) return (z > -height && xr * xr + yr * yr < rad * rad) ? kOrg : kAg;
  z -= 0.180f + shift;
  if (z < 0) return kOrg;
  z -= 0.100f + shift;
  if (z < 0) return kITO;
  return kGlass;
}

// init_material (DTmxw.cu:604-635): the materials get_mat_indev can return
void ref_material_table(dtmx_material* mats) {
  memset(mats, 0, sizeof(dtmx_material) * kNumMat);
  const double eps[kNumMat] = {1.75 * 1.75, 1.0, 1.8 * 1.8, 1.5 * 1.5};
  for (int m = 0; m < kNumMat; m++) mats[m].eps[0] = mats[m].eps[1] = mats[m].eps[2] = eps[m];
  mats[kAg].npoles = 1;
  mats[kAg].pole_kind[0] = DTMX_POLE_DRUDE;
  mats[kAg].pole[0][0] = 1.0;                      // AgP.setDrude(1.0, 136.66/3.0, 2.69e13/2/3e14, 0)
  mats[kAg].pole[0][1] = 136.66 / 3.0;
  mats[kAg].pole[0][2] = 2.69e13 / 2 / 3e14;
  mats[kAg].pole[0][3] = 0.0;
  mats[kAg].eps_inf = 1.0;                         // DispCoffsHost[IndAg].set(1, Agvec, 1, 0)
  mats[kAg].sigma = 0.0;
}

// SeismoDrops::drop (drop.cu:83-107) with DROP_DATA: Ez of the first V domain
// of every rag, the node of cell (3x-1, 3y-1, z), z fastest within a rag.
int write_rag_drop(const std::string& dir, int it, const dtmx_ref_globals* g, const std::vector<float>& ez) {
  char fname[512];
  snprintf(fname, sizeof(fname), "%s/ragEz_%05d.arr", dir.c_str(), it);
  FILE* f = fopen(fname, "wb");
  if (!f) return -1;
  const int nx = 3 * g->Np, ny = 3 * g->Na, nz = g->Nv;
  const int head[9] = {12, 0, 0, 0, 3, (int)sizeof(float), g->Nv, g->Na, g->Np};
  bool ok = fwrite(head, sizeof(int), 9, f) == 9;
  std::vector<float> row(nz);
  for (int x = 0; x < g->Np && ok; x++)
    for (int y = 0; y < g->Na && ok; y++) {
      const int i = 3 * x - 1, j = 3 * y - 1;
      for (int k = 0; k < nz; k++)
        row[k] = (i >= 0 && i < nx && j >= 0 && j < ny) ? ez[((size_t)i * ny + j) * nz + k] : 0.f;
      ok = fwrite(row.data(), sizeof(float), nz, f) == (size_t)nz;
    }
  return (fclose(f) == 0 && ok) ? 0 : -1;
}

struct SensorFile {
  int comp, x, y, z, probe;
  FILE* f;
};

int comp_of(const char* name) {
  static const char* n[6] = {"Ex", "Ey", "Ez", "Hx", "Hy", "Hz"};
  for (int c = 0; c < 6; c++)
    if (!strcmp(name, n[c])) return c;
  return -1;
}

}  // namespace

// Material index arrays of the reference geometry: each E node takes the
// material at its own half-coordinates (TEXCOFFV*, defs.h:176-181).
extern "C" int dtmx_ref_materials(const dtmx_ref_globals* g, uint8_t* idx_x, uint8_t* idx_y, uint8_t* idx_z) {
  if (!g || !idx_x || !idx_y || !idx_z) return DTMX_ERR_INVALID;
  const int nx = 3 * g->Np, ny = 3 * g->Na, nz = g->Nv;
  uint8_t* idx[3] = {idx_x, idx_y, idx_z};
  const int off[3][3] = {{0, 1, 1}, {1, 0, 1}, {1, 1, 0}};
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++)
        for (int c = 0; c < 3; c++)
          idx[c][((size_t)i * ny + j) * nz + k] =
              (uint8_t)ref_material(2 * i + off[c][0], 2 * j + off[c][1], 2 * k + off[c][2], g);
  return DTMX_OK;
}

extern "C" int dtmx_ref_material_table(dtmx_material* out, int n) {
  if (!out || n < kNumMat) return DTMX_ERR_INVALID;
  ref_material_table(out);
  return kNumMat;
}

// TFSFsrc::set (signal.hpp:99-115).  The reference's fields are ftype
// (float): every assignment rounds to float and later lines read the rounded
// value (kEnv = Omega/w is a float division); the values are returned in the
// double fields of dtmx_tfsfsrc.
extern "C" void dtmx_tfsfsrc_set(dtmx_tfsfsrc* s, double c, double impedance, double lmb) {
  s->Imp = (float)impedance;
  s->V_max = (float)c;
  s->cSrc = (float)c;
  const float wl = (float)lmb;
  const float k = (float)(2 * M_PI / wl);
  const float w = (float)(c * k);
  const float om = (float)(0.05 * w);
  s->wavelength = wl;
  s->k = k;
  s->w = w;
  s->Omega = om;
  s->kEnv = om / w;
  s->theta = (float)(0 + M_PI);
  s->phi = (float)(M_PI / 2);
  s->t0 = (float)(25 * 0.02);
  s->tw = (float)(5 * 0.02);
  s->T = (float)(125 * 0.02);
}

extern "C" int dtmx_ref_main(const dtmx_ref_globals* g, const dtmx_tfsfsrc* sp, int argc, char** argv) {
  if (!g || !sp) return -1;
  bool test_only = false, drop_data = false;
  std::string drop_dir = ".";
  for (int a = 1; a < argc; a++) {
    const std::string s = argv[a];
    if (s == "--test") test_only = true;
    else if (s == "--drop_data") drop_data = true;
    else if (s == "--help") { printf("using: DTmxw._main([prog, '--test', '--drop_dir', dir])\n"); return 0; }
    else if (s == "--drop_dir" && a + 1 < argc) drop_dir = argv[++a];
    else if ((s == "--swap_dir" || s == "--sensor" || s == "--box" || s == "--mesh" || s == "--Dmesh" || s == "--zoom" ||
              s == "--step" || s == "--bkgr_col" || s == "--mesh_col" || s == "--box_col") && a + 1 < argc)
      ++a;   // window/visualisation options: no graphics stack, accepted and ignored
    else { printf("Illegal parameters' syntax notation\n"); return 0; }
  }
  if (!test_only) printf("No GL: running headless (as with --test)\n");
  const int NDT = 3;
  const int nx = NDT * g->Np, ny = NDT * g->Na, nz = g->Nv;
  // GeoParamsHost::set checks (DTmxw.cu:308-336)
  if (g->Ns <= 0 || g->Np % g->Ns != 0) { printf("Error: Np must be dividable by Ns\n"); return -1; }
  if (g->Ntime <= 0 || g->Ns - g->Ntime < 2) { printf("Error: Ns-Ntime<2*NTorres\n"); return -1; }
  if (g->dt * std::sqrt(1 / (g->ds * g->ds) + 1 / (g->da * g->da) + 1 / (g->dv * g->dv)) > 6. / 7.) {
    printf("Error: Courant condition is not satisfied\n");
    return -1;
  }
  mkdir(drop_dir.c_str(), 0700);
  printf("Grid size: %dx%d Rags /%dx%dx%d Yee_cells/, TorreH=%d\n", g->Np, g->Na, nx, ny, nz, g->Ntime);

  dtmx_config cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.nx = nx; cfg.ny = ny; cfg.nz = nz;
  cfg.dx = g->ds; cfg.dy = g->da; cfg.dz = g->dv; cfg.dt = g->dt;
  cfg.order = 4;                                   // genDT.py:8
  cfg.geometry = DTMX_GEOM_REFERENCE;
  cfg.absorber = DTMX_ABS_SPLIT_PML;
  const int Npmlx = g->Npmlx > 0 ? g->Npmlx : 10, Npmly = g->Npmly > 0 ? g->Npmly : 10;
  const int Npmlz = g->Npmlz > 0 ? g->Npmlz : 32;  // py_consts.h:67-69
  if (Npmlx % 2 || Npmly % 2 || Npmlz % 2) { printf("Error: Npmlx, Npmly and Npmlz must be even\n"); return -1; }
  cfg.pml[0][0] = cfg.pml[0][1] = Npmlx / 2 * NDT; // Npmlx/2 rags of NDT cells
  cfg.pml[1][0] = cfg.pml[1][1] = Npmly / 2 * NDT; // Npmly/2 rags
  cfg.pml[2][1] = Npmlz / 2;                       // Npmlz/2, top face only
  cfg.spml_vmax = sp->V_max;
  cfg.probe_every = g->Ntime;                      // one sample per calcStep
  cfg.probe_capacity = g->Tsteps / g->Ntime + 2;
  dtmx_ctx* ctx = nullptr;
  int rc = dtmx_create(&cfg, &ctx);
  if (rc != DTMX_OK) {
    printf("Error: dtmx_create: %s (%s)\n", dtmx_error_string(rc), ctx ? dtmx_last_error(ctx) : "");
    if (ctx) dtmx_destroy(ctx);
    return -1;
  }
  dtmx_material mats[kNumMat];
  ref_material_table(mats);
  const size_t ncell = (size_t)nx * ny * nz;
  std::vector<uint8_t> idx[3];
  for (int c = 0; c < 3; c++) idx[c].resize(ncell);
  dtmx_ref_materials(g, idx[0].data(), idx[1].data(), idx[2].data());
  rc = dtmx_set_materials(ctx, mats, kNumMat, idx[0].data(), idx[1].data(), idx[2].data());
  if (rc != DTMX_OK) { printf("Error: materials: %s\n", dtmx_last_error(ctx)); dtmx_destroy(ctx); return -1; }
  // TF/SF dipole from the shotpoint (copy2dev(shotpoint, src), DTmxw.cu:784)
  dtmx_tfsf t;
  memset(&t, 0, sizeof(t));
  t.kind = DTMX_TFSF_DIPOLE;
  t.box_lo[0] = sp->BoxMs; t.box_hi[0] = sp->BoxPs;
  t.box_lo[1] = sp->BoxMa; t.box_hi[1] = sp->BoxPa;
  t.box_lo[2] = sp->BoxMv; t.box_hi[2] = sp->BoxPv;
  t.c = sp->cSrc; t.w = sp->w; t.kenv = sp->kEnv;
  t.tstop = sp->tStop;
  t.ntime = g->Ntime;
  rc = dtmx_set_tfsf(ctx, &t);
  if (rc != DTMX_OK) { printf("Error: TF/SF source: %s\n", dtmx_last_error(ctx)); dtmx_destroy(ctx); return -1; }
  printf("TF/SF source: Box(s,v,a) |%g-%g|x|%g-%g|x|%g-%g|\n", sp->BoxMs, sp->BoxPs, sp->BoxMv, sp->BoxPv, sp->BoxMa,
         sp->BoxPa);
  // default sensors (init_index, DTmxw.cu:524-542): a line along +x from the dipole
  const double Xdip = (sp->BoxMs + sp->BoxPs) * 0.5, Ydip = (sp->BoxMa + sp->BoxPa) * 0.5;
  const int X0 = (int)std::lround(Xdip / g->ds), Y0 = (int)std::lround(Ydip / g->da), Z0 = (int)std::lround(0.150 / g->dv);
  std::vector<SensorFile> sensors;
  static const char* names[6] = {"Ex", "Ey", "Ez", "Hx", "Hy", "Hz"};
  for (double xsen = 0.0; xsen < g->Np * NDT * g->ds / 2; xsen += 1.0) {
    const int xcrd = X0 + (int)std::lround(xsen / g->ds);
    if (xcrd < 0 || xcrd >= nx || Y0 < 0 || Y0 >= ny || Z0 < 0 || Z0 >= nz) continue;
    for (int c = 0; c < 6; c++) {
      SensorFile s{c, xcrd, Y0, Z0, -1, nullptr};
      if (dtmx_add_probe(ctx, c, xcrd, Y0, Z0, DTMX_PROBE_REFERENCE, &s.probe) != DTMX_OK) continue;
      char fname[512];
      snprintf(fname, sizeof(fname), "%s/%s-x%05dy%05dz%05d.dat", drop_dir.c_str(), names[c], xcrd, Y0, Z0);
      s.f = fopen(fname, "w");
      if (!s.f) { printf("Error openning file %s\n", fname); dtmx_destroy(ctx); return -1; }
      printf("Set sensor %s at %d %d %d\n", names[c], xcrd, Y0, Z0);
      sensors.push_back(s);
    }
  }
  (void)comp_of;
  const int nbig = g->Tsteps / g->Ntime;
  std::vector<float> trace;
  int status = 0;
  for (int s = 0; s < nbig && !status; s++) {
    const auto t0 = std::chrono::steady_clock::now();
    rc = dtmx_step(ctx, g->Ntime);
    if (rc == DTMX_OK) rc = dtmx_sync(ctx);
    if (rc != DTMX_OK) { printf("Error: step: %s\n", dtmx_last_error(ctx)); status = -1; break; }
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const double cells = (double)ncell * g->Ntime;
    printf("Step %d: Time %9.09f ms ||rate %9.09f GYee_cells/sec |total grid %dx%dx%d=%zu cells | isTFSF=%d\n", s, ms,
           1e-9 * cells / (ms * 1e-3), nx, ny, nz, ncell, (s + 1) * g->Ntime * g->dt < sp->tStop);
    if (drop_data) {
      std::vector<float> ez(ncell);
      if (dtmx_get_field(ctx, DTMX_EZ, ez.data()) != DTMX_OK || write_rag_drop(drop_dir, s, g, ez) != 0) {
        printf("Error: field drop %d: %s\n", s, dtmx_last_error(ctx));
        status = -1;
        break;
      }
    }
    if (!sensors.empty()) {
      const int cap = g->Tsteps / g->Ntime + 2;
      int ns = 0;
      trace.assign((size_t)sensors.size() * cap, 0.f);
      dtmx_read_probes(ctx, trace.data(), cap, &ns);
      for (auto& sf : sensors) {
        fprintf(sf.f, "%g\n", (double)trace[(size_t)sf.probe * cap + ns - 1]);
        fflush(sf.f);
      }
    }
  }
  for (auto& sf : sensors) fclose(sf.f);
  dtmx_destroy(ctx);
  return status;
}
