// Driver of the reference's own CUDA build (oracle/_ref): what the
// reference's run.py does through its SWIG module, in C++ (no SWIG here).
//
// run.py:17-38 puts the TF/SF dipole at the middle of the x-y plane, 0.23
// above z = 0 (center = [GridNx/2*dx, GridNy/2*dy, 0.150+0.08], GridNx/2 an
// integer division in Python 2), a box of +-5 cells around it, sets the source
// with TFSFsrc::set(cL, cL, 0.5 cL), cL = 1/1.75, and the stop time
// boxDiag/cL + 20*2*pi/w + t0 + 10*dt, then calls _main(sys.argv).  Here
// Tsteps comes from --steps (run.py sets 1000000) and the sensor files go to
// --drop_dir; _main runs headless (--test).
//
// --box_shift f moves the TF/SF box by f cells along every axis.  run.py's
// box faces lie exactly on node planes (+-5 cells around a node), so whether
// a face node counts as inside depends on the rounding of the reference's
// inSF test (signal.hpp:153-160) and the FP32 and FP64 builds disagree there;
// a shift of a fraction of a cell takes that ambiguity away.
//
// Usage: ref_run --steps N --drop_dir DIR [--box_shift f]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "py_consts.h"

extern int Tsteps;
int _main(int argc, char** argv);

int main(int argc, char** argv) {
  int steps = 0;
  double shift = 0;
  std::string drop = ".";
  for (int a = 1; a + 1 < argc; a += 2) {
    if (!strcmp(argv[a], "--steps")) steps = atoi(argv[a + 1]);
    else if (!strcmp(argv[a], "--drop_dir")) drop = argv[a + 1];
    else if (!strcmp(argv[a], "--box_shift")) shift = atof(argv[a + 1]);
    else { fprintf(stderr, "usage: %s --steps N --drop_dir DIR\n", argv[0]); return 2; }
  }
  if (steps <= 0) { fprintf(stderr, "usage: %s --steps N --drop_dir DIR\n", argv[0]); return 2; }
  // the module's globals as run.py reads them (cvar.GridNx, cvar.ds, ...)
  const double dx = ds, dy = da, dz = dv, dtt = dt;
  const double center[3] = {(GridNx / 2) * dx, (GridNy / 2) * dy, 0.150 + 0.08 + 0 * (GridNz / 2) * dz};
  TFSFsrc& SS = shotpoint;
  SS.srcXs = center[0]; SS.srcXa = center[1]; SS.srcXv = center[2];
  SS.BoxMs = SS.srcXs - 5 * dx; SS.BoxPs = SS.srcXs + 5 * dx;
  SS.BoxMa = SS.srcXa - 5 * dy; SS.BoxPa = SS.srcXa + 5 * dy;
  SS.BoxMv = SS.srcXv - 5 * dz; SS.BoxPv = SS.srcXv + 5 * dz;
  if (shift != 0) {
    SS.BoxMs = SS.BoxMs + shift * dx; SS.BoxPs = SS.BoxPs + shift * dx;
    SS.BoxMa = SS.BoxMa + shift * dy; SS.BoxPa = SS.BoxPa + shift * dy;
    SS.BoxMv = SS.BoxMv + shift * dz; SS.BoxPv = SS.BoxPv + shift * dz;
  }
  const double a = (double)SS.BoxPs - SS.BoxMs, b = (double)SS.BoxPa - SS.BoxMa, c = (double)SS.BoxMv - SS.BoxPv;
  const double boxDiagLength = std::sqrt(a * a + b * b + c * c);
  const double cL = 1.0 / 1.75;
  SS.set(cL, cL, 0.5 * cL);
  SS.tStop = boxDiagLength / cL + 20 * 2 * M_PI / (double)SS.w + (double)SS.t0 + 10 * dtt;
  Tsteps = steps;
  std::string d = drop;
  char a0[] = "ref_run", a1[] = "--test", a2[] = "--drop_dir";
  char* av[] = {a0, a1, a2, &d[0], nullptr};
  return _main(4, av);
}
