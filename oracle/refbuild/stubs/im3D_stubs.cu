// Definitions that the reference's visualiser (im3D.cu, GLUT + cuFFT) would
// provide to its host code, for building oracle/_ref without a graphics
// stack.  The --test path of _main (DTmxw.cu:797-808) calls none of them; the
// linker still needs the symbols that DTmxw.cu names.
#include "params.h"

image2D im2D;
bool recalc_at_once = true;
float calcTime = 0, calcPerf = 0;
int TimeStep = 0;
void add_sensor(int, int, int) {}
char* im3D_pars::reset_title() {
  static char title[] = "im3D";
  return title;
}
void im3D_pars::print_help() {}
bool im3D_pars::key_func(unsigned char, int, int) { return false; }
void im3D_pars::recalc_func() {}
void im3D_pars::mouse_func(int, int, int, int) {}
void im3D_pars::motion_func(int, int) {}
void im3D_pars::init3D(Arr3D_pars&) {}
void im3D_pars::initCuda(Arr3D_pars&) {}
