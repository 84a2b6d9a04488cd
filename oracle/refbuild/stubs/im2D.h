// Headless stand-in for the reference's im2D.h, used only to build oracle/_ref.
//
// The reference's im2D.h opens a GLUT window and writes PNG files
// (GL/glut.h, cuda_gl_interop.h, png.h); neither machine here has a graphics
// stack, and the --test path of _main (DTmxw.cu:797-808) draws nothing.  This
// header keeps the names that the reference's host code uses (exit_if_ERR,
// image2D, the glut* registration calls) with no window behind them.
#ifndef IM2D_H
#define IM2D_H
#include <cstdio>
#include <cuda_runtime.h>

extern int type_diag_flag;
inline void exit_if_ERR(cudaError_t rs) {
  if (rs == cudaSuccess) return;
  fprintf(stderr, "%s \n", cudaGetErrorString(rs));
  throw(-1);
}
struct image2D {
  int Nx, Ny;
  void get_device(int = 2, int = 1) {}
  void init_image(int, char**, int nx, int ny, const char*) { Nx = nx; Ny = ny; }
  void draw(const char*) {}
};
// event timer on the legacy stream (start, stop -> milliseconds)
struct cudaTimer {
  cudaEvent_t t0, t1;
  cudaTimer() { cudaEventCreate(&t0); cudaEventCreate(&t1); }
  ~cudaTimer() { cudaEventDestroy(t0); cudaEventDestroy(t1); }
  void start() { cudaEventRecord(t0, 0); cudaEventSynchronize(t0); }
  float stop() {
    float ms = 0;
    cudaEventRecord(t1, 0);
    cudaEventSynchronize(t1);
    cudaEventElapsedTime(&ms, t0, t1);
    return ms;
  }
  float restart() { const float ms = stop(); start(); return ms; }
};
template <class F> inline void glutIdleFunc(F) {}
template <class F> inline void glutKeyboardFunc(F) {}
template <class F> inline void glutMouseFunc(F) {}
template <class F> inline void glutMotionFunc(F) {}
template <class F> inline void glutDisplayFunc(F) {}
inline void glutPostRedisplay() {}
inline void glutMainLoop() {}
#endif  // IM2D_H
