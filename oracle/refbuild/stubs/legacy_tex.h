// Stand-ins for CUDA's texture references, force-included (-include) into the
// reference's translation units when building oracle/_ref.
//
// CUDA 12 removed texture references (texture<T,dim,mode>, tex2D/tex3D on a
// reference, cudaBindTextureToArray, cudaUnbindTexture).  The reference
// declares some (DTmxw.cu:55-60, texmodel.cu:14-18, defs.h:161,168) for its
// visualiser and its seismic leftover model; its Maxwell kernels take the
// materials from get_mat_indev instead (COFFS_IN_DEVICE, py_consts.h:26,
// defs.h:184-190).  These stand-ins keep those declarations compiling; a
// fetch through one returns zero and a bind does nothing.
#pragma once
#include <cuda_runtime.h>

template <class T, int dim = 1, int mode = 0>
struct texture {
  int normalized;
  int filterMode;
  int addressMode[3];
};
// A fetch names a host-side object, which device code may not reference: the
// fetches through a texture reference become the constant 0 (a call of the
// texture-object form, tex3D<T>(...), is not followed by '(' and is left alone).
#define tex3D(ref, ...) 0
#define tex2D(ref, ...) 0
template <class T, int d, int m>
inline cudaError_t cudaBindTextureToArray(const texture<T, d, m>&, cudaArray_const_t) { return cudaSuccess; }
template <class T, int d, int m>
inline cudaError_t cudaBindTextureToArray(const texture<T, d, m>&, cudaArray_const_t, const cudaChannelFormatDesc&) {
  return cudaSuccess;
}
template <class T, int d, int m>
inline cudaError_t cudaUnbindTexture(const texture<T, d, m>&) { return cudaSuccess; }
