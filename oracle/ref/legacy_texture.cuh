// legacy_texture.cuh -- force-included when the reference's own CUDA sources
// are compiled into oracle/_ref/ (test infrastructure, never shipped).
//
// The reference binds its inputs through texture references
// (cuConstants.cuh:37-40, 49-50: `texture<T, 2, cudaReadModeElementType> tex_x;`),
// an API that CUDA 12 removed.  This header restores the small part of it the
// reference uses on top of texture objects, so that its .cu files compile
// unmodified where they lie:
//   * `texture` is a macro for a __device__ variable holding a
//     cudaTextureObject_t (a texture reference is a device-visible global);
//   * tex2D(ref, x, y) fetches through that object;
//   * cudaBindTexture2D / cudaBindTextureToArray create the object with the
//     legacy defaults (unnormalised coordinates, point sampling, clamp
//     addressing, element-type reads) and store it into the variable;
//   * cudaUnbindTexture destroys it.
// Every system header the reference includes is included first, so the macro
// reaches only the reference's own declarations.
#pragma once

#include <cuda_runtime.h>
#include <cuComplex.h>
#include <cuda_occupancy.h>
#include <cuda_profiler_api.h>
#include <device_launch_parameters.h>
#include <math_constants.h>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <complex>
#include <cmath>
#include <cstdio>
#include <ctime>
#include <iostream>
#include <fstream>
#include <string>
#include <omp.h>

template <class T, int Dim, enum cudaTextureReadMode Mode>
struct legacy_texture_ref {
  cudaTextureObject_t obj;
};

template <class T, int Dim, enum cudaTextureReadMode Mode>
__device__ __forceinline__ T tex2D(const legacy_texture_ref<T, Dim, Mode> &r, float x, float y) {
  return ::tex2D<T>(r.obj, x, y);
}

namespace legacy_texture_detail {
inline cudaTextureDesc legacy_desc() {
  cudaTextureDesc td = {};
  td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModePoint;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  return td;
}
}  // namespace legacy_texture_detail

template <class T, int Dim, enum cudaTextureReadMode Mode>
static cudaError_t cudaBindTexture2D(size_t *offset, const legacy_texture_ref<T, Dim, Mode> &sym,
                                     const void *ptr, const cudaChannelFormatDesc &desc,
                                     size_t width, size_t height, size_t pitch) {
  if (offset) *offset = 0;
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypePitch2D;
  rd.res.pitch2D.devPtr = const_cast<void *>(ptr);
  rd.res.pitch2D.desc = desc;
  rd.res.pitch2D.width = width;
  rd.res.pitch2D.height = height;
  rd.res.pitch2D.pitchInBytes = pitch;
  const cudaTextureDesc td = legacy_texture_detail::legacy_desc();
  legacy_texture_ref<T, Dim, Mode> h;
  cudaError_t e = cudaCreateTextureObject(&h.obj, &rd, &td, nullptr);
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(sym, &h, sizeof(h));
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
static cudaError_t cudaBindTextureToArray(const legacy_texture_ref<T, Dim, Mode> &sym,
                                          cudaArray_const_t array, const cudaChannelFormatDesc &) {
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = const_cast<cudaArray_t>(array);
  const cudaTextureDesc td = legacy_texture_detail::legacy_desc();
  legacy_texture_ref<T, Dim, Mode> h;
  cudaError_t e = cudaCreateTextureObject(&h.obj, &rd, &td, nullptr);
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(sym, &h, sizeof(h));
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
static cudaError_t cudaUnbindTexture(const legacy_texture_ref<T, Dim, Mode> &sym) {
  legacy_texture_ref<T, Dim, Mode> h;
  cudaError_t e = cudaMemcpyFromSymbol(&h, sym, sizeof(h));
  if (e != cudaSuccess) return e;
  return cudaDestroyTextureObject(h.obj);
}

#define texture __device__ legacy_texture_ref
