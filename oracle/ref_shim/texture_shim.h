// Stand-in for the texture-reference API that CUDA 12 removed, so that the
// reference's applications/fct_wfbp/include/cuda_kernels.cuh compiles
// unmodified from its own source tree. Its one texture reference (line 9)
// becomes a __device__ struct holding a texture object, and tex2D on it
// forwards to tex2D on that object (same clamp / linear / unnormalised
// sampling that ReconstructionMachine.cu:176-180 configures). Include this
// after every CUDA header and immediately before cuda_kernels.cuh.
// TEST INFRASTRUCTURE ONLY (oracle side).
#pragma once
#include <cuda_runtime.h>

template <class T, int Dim, enum cudaTextureReadMode Mode>
struct shim_texture_ref {
  cudaTextureObject_t obj;
};

template <class T, int Dim, enum cudaTextureReadMode Mode>
__device__ __forceinline__ T tex2D(const shim_texture_ref<T, Dim, Mode>& t, float x, float y) {
  return tex2D<T>(t.obj, x, y);
}

#define texture __device__ shim_texture_ref
