// Helical Q-weighted backprojection (sm_100a).
//
// Algorithm of backproject_kernel (cuda_kernels.cuh:198-287): for every voxel
// inside the acquisition FOV and every view angle theta~ of a half turn, the
// views j = theta~ + k*P/2 of all half turns k are Q-weighted, bilinear
// samples of the filtered rows are averaged with weights W(q), and
// (2 pi / P) * sum(W g) / sum(W) is added to the voxel (NaN when no half turn
// contributes, like the reference).
//
// Layout of the work: one thread owns one (x, y) column and ZS consecutive
// native slices (a z-slab). Everything that depends only on the column and
// the view -- p_hat, l_hat, asin term, the channel index and its weight -- is
// computed once per (column, view) and reused for the ZS slices; only the
// row coordinate, which is linear in z, is evaluated per voxel. A CTA covers a
// 16 x 8 column tile and skips, uniformly, the views whose table position
// fails the reference's z cull (|z_j - z| > z_rot) for every slice of its slab.
#include "wfbp_internal.h"

#include <type_traits>

namespace {

constexpr int BP_TX = 16, BP_TY = 8, BP_THREADS = BP_TX * BP_TY;

// W(q) of cuda_kernels.cuh:79-93 written as cos^2(x) = (1 + cos 2x)/2 with
// 2x = pi * clamp((|q| - 0.6)/0.4, 0, 1); 1 for |q| < 0.6, 0 for |q| >= 1.
__device__ __forceinline__ float q_weight(float qh) {
  float t = __saturatef(fmaf(fabsf(qh), 2.5f, -1.5f));
  return fmaf(0.5f, __cosf(3.14159265f * t), 0.5f);
}

__device__ __forceinline__ float ld_tap(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ld_tap(const __half* p) { return __half2float(__ldg(p)); }

// T = float: FP32 filtered rows. T = __half: FP16 rows, row r of view j
// stored as y / scale[j][r] (scales != nullptr).
template <int ZS, bool COUNT, typename T>
__global__ void __launch_bounds__(BP_THREADS)
k_bp(const T* __restrict__ D, const float* __restrict__ scales, float* __restrict__ vol,
     const float2* __restrict__ view_sc, const float* __restrict__ view_z, const float* __restrict__ zslices,
     BPParams p, unsigned long long* __restrict__ count) {
  constexpr bool SCALED = !std::is_same<T, float>::value;
  const int ix = blockIdx.x * BP_TX + (threadIdx.x % BP_TX);
  const int iy = blockIdx.y * BP_TY + (threadIdx.x / BP_TX);
  const int s0 = blockIdx.z * ZS;
  const bool in_grid = ix < p.nx && iy < p.ny;
  // voxel centre (cuda_kernels.cuh:215-216)
  const float x = ((float)ix - 0.5f * ((float)p.nx - 1.0f)) * p.fov / (float)p.nx + p.x0;
  const float y = ((float)iy - 0.5f * ((float)p.ny - 1.0f)) * p.fov / (float)p.ny + p.y0;

  float z[ZS];
  float zmin = 3.0e38f, zmax = -3.0e38f;
  unsigned zvalid = 0;
#pragma unroll
  for (int i = 0; i < ZS; i++) {
    int s = s0 + i;
    z[i] = s < p.nz ? zslices[s] : 0.0f;
    if (s < p.nz) {
      zvalid |= 1u << i;
      zmin = fminf(zmin, z[i]);
      zmax = fmaxf(zmax, z[i]);
    }
  }
  const bool active = in_grid && !(x * x + y * y > p.fov_half2);  // cuda_kernels.cuh:220

  float vacc[ZS];
#pragma unroll
  for (int i = 0; i < ZS; i++) vacc[i] = 0.0f;
  unsigned long long cnt = 0;

  if (active) {
    const size_t view_elems = (size_t)p.nr * p.nch;
    for (int t = 0; t < p.P2; t++) {
      float ag[ZS], aw[ZS];
#pragma unroll
      for (int i = 0; i < ZS; i++) { ag[i] = 0.0f; aw[i] = 0.0f; }
      for (int k = 0; k < p.K; k++) {
        const int j = t + k * p.P2;
        const float zt = __ldg(view_z + j);
        if (zt < zmin - p.z_rot || zt > zmax + p.z_rot) continue;  // fails the z cull for the whole slab
        const float2 sc = __ldg(view_sc + j);
        const float p_hat = x * sc.x - y * sc.y;
        const float l_hat = sqrtf(p.R2 - p_hat * p_hat) - x * sc.y - y * sc.x;
        const float A = p.zr2pi * asinf(p.rR * p_hat);
        const float inv = 1.0f / (l_hat * p.tanc);
        const float p_idx = p.kp - (p_hat * p.ps + p.c0);   // p-flip, cuda_kernels.cuh:247,251
        const float pf = floorf(p_idx);
        if (!(pf >= 0.0f && ceilf(p_idx) <= p.ncm2)) continue;  // cuda_kernels.cuh:259-263
        const float wp = p_idx - pf;
        const T* Dv = D + (size_t)j * view_elems + (int)pf;
        const float* Sv = SCALED ? scales + (size_t)j * p.nr : nullptr;
#pragma unroll
        for (int i = 0; i < ZS; i++) {
          const float dz = z[i] - zt;
          const float qh = (dz + A) * inv;
          const float q_idx = (qh + 1.0f) * p.hn;
          const bool ok = ((zvalid >> i) & 1u) && fabsf(dz) <= p.z_rot && q_idx >= 0.0f && q_idx <= p.nrm2;
          const float qf = floorf(q_idx);
          const float wq = q_idx - qf;
          int r = (int)qf;
          r = min(max(r, 0), p.nr - 2);
          const T* d0 = Dv + r * p.nch;
          const float d00 = ld_tap(d0), d01 = ld_tap(d0 + 1), d10 = ld_tap(d0 + p.nch), d11 = ld_tap(d0 + p.nch + 1);
          float top = fmaf(wp, d01 - d00, d00);
          float bot = fmaf(wp, d11 - d10, d10);
          if (SCALED) {
            top *= __ldg(Sv + r);
            bot *= __ldg(Sv + r + 1);
          }
          const float g = fmaf(wq, bot - top, top);
          const float W = ok ? q_weight(qh) : 0.0f;
          ag[i] = fmaf(W, g, ag[i]);
          aw[i] += W;
          if (COUNT) cnt += ok ? 1 : 0;
        }
      }
#pragma unroll
      for (int i = 0; i < ZS; i++) vacc[i] += p.dtheta * (1.0f / aw[i]) * ag[i];  // cuda_kernels.cuh:283
    }
  }
  if (in_grid) {
    const size_t plane = (size_t)p.nx * p.ny;
#pragma unroll
    for (int i = 0; i < ZS; i++)
      if ((zvalid >> i) & 1u) vol[(size_t)(s0 + i) * plane + (size_t)iy * p.nx + ix] = vacc[i];
  }
  if (COUNT) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(count, cnt);
  }
}

}  // namespace

namespace {
template <typename T>
cudaError_t launch_bp(const T* D, const float* scales, float* vol, const float2* sc, const float* vz,
                      const float* zs, const BPParams& p, unsigned long long* count, cudaStream_t s) {
  constexpr int ZS = 8;
  dim3 grid((unsigned)((p.nx + BP_TX - 1) / BP_TX), (unsigned)((p.ny + BP_TY - 1) / BP_TY),
            (unsigned)((p.nz + ZS - 1) / ZS));
  if (count)
    k_bp<ZS, true, T><<<grid, BP_THREADS, 0, s>>>(D, scales, vol, sc, vz, zs, p, count);
  else
    k_bp<ZS, false, T><<<grid, BP_THREADS, 0, s>>>(D, scales, vol, sc, vz, zs, p, count);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_backproject_f32(const float* D, float* vol, const float2* sc, const float* vz, const float* zs,
                                   const BPParams& p, unsigned long long* count, cudaStream_t s) {
  return launch_bp<float>(D, nullptr, vol, sc, vz, zs, p, count, s);
}

cudaError_t launch_backproject_f16(const __half* D, const float* scales, float* vol, const float2* sc,
                                   const float* vz, const float* zs, const BPParams& p, unsigned long long* count,
                                   cudaStream_t s) {
  return launch_bp<__half>(D, scales, vol, sc, vz, zs, p, count, s);
}
