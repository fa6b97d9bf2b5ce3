// Runs the reference's own WFBP kernels (applications/fct_wfbp/include/
// cuda_kernels.cuh, compiled unmodified from the reference tree) with the
// stage logic of applications/fct_wfbp/src/ReconstructionMachine.cu
// restated here: RebinAndFilter (RM:141-306), Backproject (RM:308-385) and
// ApplyFinalSliceThicknessing (RM:387-434), with the reference's launch
// shapes, cuFFT plans and per-row loop. Differences from RM.cu: inputs come
// from the caller instead of a DICOM reader, the texture reference is a
// texture object (texture_shim.h), the rebinned sheet has N_fft floats of
// slack so the rebin grid's writes past the last view stay in the allocation,
// and errors return a status instead of exit().
// TEST INFRASTRUCTURE ONLY: produces reference outputs to pin the oracle.
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdio.h>
#include <string.h>
#include <vector>

#include "recon_structs.h"
#include "texture_shim.h"
#include "cuda_kernels.cuh"
#undef texture

#define SHIM_TRY(x)                                                            \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess) {                                                   \
      fprintf(stderr, "ref shim: %s: %s\n", #x, cudaGetErrorString(e_));       \
      return 1;                                                                \
    }                                                                          \
  } while (0)
#define SHIM_FFT(x)                                                            \
  do {                                                                         \
    cufftResult r_ = (x);                                                      \
    if (r_ != CUFFT_SUCCESS) {                                                 \
      fprintf(stderr, "ref shim: %s: cufft %d\n", #x, (int)r_);                \
      return 2;                                                                \
    }                                                                          \
  } while (0)

extern "C" __attribute__((visibility("default"))) int ref_shim_run(
    const CTGeometry* cg_in, const ReconConfig* rp_in, const GPUPrecompute* gp_in, const float* raw,
    const float* taps_fft, const float* tube, const float* table, const float* z_native, int nz,
    const float* z_req, int nzr, float* filtered_out, float* native_out, float* volume_out) {
  CTGeometry cg = *cg_in;
  ReconConfig rp = *rp_in;
  GPUPrecompute gp = *gp_in;
  const size_t V = cg.total_number_of_projections, nr = cg.num_detector_rows, nch = cg.num_detector_cols;
  const size_t N = cg.num_detector_cols_padded_fft;
  if (nch > 1024 || rp.nx % 32 || rp.ny % 32) return 3;

  // RM:147-162 reshape into flipped row sheets
  std::vector<float> sheets(V * nr * nch);
  for (size_t i = 0; i < V; i++)
    for (size_t j = 0; j < nr; j++)
      for (size_t k = 0; k < nch; k++)
        sheets[(nch - 1 - k) + i * nch + (nr - 1 - j) * nch * V] = raw[k + j * nch + i * nch * nr];

  // RM:171-180 texture over a nch x V array, clamp / linear / unnormalised
  cudaChannelFormatDesc desc = cudaCreateChannelDesc<float>();
  cudaArray_t arr;
  SHIM_TRY(cudaMallocArray(&arr, &desc, nch, V));
  cudaResourceDesc res;
  memset(&res, 0, sizeof(res));
  res.resType = cudaResourceTypeArray;
  res.res.array.array = arr;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  cudaTextureObject_t tex;
  SHIM_TRY(cudaCreateTextureObject(&tex, &res, &td, NULL));
  shim_texture_ref<float, cudaTextureType2D, cudaReadModeElementType> tref;
  tref.obj = tex;
  SHIM_TRY(cudaMemcpyToSymbol(tex_row_sheet, &tref, sizeof(tref)));

  // RM:183-191
  float *d_rebin, *d_filtered;
  SHIM_TRY(cudaMalloc(&d_rebin, (N * V + N) * sizeof(float)));
  SHIM_TRY(cudaMemset(d_rebin, 0, (N * V + N) * sizeof(float)));
  SHIM_TRY(cudaMalloc(&d_filtered, nch * nr * V * sizeof(float)));
  // RM:194-201
  SHIM_TRY(cudaMemcpyToSymbol(d_cg, &cg, sizeof(CTGeometry)));
  SHIM_TRY(cudaMemcpyToSymbol(d_rp, &rp, sizeof(ReconConfig)));
  SHIM_TRY(cudaMemcpyToSymbol(d_gpu_precompute, &gp, sizeof(GPUPrecompute)));

  // generate_filter's device part (RM:515-543): R2C of the fftshifted taps
  float* d_taps;
  cufftComplex* d_filter;
  SHIM_TRY(cudaMalloc(&d_taps, N * sizeof(float)));
  SHIM_TRY(cudaMemcpy(d_taps, taps_fft, N * sizeof(float), cudaMemcpyHostToDevice));
  SHIM_TRY(cudaMalloc(&d_filter, (N / 2 + 1) * sizeof(cufftComplex)));
  cufftHandle fplan;
  SHIM_FFT(cufftPlan1d(&fplan, (int)N, CUFFT_R2C, 1));
  SHIM_FFT(cufftExecR2C(fplan, d_taps, d_filter));
  cufftDestroy(fplan);

  // RM:206-231
  cufftHandle pf, pr;
  int NX = (int)N, BATCH = (int)V;
  SHIM_FFT(cufftPlanMany(&pf, 1, &NX, NULL, 1, 0, NULL, 1, 0, CUFFT_R2C, BATCH));
  SHIM_FFT(cufftPlanMany(&pr, 1, &NX, NULL, 1, 0, NULL, 1, 0, CUFFT_C2R, BATCH));
  int fft_out = NX / 2 + 1;
  cufftComplex* d_four;
  SHIM_TRY(cudaMalloc(&d_four, (size_t)fft_out * V * sizeof(cufftComplex)));

  // RM:241-292
  for (size_t i = 0; i < nr; i++) {
    SHIM_TRY(cudaMemcpy2DToArray(arr, 0, 0, &sheets[i * nch * V], nch * sizeof(float), nch * sizeof(float), V,
                                 cudaMemcpyHostToDevice));
    dim3 rebin_threads(8, 8);
    dim3 rebin_blocks((unsigned)(N / rebin_threads.x), (unsigned)(V / rebin_threads.y));
    rebin_kernel<<<rebin_blocks, rebin_threads>>>(d_rebin);
    SHIM_TRY(cudaPeekAtLastError());
    SHIM_FFT(cufftExecR2C(pf, (cufftReal*)d_rebin, d_four));
    SHIM_TRY(cudaDeviceSynchronize());
    int channel_threads = fft_out;
    if (channel_threads > 1024) channel_threads = 512;
    dim3 filter_threads(channel_threads, 1);
    dim3 filter_blocks((unsigned)((fft_out + channel_threads - 1) / channel_threads), (unsigned)(V / filter_threads.y));
    multiply_filter<<<filter_blocks, filter_threads>>>(d_four, d_filter);
    SHIM_TRY(cudaPeekAtLastError());
    SHIM_TRY(cudaDeviceSynchronize());
    SHIM_FFT(cufftExecC2R(pr, d_four, (cufftReal*)d_rebin));
    SHIM_TRY(cudaDeviceSynchronize());
    dim3 reshape_threads((unsigned)nch, 1);
    dim3 reshape_blocks(1, (unsigned)(V / filter_threads.y));
    reshape_rebin_into_final_array<<<reshape_blocks, reshape_threads>>>(d_filtered, d_rebin, (int)i);
    SHIM_TRY(cudaPeekAtLastError());
  }
  SHIM_TRY(cudaDeviceSynchronize());
  cufftDestroy(pf);
  cufftDestroy(pr);
  if (filtered_out) SHIM_TRY(cudaMemcpy(filtered_out, d_filtered, nch * nr * V * sizeof(float), cudaMemcpyDeviceToHost));

  // RM:308-361
  float *d_tube, *d_table, *d_zn, *d_vol;
  SHIM_TRY(cudaMalloc(&d_tube, V * sizeof(float)));
  SHIM_TRY(cudaMemcpy(d_tube, tube, V * sizeof(float), cudaMemcpyHostToDevice));
  SHIM_TRY(cudaMalloc(&d_table, V * sizeof(float)));
  SHIM_TRY(cudaMemcpy(d_table, table, V * sizeof(float), cudaMemcpyHostToDevice));
  SHIM_TRY(cudaMalloc(&d_zn, nz * sizeof(float)));
  SHIM_TRY(cudaMemcpy(d_zn, z_native, nz * sizeof(float), cudaMemcpyHostToDevice));
  SHIM_TRY(cudaMalloc(&d_vol, rp.nx * rp.ny * nz * sizeof(float)));
  SHIM_TRY(cudaMemset(d_vol, 0, rp.nx * rp.ny * nz * sizeof(float)));
  dim3 bp_threads(32, 32, 1);
  dim3 bp_blocks((unsigned)(rp.nx / bp_threads.x), (unsigned)(rp.ny / bp_threads.y), (unsigned)(nz / bp_threads.z));
  size_t smem = rp.nx * sizeof(float) + rp.ny * sizeof(float);
  backproject_kernel<<<bp_blocks, bp_threads, smem>>>(d_filtered, d_vol, d_tube, d_table, d_zn);
  SHIM_TRY(cudaDeviceSynchronize());
  SHIM_TRY(cudaPeekAtLastError());
  if (native_out) SHIM_TRY(cudaMemcpy(native_out, d_vol, rp.nx * rp.ny * nz * sizeof(float), cudaMemcpyDeviceToHost));

  // RM:387-426
  float *d_final, *d_zr;
  SHIM_TRY(cudaMalloc(&d_final, rp.nx * rp.ny * nzr * sizeof(float)));
  SHIM_TRY(cudaMalloc(&d_zr, nzr * sizeof(float)));
  SHIM_TRY(cudaMemcpy(d_zr, z_req, nzr * sizeof(float), cudaMemcpyHostToDevice));
  dim3 th_threads(32, 32, 1);
  dim3 th_blocks((unsigned)(rp.nx / th_threads.x), (unsigned)(rp.ny / th_threads.y), (unsigned)(nzr / th_threads.z));
  thicken_slices<<<th_blocks, th_threads>>>(d_vol, d_final, d_zn, d_zr);
  SHIM_TRY(cudaPeekAtLastError());
  SHIM_TRY(cudaDeviceSynchronize());
  if (volume_out) SHIM_TRY(cudaMemcpy(volume_out, d_final, rp.nx * rp.ny * nzr * sizeof(float), cudaMemcpyDeviceToHost));

  cudaFree(d_final); cudaFree(d_zr); cudaFree(d_vol); cudaFree(d_zn); cudaFree(d_table); cudaFree(d_tube);
  cudaFree(d_four); cudaFree(d_filter); cudaFree(d_taps); cudaFree(d_filtered); cudaFree(d_rebin);
  cudaDestroyTextureObject(tex);
  cudaFreeArray(arr);
  return 0;
}

// Texture-unit probe: samples a w x h float texture (clamp, linear,
// unnormalised) at n coordinates, to compare the hardware's fractional
// weights with the oracle's 8-bit emulation.
__global__ void shim_tex_probe(cudaTextureObject_t t, const float2* xy, float* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = tex2D<float>(t, xy[i].x, xy[i].y);
}

extern "C" __attribute__((visibility("default"))) int ref_shim_tex_probe(const float* img, int w, int h,
                                                                          const float* xy, int n, float* out) {
  cudaChannelFormatDesc desc = cudaCreateChannelDesc<float>();
  cudaArray_t arr;
  SHIM_TRY(cudaMallocArray(&arr, &desc, w, h));
  SHIM_TRY(cudaMemcpy2DToArray(arr, 0, 0, img, w * sizeof(float), w * sizeof(float), h, cudaMemcpyHostToDevice));
  cudaResourceDesc res;
  memset(&res, 0, sizeof(res));
  res.resType = cudaResourceTypeArray;
  res.res.array.array = arr;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  cudaTextureObject_t tex;
  SHIM_TRY(cudaCreateTextureObject(&tex, &res, &td, NULL));
  float2* d_xy;
  float* d_out;
  SHIM_TRY(cudaMalloc(&d_xy, n * sizeof(float2)));
  SHIM_TRY(cudaMalloc(&d_out, n * sizeof(float)));
  SHIM_TRY(cudaMemcpy(d_xy, xy, n * sizeof(float2), cudaMemcpyHostToDevice));
  shim_tex_probe<<<(n + 255) / 256, 256>>>(tex, d_xy, d_out, n);
  SHIM_TRY(cudaDeviceSynchronize());
  SHIM_TRY(cudaMemcpy(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(d_xy); cudaFree(d_out);
  cudaDestroyTextureObject(tex);
  cudaFreeArray(arr);
  return 0;
}
