// Internal declarations of the B200 WFBP library (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/freect_wfbp.h"

// Geometry constants every backprojection launch needs, derived once per
// context from GPUPrecompute (recon_structs.h:52-83) and ReconConfig.
struct BPParams {
  int nx, ny, nz;            // native volume
  int nch, nr, V;            // filtered projections [V][nr][nch]
  int P2, K;                 // views per half turn, half turns
  float fov, x0, y0;         // recon_fov, x_origin, y_origin
  float fov_half2;           // half_acquisition_fov_squared
  float z_rot;
  float R2;                  // distance_source_to_isocenter_squared
  float rR;                  // recip_distance_source_to_isocenter
  float zr2pi;               // z_rot_over_2_pi
  float tanc;                // tanf_theta_cone
  float ps;                  // pixel_scale
  float c0;                  // detector_central_col
  float kp;                  // (float)(nch + 1.75): the p-flip of cuda_kernels.cuh:251
  float hn;                  // 0.5 * (nr - 1)
  float nrm2;                // nr - 2 (last valid floor row)
  float ncm2;                // nch - 2
  float dtheta;              // two_pi_over_projections_per_rotation
};

struct RebinParams {
  int V, nr, nch;            // views, rows, channels (no FFS)
  float dth;                 // 2*3.14159265f / P  (cuda_kernels.cuh:15)
  int q8;                    // 8-bit fractional weights
};

struct wfbp_ctx {
  CTGeometry cg;
  ReconConfig rp;
  GPUPrecompute gp;
  wfbp_ext ext;
  int device = 0;

  int V = 0, nr = 0, nch = 0, P = 0, P2 = 0, K = 0, nx = 0, ny = 0, nz = 0, nzr = 0;
  int n_readings = 0, raw_rows = 0, raw_ch = 0;
  std::vector<float> z_native, z_req;
  std::vector<float> taps;          // symmetric half taps h[0..nch-1]
  std::vector<int> thick_off;       // CSR over requested slices
  std::vector<int> thick_idx;
  std::vector<float> thick_w;

  // device tables
  float* d_taps = nullptr;          // [nch]
  float* d_chan_beta = nullptr;     // [nch]
  float* d_chan_bidx = nullptr;     // [nch], NaN where the rebin writes 0
  float2* d_view_sc = nullptr;      // [V] (sinf, cosf) of the tube angle
  float* d_view_z = nullptr;        // [V] table position
  float* d_z_native = nullptr;      // [nz]
  int* d_thick_off = nullptr;
  int* d_thick_idx = nullptr;
  float* d_thick_w = nullptr;
  float* d_thick_ws = nullptr;      // [nzr] sum of weights

  // mixed precision: Toeplitz operand planes for the tensor-core filter
  int tc_kp = 0, tc_np = 0, tc_bn = 0;
  float taps_l1 = 0.0f;             // sum over |d| < nch of |h[d]|
  void* d_bplanes = nullptr;        // bf16 [2][tc_np][tc_kp]
  int* d_err = nullptr;             // device-side error word (bounded waits)

  // context-owned scratch for wfbp_run / wfbp_run_host
  void* s_rebinned = nullptr;
  void* s_filtered = nullptr;
  float* s_scales = nullptr;
  float* s_vol_native = nullptr;
  float* s_raw = nullptr;
  float* s_vol = nullptr;

  bool views_set = false;
  std::string err;
};

// kernels (launchers return cudaError_t of the launch)
cudaError_t launch_view_tables(const float* d_tube, const float* d_table, float2* d_sc, float* d_z, int V,
                               cudaStream_t s);
cudaError_t launch_rebin_tables(float* d_beta, float* d_bidx, int nch, float c0, float dcol, float sdd,
                                cudaStream_t s);
cudaError_t launch_rebin_f32(const float* raw, float* out, const float* d_beta, const float* d_bidx,
                             const RebinParams& p, cudaStream_t s);
cudaError_t launch_filter_f32(const float* x, float* y, const float* d_taps, long rows, int nch, cudaStream_t s);
cudaError_t launch_backproject_f32(const float* D, float* vol, const float2* sc, const float* vz,
                                   const float* zs, const BPParams& p, unsigned long long* count,
                                   cudaStream_t s);
cudaError_t launch_backproject_f16(const __half* D, const float* scales, float* vol, const float2* sc,
                                   const float* vz, const float* zs, const BPParams& p, unsigned long long* count,
                                   cudaStream_t s);
cudaError_t launch_rebin_split(const float* raw, void* planes, float* row_scale, const float* d_beta,
                               const float* d_bidx, const RebinParams& p, int kp, float taps_l1, cudaStream_t s);
cudaError_t launch_filter_tc(const void* a_planes, const void* b_planes, int M, int nch, int kp, int np, int bn,
                             float* y32, __half* y16, const float* row_scale_in, float* row_scale_out, int* err,
                             cudaStream_t s);
int tc_choose_bn(int nch);
cudaError_t launch_thicken(const float* vn, float* out, const int* off, const int* idx, const float* w,
                           const float* ws, int nxy, int nzr, cudaStream_t s);
cudaError_t launch_synth(const wfbp_synth_scan& scan, const wfbp_ellipsoid* d_e, int ne, float* out,
                         cudaStream_t s);
