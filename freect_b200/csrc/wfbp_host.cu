// Host side of the B200 WFBP library: the C ABI of include/freect_wfbp.h.
//
// What the reference does in ReconstructionMachine (applications/fct_wfbp/src/
// ReconstructionMachine.cu) is split here into a context (geometry, slice
// lists, filter taps, per-view tables, thickening weights) and four
// asynchronous stages on a caller-chosen stream. Errors come back as status
// codes with a message in the context instead of exit().
#include "wfbp_internal.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>

#include <nvtx3/nvToolsExt.h>

#define WFBP_API extern "C" __attribute__((visibility("default")))

namespace {

int fail(wfbp_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

std::string hex_word(int h) {
  char b[16];
  snprintf(b, sizeof(b), "%x", (unsigned)h);
  return b;
}

#define CUDA_TRY(ctx, call)                                                                  \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      return fail((ctx), e_ == cudaErrorMemoryAllocation ? WFBP_ERR_OOM : WFBP_ERR_CUDA,      \
                  std::string(#call) + ": " + cudaGetErrorName(e_) + " " + cudaGetErrorString(e_)); \
    }                                                                                        \
  } while (0)

size_t next_pow2_at_least(size_t n) {
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

// r(t) of generate_filter (ReconstructionMachine.cu:493-498): sin and cos of
// the float argument in double precision, result stored as float.
float ramp_r(float t) {
  float v = (float)(sin((double)t) / (double)t + (cos((double)t) - 1.0f) / (double)(t * t));
  if (t == 0) v = 0.5f;
  return v;
}

int slice_lists(const CTGeometry* cg, const ReconConfig* rp, std::vector<float>& native, std::vector<float>& req) {
  native.clear();
  req.clear();
  const size_t cap = 1u << 22;
  if (rp->start_pos != rp->end_pos) {
    float span = rp->end_pos - rp->start_pos;
    float d_native = cg->collimated_slice_width * fabsf(span) / span;
    float d_req = rp->slice_pitch * fabsf(span) / span;
    if (!(fabsf(d_native) > 0) || !(fabsf(d_req) > 0)) return WFBP_ERR_INVALID_ARG;
    if (d_req > 0) {
      for (float loc = rp->start_pos; loc < rp->end_pos; loc += d_native) {
        native.push_back(loc);
        if (native.size() > cap) return WFBP_ERR_INVALID_ARG;
      }
      for (float loc = rp->start_pos; loc < rp->end_pos; loc += d_req) {
        req.push_back(loc);
        if (req.size() > cap) return WFBP_ERR_INVALID_ARG;
      }
    } else {
      for (float loc = rp->start_pos; loc > rp->end_pos; loc += d_native) {
        native.push_back(loc);
        if (native.size() > cap) return WFBP_ERR_INVALID_ARG;
      }
      for (float loc = rp->start_pos; loc > rp->end_pos; loc += d_req) {
        req.push_back(loc);
        if (req.size() > cap) return WFBP_ERR_INVALID_ARG;
      }
    }
  } else {
    native.push_back(rp->start_pos);
    req.push_back(rp->start_pos);
  }
  return WFBP_OK;
}

// Effective geometry of a flying-focal-spot scan: readings cycle through G
// focal states (fct_icd's order, applications/fct_icd/src/
// generate_system_matrix_ffs.cpp:242-290); one view per G readings, 2x
// channels (phi) / rows (z) at half the spacing, central channel 2 c0 + 1/2.
void ffs_effective(const CTGeometry* in, CTGeometry* out) {
  *out = *in;
  const int fp = in->ffs_phi ? 2 : 1, fz = in->ffs_z ? 2 : 1, G = fp * fz;
  out->total_number_of_projections = in->total_number_of_projections / G;
  out->projections_per_rotation = in->projections_per_rotation / G;
  out->num_detector_cols = in->num_detector_cols * fp;
  out->num_detector_cols_padded = 2 * out->num_detector_cols;
  out->num_detector_cols_padded_fft = next_pow2_at_least(2 * out->num_detector_cols);
  out->num_detector_rows = in->num_detector_rows * fz;
  out->num_detector_rows_padded = 2 * out->num_detector_rows;
  out->detector_pixel_size_col = in->detector_pixel_size_col / fp;
  out->detector_pixel_size_row = in->detector_pixel_size_row / fz;
  out->detector_central_col = in->ffs_phi ? 2.0f * in->detector_central_col + 0.5f : in->detector_central_col;
  out->detector_central_row = ((float)out->num_detector_rows - 1.0f) / 2.0f;
  out->collimated_slice_width =
      out->distance_source_to_isocenter * (out->detector_pixel_size_row / out->distance_source_to_detector);
  const float cone_offset = ((float)(out->num_detector_rows - 1)) / 2.0f;
  out->theta_cone =
      2.0f * (float)atan((double)(cone_offset * out->collimated_slice_width / out->distance_source_to_isocenter));
  out->acquisition_field_of_view =
      2.0f * out->distance_source_to_isocenter *
      (float)sin((double)((((float)out->num_detector_cols - 1.0f) / 2.0f) * out->detector_pixel_size_col *
                          (1.0f / out->distance_source_to_detector)));
}

int make_taps(const CTGeometry* cg, int window, float c, float a, const float* user, int n_user, float* taps, int n) {
  const float ds = cg->detector_pixel_size_col * cg->distance_source_to_isocenter / cg->distance_source_to_detector;
  if (!(ds > 0)) return WFBP_ERR_INVALID_ARG;
  if (window == WFBP_FILTER_REFERENCE) {
    const float pi_f = 3.141592653589f;  // ReconstructionMachine.cu:490
    for (int i = 0; i < n; i++)
      taps[i] = (c * c / (2.0f * ds)) * (a * ramp_r(c * pi_f * i) + (((1.0f - a) / 2.0f) * ramp_r(pi_f * c * i + pi_f)) +
                                         (((1.0f - a) / 2.0f) * ramp_r(pi_f * c * i - pi_f)));
  } else if (window == WFBP_FILTER_SHEPP_LOGAN) {
    for (int i = 0; i < n; i++) taps[i] = (float)(-2.0 / (M_PI * M_PI * (double)ds * (4.0 * i * (double)i - 1.0)));
  } else if (window == WFBP_FILTER_USER) {
    if (!user || n_user < 1) return WFBP_ERR_INVALID_ARG;
    for (int i = 0; i < n; i++) taps[i] = i < n_user ? user[i] : 0.0f;
  } else {
    return WFBP_ERR_INVALID_ARG;
  }
  return WFBP_OK;
}


void free_dev(void*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}
template <class T>
void free_dev(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

void release(wfbp_ctx* ctx) {
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  free_dev(ctx->d_taps);
  free_dev(ctx->d_chan_beta);
  free_dev(ctx->d_chan_bidx);
  free_dev(ctx->d_view_sc);
  free_dev(ctx->d_view_sc64);
  free_dev(ctx->d_view_z64);
  free_dev(ctx->d_chan64);
  free_dev(ctx->d_view_z);
  free_dev(ctx->d_z_native);
  free_dev(ctx->d_thick_off);
  free_dev(ctx->d_thick_idx);
  free_dev(ctx->d_thick_w);
  free_dev(ctx->d_thick_ws);
  free_dev(ctx->d_fuse_slab);
  free_dev(ctx->d_fuse_req);
  free_dev(ctx->d_fuse_bnd);
  free_dev(ctx->d_fuse_slab_tab);
  free_dev(ctx->d_fuse_tab);
  free_dev(ctx->d_bplanes);
  free_dev(ctx->d_err);
  free_dev(ctx->d_thickT_off);
  free_dev(ctx->d_thickT_idx);
  free_dev(ctx->d_thickT_w);
  free_dev(ctx->d_radj_cnt);
  free_dev(ctx->d_radj_idx);
  free_dev(ctx->d_radj_w);
  free_dev(ctx->d_tg_partial);
  free_dev(ctx->d_adj_scale);
  free_dev(ctx->d_adj_gvt);
  for (auto& e : ctx->ev_copy) cudaEventDestroy(e);
  ctx->ev_copy.clear();
  if (ctx->s_copy) cudaStreamDestroy(ctx->s_copy);
  if (ctx->s_back) cudaStreamDestroy(ctx->s_back);
  ctx->s_copy = nullptr;
  for (auto& b : ctx->s_bp) {
    if (b) cudaStreamDestroy(b);
    b = nullptr;
  }
  free_dev(ctx->s_rebinned);
  free_dev(ctx->s_filtered);
  free_dev(ctx->s_scales);
  free_dev(ctx->s_vol_native);
  free_dev(ctx->s_raw);
  free_dev(ctx->s_vol);
  free_dev(ctx->s_af);
  cudaSetDevice(prev);
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

BPParams bp_params(const wfbp_ctx* ctx) {
  BPParams p;
  p.nx = ctx->nx; p.ny = ctx->ny; p.nz = ctx->nz;
  p.nch = ctx->nch; p.nr = ctx->nr; p.V = ctx->V;
  p.P2 = ctx->gp.projections_per_half_turn;
  p.K = ctx->gp.n_half_turns;
  p.fov = ctx->rp.recon_fov; p.x0 = ctx->rp.x_origin; p.y0 = ctx->rp.y_origin;
  p.fov_half2 = ctx->gp.half_acquisition_fov_squared;
  p.z_rot = ctx->cg.z_rot;
  p.R2 = ctx->gp.distance_source_to_isocenter_squared;
  p.rR = ctx->gp.recip_distance_source_to_isocenter;
  p.zr2pi = ctx->gp.z_rot_over_2_pi;
  p.tanc = ctx->gp.tanf_theta_cone;
  p.ps = ctx->gp.pixel_scale;
  p.c0 = ctx->cg.detector_central_col;
  p.kp = (float)((double)ctx->nch + 1.75);
  p.hn = 0.5f * ((float)ctx->nr - 1.0f);
  p.nrm2 = (float)(ctx->nr - 2);
  p.ncm2 = (float)(ctx->nch - 2);
  p.dtheta = ctx->gp.two_pi_over_projections_per_rotation;
  p.sc64 = ctx->d_view_sc64;
  p.z64 = ctx->d_view_z64;
  return p;
}

// Stage buffer sizes for a filtered-row layout.
//   rebinned: FP32 [V][nr][nch], or (mixed) FP16 operand planes
//             [2][V*nrv][kp], row scales [V*nrv], view scales [V] and the
//             views' operand scales [V], each 256-byte aligned
//   filtered: reference layout [V][nr][nch] FP32/FP16, or backprojection
//             layout [V][nch][nrp] of 4-byte elements (FP32 or half2 pairs)
//   scales:   FP32 [V][nr] row scales (mixed, reference layout) or [V] view
//             scales (mixed, backprojection layout)
size_t al256(size_t n) { return (n + 255) & ~size_t(255); }

void stage_bytes(const wfbp_ctx* ctx, int layout, size_t* reb, size_t* filt, size_t* scal) {
  const size_t samples = (size_t)ctx->V * ctx->nr * ctx->nch;
  const bool bpl = layout == WFBP_LAYOUT_BACKPROJECTION;
  const size_t bpl_bytes = 4 * (size_t)ctx->V * ctx->nch * (size_t)std::max(ctx->bpt.nrp, 1);
  if (ctx->ext.precision == WFBP_PRECISION_MIXED) {
    const size_t rows = (size_t)ctx->V * ctx->nrv;
    *reb = al256(2 * rows * (size_t)ctx->tc_kp * sizeof(uint16_t)) + al256(rows * sizeof(float)) +
           al256((size_t)ctx->V * sizeof(float)) + (size_t)ctx->V * sizeof(float);
    *filt = bpl ? bpl_bytes : sizeof(uint16_t) * samples;
    *scal = bpl ? (size_t)ctx->V * sizeof(float) : (size_t)ctx->V * ctx->nr * sizeof(float);
  } else {
    *reb = sizeof(float) * samples;
    *filt = bpl ? bpl_bytes : sizeof(float) * samples;
    *scal = 0;
  }
}

template <class P>
void mixed_scale_ptrs(const wfbp_ctx* ctx, P rebinned, float** row_sc, float** view_sc, float** op_sc) {
  const size_t rows = (size_t)ctx->V * ctx->nrv;
  uint8_t* b = const_cast<uint8_t*>(reinterpret_cast<const uint8_t*>(rebinned));
  const size_t o_row = al256(2 * rows * (size_t)ctx->tc_kp * sizeof(uint16_t));
  const size_t o_view = o_row + al256(rows * sizeof(float));
  *row_sc = reinterpret_cast<float*>(b + o_row);
  *view_sc = reinterpret_cast<float*>(b + o_view);
  *op_sc = reinterpret_cast<float*>(b + o_view + al256((size_t)ctx->V * sizeof(float)));
}

// Sizes the TMA-staged backprojection for this geometry: the column tile, the
// channel window each view needs for it, and the most views of one theta~ that
// can reach a slab. Returns false if no configuration fits in shared
// memory (the generic kernel is used then).
// Slab-level view reach and the most views of one theta~ that can reach a
// 32-slice slab (a bound for 16-slice slabs too); both depend only on the
// geometry and the table positions.
void bp_reach(wfbp_ctx* ctx, const std::vector<float>& table) {
  const double R = ctx->cg.distance_source_to_isocenter;
  const double rmax = 0.5 * ctx->cg.acquisition_field_of_view;
  const double tanc = ctx->gp.tanf_theta_cone;
  // |z - z_j| <= |A| + l_hat tan for any valid (voxel, view); tighter than z_rot
  const double cone = (R + rmax) * tanc + (ctx->cg.z_rot / (2 * M_PI)) * asin(std::min(1.0, rmax / R));
  const double reach = std::min((double)ctx->cg.z_rot, cone) + 1e-3 * (1.0 + fabs(ctx->cg.z_rot));
  int nv_max = 0;
  const int nslab = (ctx->nz + 31) / 32;
  for (int sl = 0; sl < nslab; sl++) {
    float zmn = 3e38f, zmx = -3e38f;
    for (int i = sl * 32; i < std::min(ctx->nz, sl * 32 + 32); i++) {
      zmn = std::min(zmn, ctx->z_native[i]);
      zmx = std::max(zmx, ctx->z_native[i]);
    }
    const float lo = zmn - (float)reach, hi = zmx + (float)reach;
    for (int t = 0; t < ctx->P2; t++) {
      int n = 0;
      for (int k = 0; k < ctx->K; k++) {
        const float zt = table[t + k * ctx->P2];
        if (!(zt < lo || zt > hi)) n++;
      }
      nv_max = std::max(nv_max, n);
    }
  }
  ctx->bp_reach = (float)reach;
  ctx->bp_nv_max = std::max(1, nv_max);
  // A sample with its row in [0, nr - 2] has |z - z_j| <= cone; below z_rot
  // by a margin for rounding, the cull of cuda_kernels.cuh:232 never removes
  // one and the backprojection's records drop its row range
  ctx->bp_zcull = cone < (double)ctx->cg.z_rot * (1.0 - 1e-3) ? 0 : 1;
}

// Sizes one TMA backprojection configuration; false if it does not fit.
bool size_bp_tile(const wfbp_ctx* ctx, int tx, int ty, int cu, int nw, int slab, BPTile* out) {
  const double vx = ctx->rp.recon_fov / ctx->nx, vy = ctx->rp.recon_fov / ctx->ny;
  BPTile b;
  b.tx = tx;
  b.ty = ty;
  b.cu = cu;
  b.nw = nw;
  b.slab = slab;
  b.zb0 = 0;
  b.nzb = 0;
  b.zc = ctx->bp_zcull;
  const double ext = sqrt(pow((b.tx - 1) * vx, 2) + pow((b.ty - 1) * vy, 2));
  b.W = (int)ceil(ext * ctx->gp.pixel_scale) + 5;
  b.W = std::max(4, std::min(b.W, 256));
  b.nrp = (ctx->nr + 3) / 4 * 4;
  b.nv_max = ctx->bp_nv_max;
  b.slot_bytes = (int)((b.W * b.nrp * 4 + 127) / 128 * 128);
  b.reach = ctx->bp_reach;
  b.smem_bytes = 0;
  if (!bp_tma_supported(b) || b.nrp > 256 || b.W > ctx->nch) return false;
  const size_t smem = bp_tma_smem_bytes(b, 4);
  if (smem > 220 * 1024) return false;
  b.smem_bytes = (int)smem;
  *out = b;
  return true;
}

// (tile x, tile y, columns per pass, consumer warps, slab slices)
const int kBpCandidates[][5] = {
    {16, 16, 4, 16, 32}, {16, 16, 8, 16, 32}, {16, 8, 4, 16, 32},  {16, 8, 8, 16, 32},  {8, 16, 4, 16, 32},
    {8, 16, 8, 16, 32},  {8, 8, 4, 16, 32},   {16, 10, 4, 20, 32}, {16, 10, 8, 20, 32}, {10, 16, 4, 20, 32},
    {12, 8, 4, 24, 32},  {16, 16, 4, 16, 16}, {16, 16, 8, 16, 16}, {16, 10, 4, 20, 16}, {16, 20, 4, 20, 16},
    {16, 20, 8, 20, 16}, {16, 8, 4, 8, 32},   {8, 16, 4, 8, 32},   {16, 8, 8, 8, 32},   {8, 16, 8, 8, 32},
    {16, 8, 4, 8, 16},   {16, 8, 8, 8, 16},   {8, 16, 8, 8, 16}};

// ext.bp_slab, when set, admits only configurations with slabs of that height
bool slab_allowed(const wfbp_ctx* ctx, int slab) { return ctx->ext.bp_slab == 0 || ctx->ext.bp_slab == slab; }

bool choose_bp_tile(wfbp_ctx* ctx, const std::vector<float>& table) {
  bp_reach(ctx, table);
  for (auto& c : kBpCandidates) {
    if (!slab_allowed(ctx, c[4])) continue;
    BPTile b;
    if (size_bp_tile(ctx, c[0], c[1], c[2], c[3], c[4], &b)) {
      ctx->bpt = b;
      return true;
    }
  }
  return false;
}

}  // namespace

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------

WFBP_API int wfbp_configure_geometry(const wfbp_scan_meta* m, const float* table, CTGeometry* cg, GPUPrecompute* gp) {
  if (!m || !table || !cg || !gp) return WFBP_ERR_INVALID_ARG;
  if (m->projections_per_rotation < 2 || m->total_num_projections <= m->projections_per_rotation ||
      m->detector_channels < 4 || m->detector_rows < 2 || !(m->dist_source_to_detector > 0) ||
      !(m->dist_source_to_isocenter > 0) || !(m->detector_transverse_spacing > 0) ||
      !(m->detector_axial_spacing > 0))
    return WFBP_ERR_INVALID_ARG;
  memset(cg, 0, sizeof(*cg));
  memset(gp, 0, sizeof(*gp));
  // ReconstructionMachine.cu:48-69
  cg->total_number_of_projections = (size_t)m->total_num_projections;
  cg->projections_per_rotation = (size_t)m->projections_per_rotation;
  cg->detector_pixel_size_col = m->detector_transverse_spacing;
  cg->detector_pixel_size_row = m->detector_axial_spacing;
  cg->num_detector_cols = (size_t)m->detector_channels;
  cg->num_detector_cols_padded = 2 * (size_t)m->detector_channels;
  cg->num_detector_cols_padded_fft = next_pow2_at_least(2 * (size_t)m->detector_channels);
  cg->num_detector_rows = (size_t)m->detector_rows;
  cg->num_detector_rows_padded = 2 * (size_t)m->detector_rows;
  cg->detector_central_col = m->detector_central_channel;
  cg->detector_central_row = m->detector_central_row;
  cg->distance_source_to_isocenter = m->dist_source_to_isocenter;
  cg->distance_source_to_detector = m->dist_source_to_detector;
  cg->collimated_slice_width = m->dist_source_to_isocenter * (m->detector_axial_spacing / m->dist_source_to_detector);
  cg->z_rot = fabsf(table[m->projections_per_rotation] - table[0]);
  float cone_offset = ((float)(cg->num_detector_rows - 1)) / 2.0f;
  cg->theta_cone = 2.0f * (float)atan((double)(cone_offset * cg->collimated_slice_width / cg->distance_source_to_isocenter));
  cg->acquisition_field_of_view =
      2.0f * cg->distance_source_to_isocenter *
      (float)sin((double)((((float)cg->num_detector_cols - 1.0f) / 2.0f) * m->detector_transverse_spacing *
                          (1.0f / cg->distance_source_to_detector)));
  cg->anode_angle = m->anode_angle;
  cg->ffs_phi = (m->ffs_mode & WFBP_FFS_PHI) != 0;
  cg->ffs_z = (m->ffs_mode & WFBP_FFS_Z) != 0;
  cg->ffs_diag = false;
  // recon_structs.h:69-83
  const float pi_f = 3.1415926535897f;
  gp->half_acquisition_fov = 0.5f * cg->acquisition_field_of_view;
  gp->half_acquisition_fov_squared = gp->half_acquisition_fov * gp->half_acquisition_fov;
  gp->projections_per_half_turn = (int)(cg->projections_per_rotation / 2);
  gp->n_half_turns = (int)(cg->total_number_of_projections / (size_t)gp->projections_per_half_turn);
  gp->distance_source_to_isocenter_squared = cg->distance_source_to_isocenter * cg->distance_source_to_isocenter;
  gp->z_rot_over_2_pi = cg->z_rot / (2.0f * pi_f);
  gp->recip_distance_source_to_detector = 1.0f / cg->distance_source_to_detector;
  gp->recip_distance_source_to_isocenter = 1.0f / cg->distance_source_to_isocenter;
  gp->tanf_theta_cone = (float)tan((double)(cg->theta_cone / 2.0f));
  gp->pixel_scale = cg->distance_source_to_detector / (cg->distance_source_to_isocenter * cg->detector_pixel_size_col);
  gp->two_pi_over_projections_per_rotation = 2.0f * pi_f / (float)cg->projections_per_rotation;
  return WFBP_OK;
}

WFBP_API int wfbp_effective_geometry(const CTGeometry* cg, CTGeometry* eff) {
  if (!cg || !eff) return WFBP_ERR_INVALID_ARG;
  ffs_effective(cg, eff);
  return WFBP_OK;
}

WFBP_API int wfbp_slice_locations(const CTGeometry* cg, const ReconConfig* rp, float* native_z, int native_cap,
                                  int* n_native, float* requested_z, int requested_cap, int* n_requested) {
  if (!cg || !rp) return WFBP_ERR_INVALID_ARG;
  std::vector<float> nat, req;
  int st = slice_lists(cg, rp, nat, req);
  if (st) return st;
  if (n_native) *n_native = (int)nat.size();
  if (n_requested) *n_requested = (int)req.size();
  if (native_z) std::copy(nat.begin(), nat.begin() + std::min<size_t>(nat.size(), (size_t)std::max(native_cap, 0)), native_z);
  if (requested_z)
    std::copy(req.begin(), req.begin() + std::min<size_t>(req.size(), (size_t)std::max(requested_cap, 0)), requested_z);
  return WFBP_OK;
}

WFBP_API int wfbp_filter_taps(const CTGeometry* cg, int window, float c, float a, float* taps, int n) {
  if (!cg || !taps || n < 1) return WFBP_ERR_INVALID_ARG;
  return make_taps(cg, window, c, a, nullptr, 0, taps, n);
}

WFBP_API const char* wfbp_status_string(int status) {
  switch (status) {
    case WFBP_OK: return "WFBP_OK";
    case WFBP_ERR_INVALID_ARG: return "WFBP_ERR_INVALID_ARG";
    case WFBP_ERR_OOM: return "WFBP_ERR_OOM";
    case WFBP_ERR_CUDA: return "WFBP_ERR_CUDA";
    case WFBP_ERR_TIMEOUT: return "WFBP_ERR_TIMEOUT";
    case WFBP_ERR_UNSUPPORTED: return "WFBP_ERR_UNSUPPORTED";
    case WFBP_ERR_STATE: return "WFBP_ERR_STATE";
  }
  return "WFBP_ERR_UNKNOWN";
}

WFBP_API const char* wfbp_last_error(const wfbp_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

namespace {
// Native / requested slice lists -> thickening weights (cuda_kernels.cuh:
// 303-317, float arithmetic), their transpose for the adjoint, and the device
// tables; re-sizes the backprojection launch when the views are known.
int setup_slices(wfbp_ctx* ctx) {
  ctx->adj_scale_valid = false;
  ctx->fuse_slab = 0;
  ctx->nz = (int)ctx->z_native.size();
  ctx->nzr = (int)ctx->z_req.size();
  ctx->gp.n_slices_native = ctx->nz;
  ctx->gp.n_slices_requested = ctx->nzr;
  ctx->thick_off.assign(ctx->nzr + 1, 0);
  ctx->thick_idx.clear();
  ctx->thick_w.clear();
  std::vector<float> ws(ctx->nzr, 0.0f);
  for (int r = 0; r < ctx->nzr; r++) {
    ctx->thick_off[r] = (int)ctx->thick_idx.size();
    float wsum = 0.0f;
    for (int i = 0; i < ctx->nz; i++) {
      float w = fmaxf(0.0f, 1.0f - fabsf(ctx->z_native[i] - ctx->z_req[r]) / ctx->rp.slice_thickness);
      if (w == 0.0f) continue;
      wsum += w;
      ctx->thick_idx.push_back(i);
      ctx->thick_w.push_back(w);
    }
    ws[r] = wsum;
  }
  ctx->thick_off[ctx->nzr] = (int)ctx->thick_idx.size();
  // transposed CSR for the adjoint: native slice -> (requested slice, w / sum w)
  std::vector<int> tT_off(ctx->nz + 1, 0), tT_idx(ctx->thick_idx.size());
  std::vector<float> tT_w(ctx->thick_idx.size());
  for (size_t t = 0; t < ctx->thick_idx.size(); t++) tT_off[ctx->thick_idx[t] + 1]++;
  for (int n = 0; n < ctx->nz; n++) tT_off[n + 1] += tT_off[n];
  {
    std::vector<int> fill(tT_off.begin(), tT_off.end() - 1);
    for (int r = 0; r < ctx->nzr; r++)
      for (int t = ctx->thick_off[r]; t < ctx->thick_off[r + 1]; t++) {
        const int n = ctx->thick_idx[t];
        tT_idx[fill[n]] = r;
        tT_w[fill[n]] = ctx->thick_w[t] / ws[r];
        fill[n]++;
      }
  }
  DeviceGuard g(ctx->device);
  free_dev(ctx->d_z_native);
  free_dev(ctx->d_thick_off);
  free_dev(ctx->d_thick_idx);
  free_dev(ctx->d_thick_w);
  free_dev(ctx->d_thick_ws);
  free_dev(ctx->d_thickT_off);
  free_dev(ctx->d_thickT_idx);
  free_dev(ctx->d_thickT_w);
  // the volume sizes may change: the context's own scratch is re-allocated on demand
  free_dev(ctx->s_vol_native);
  free_dev(ctx->s_vol);
  auto up = [&](void** dst, const void* src, size_t bytes) -> cudaError_t {
    cudaError_t e1 = cudaMalloc(dst, bytes > 0 ? bytes : 4);
    if (e1 != cudaSuccess) return e1;
    if (src && bytes) return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    return cudaSuccess;
  };
  cudaError_t ce = cudaSuccess;
  if (!ce) ce = up((void**)&ctx->d_z_native, ctx->z_native.data(), sizeof(float) * ctx->nz);
  if (!ce) ce = up((void**)&ctx->d_thick_off, ctx->thick_off.data(), sizeof(int) * ctx->thick_off.size());
  if (!ce) ce = up((void**)&ctx->d_thick_idx, ctx->thick_idx.data(), sizeof(int) * ctx->thick_idx.size());
  if (!ce) ce = up((void**)&ctx->d_thick_w, ctx->thick_w.data(), sizeof(float) * ctx->thick_w.size());
  if (!ce) ce = up((void**)&ctx->d_thick_ws, ws.data(), sizeof(float) * ws.size());
  if (!ce) ce = up((void**)&ctx->d_thickT_off, tT_off.data(), sizeof(int) * tT_off.size());
  if (!ce) ce = up((void**)&ctx->d_thickT_idx, tT_idx.data(), sizeof(int) * tT_idx.size());
  if (!ce) ce = up((void**)&ctx->d_thickT_w, tT_w.data(), sizeof(float) * tT_w.size());
  if (ce) return fail(ctx, ce == cudaErrorMemoryAllocation ? WFBP_ERR_OOM : WFBP_ERR_CUDA, "slice tables");
  if (ctx->views_set) {
    const int nrp = ctx->bpt.nrp;
    ctx->bp_tma_ok = choose_bp_tile(ctx, ctx->view_table);
    ctx->bpt.nrp = nrp;
  }
  return WFBP_OK;
}
}  // namespace

WFBP_API int wfbp_recon_kernel_filter(int recon_kernel, int* window, float* c, float* a) {
  if (!window || !c || !a) return WFBP_ERR_INVALID_ARG;
  // ramp.m: a = 1 ramp, 0.5 Hann, 0.54 Hamming; c = 1 (no cut-off)
  switch (recon_kernel) {
    case WFBP_RECON_KERNEL_RAMLAK: *window = WFBP_FILTER_REFERENCE; *c = 1.0f; *a = 1.0f; return WFBP_OK;
    case WFBP_RECON_KERNEL_SHEPP_LOGAN: *window = WFBP_FILTER_SHEPP_LOGAN; *c = 1.0f; *a = 1.0f; return WFBP_OK;
    case WFBP_RECON_KERNEL_HANN: *window = WFBP_FILTER_REFERENCE; *c = 1.0f; *a = 0.5f; return WFBP_OK;
    case WFBP_RECON_KERNEL_HAMMING: *window = WFBP_FILTER_REFERENCE; *c = 1.0f; *a = 0.54f; return WFBP_OK;
    default: return WFBP_ERR_INVALID_ARG;
  }
}

WFBP_API int wfbp_ctx_create(const CTGeometry* cg, const ReconConfig* rp, const wfbp_ext* ext, int device,
                             wfbp_ctx** out) {
  if (!cg || !rp || !out) return WFBP_ERR_INVALID_ARG;
  *out = nullptr;
  wfbp_ext e;
  memset(&e, 0, sizeof(e));
  e.version = WFBP_EXT_VERSION;
  e.precision = WFBP_PRECISION_FP32;
  e.filter_window = WFBP_FILTER_REFERENCE;
  e.filter_c = 1.0f;
  e.filter_a = 1.0f;
  if (ext) {
    if (ext->version != WFBP_EXT_VERSION) return WFBP_ERR_INVALID_ARG;
    e = *ext;
  }
  if (e.precision != WFBP_PRECISION_FP32 && e.precision != WFBP_PRECISION_MIXED) return WFBP_ERR_INVALID_ARG;
  // ReconConfig.recon_kernel picks the filter when the extension leaves it at
  // its default (fct_wfbp parses the field, parse_config.cpp:53, but
  // generate_filter ignores it, ReconstructionMachine.cu:204)
  if (e.filter_window == WFBP_FILTER_REFERENCE &&
      ((e.filter_c == 1.0f && e.filter_a == 1.0f) || (e.filter_c == 0.0f && e.filter_a == 0.0f))) {
    if (wfbp_recon_kernel_filter(rp->recon_kernel, &e.filter_window, &e.filter_c, &e.filter_a))
      return WFBP_ERR_INVALID_ARG;
  }
  if (e.bp_slab != 0 && e.bp_slab != 16 && e.bp_slab != 32) return WFBP_ERR_INVALID_ARG;
  if (e.adjoint_scale_table != 0 && e.adjoint_scale_table != -1) return WFBP_ERR_INVALID_ARG;
  if (e.filtered_layout != WFBP_LAYOUT_REFERENCE && e.filtered_layout != WFBP_LAYOUT_BACKPROJECTION)
    return WFBP_ERR_INVALID_ARG;
  if (e.precision == WFBP_PRECISION_MIXED && cg->num_detector_rows > 128) return WFBP_ERR_UNSUPPORTED;
  if (cg->ffs_diag) return WFBP_ERR_UNSUPPORTED;
  // With a flying focal spot the stages work on the effective geometry; the
  // raw frames keep the reading geometry `cg_read`.
  const CTGeometry* cg_read = cg;
  CTGeometry cg_eff;
  const int G = (cg->ffs_phi ? 2 : 1) * (cg->ffs_z ? 2 : 1);
  if (G > 1) {
    if (cg->total_number_of_projections % G || cg->projections_per_rotation % G) return WFBP_ERR_INVALID_ARG;
    ffs_effective(cg, &cg_eff);
    cg = &cg_eff;
  }
  if (cg->projections_per_rotation < 2 || cg->total_number_of_projections <= cg->projections_per_rotation / 2 ||
      cg->num_detector_cols < 4 || cg->num_detector_rows < 2 || rp->nx < 1 || rp->ny < 1 ||
      !(rp->recon_fov > 0) || !(rp->slice_thickness > 0) || !(cg->distance_source_to_isocenter > 0) ||
      !(cg->distance_source_to_detector > 0) || !(cg->detector_pixel_size_col > 0) ||
      !(cg->collimated_slice_width > 0) || cg->num_detector_cols > 8192 || cg->num_detector_rows > 1024 ||
      cg->total_number_of_projections > (1u << 24) || rp->nx > 8192 || rp->ny > 8192 ||
      std::isnan(rp->adaptive_filtration_s))
    return WFBP_ERR_INVALID_ARG;

  wfbp_ctx* ctx = new (std::nothrow) wfbp_ctx();
  if (!ctx) return WFBP_ERR_OOM;
  ctx->cg = *cg;
  ctx->cg_read = *cg_read;
  ctx->G = G;
  ctx->rp = *rp;
  ctx->ext = e;
  ctx->device = device;
  ctx->V = (int)cg->total_number_of_projections;
  ctx->nr = (int)cg->num_detector_rows;
  ctx->nch = (int)cg->num_detector_cols;
  ctx->P = (int)cg->projections_per_rotation;
  ctx->n_readings = (int)cg_read->total_number_of_projections;
  ctx->raw_rows = (int)cg_read->num_detector_rows;
  ctx->raw_ch = (int)cg_read->num_detector_cols;
  ctx->nx = (int)rp->nx;
  ctx->ny = (int)rp->ny;
  ctx->bpt.nrp = (ctx->nr + 3) / 4 * 4;

  // derived constants (recon_structs.h:69-83) from the given geometry
  const float pi_f = 3.1415926535897f;
  GPUPrecompute& gp = ctx->gp;
  memset(&gp, 0, sizeof(gp));
  gp.half_acquisition_fov = 0.5f * cg->acquisition_field_of_view;
  gp.half_acquisition_fov_squared = gp.half_acquisition_fov * gp.half_acquisition_fov;
  gp.projections_per_half_turn = (int)(cg->projections_per_rotation / 2);
  gp.n_half_turns = (int)(cg->total_number_of_projections / (size_t)gp.projections_per_half_turn);
  gp.distance_source_to_isocenter_squared = cg->distance_source_to_isocenter * cg->distance_source_to_isocenter;
  gp.z_rot_over_2_pi = cg->z_rot / (2.0f * pi_f);
  gp.recip_distance_source_to_detector = 1.0f / cg->distance_source_to_detector;
  gp.recip_distance_source_to_isocenter = 1.0f / cg->distance_source_to_isocenter;
  gp.tanf_theta_cone = (float)tan((double)(cg->theta_cone / 2.0f));
  gp.pixel_scale = cg->distance_source_to_detector / (cg->distance_source_to_isocenter * cg->detector_pixel_size_col);
  gp.two_pi_over_projections_per_rotation = 2.0f * pi_f / (float)cg->projections_per_rotation;
  ctx->P2 = gp.projections_per_half_turn;
  ctx->K = gp.n_half_turns;

  int st = slice_lists(cg, rp, ctx->z_native, ctx->z_req);
  if (st) { delete ctx; return st; }

  ctx->taps.resize(ctx->nch);
  st = make_taps(cg, e.filter_window, e.filter_c, e.filter_a, e.user_taps, e.n_user_taps, ctx->taps.data(), ctx->nch);
  if (st) { delete ctx; return st; }

  DeviceGuard g(device);
  auto alloc_copy = [&](void** dst, const void* src, size_t bytes) -> cudaError_t {
    cudaError_t e1 = cudaMalloc(dst, bytes > 0 ? bytes : 4);
    if (e1 != cudaSuccess) return e1;
    if (src && bytes) return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    return cudaSuccess;
  };
  cudaError_t ce = cudaSuccess;
  if (!ce) ce = alloc_copy((void**)&ctx->d_taps, ctx->taps.data(), sizeof(float) * ctx->nch);
  if (!ce) ce = alloc_copy((void**)&ctx->d_chan_beta, nullptr, sizeof(float) * ctx->nch);
  if (!ce) ce = alloc_copy((void**)&ctx->d_chan_bidx, nullptr, sizeof(float) * ctx->nch);
  if (!ce) ce = alloc_copy((void**)&ctx->d_view_sc, nullptr, sizeof(float2) * ctx->V);
  if (!ce) ce = alloc_copy((void**)&ctx->d_view_sc64, nullptr, sizeof(double2) * ctx->V);
  if (!ce) ce = alloc_copy((void**)&ctx->d_view_z64, nullptr, sizeof(double) * ctx->V);
  if (!ce) ce = alloc_copy((void**)&ctx->d_view_z, nullptr, sizeof(float) * ctx->V);
  if (!ce) ce = alloc_copy((void**)&ctx->d_err, nullptr, sizeof(int));
  // adaptive filtration (ReconConfig.adaptive_filtration_s > 0): the filtered
  // readings live in context memory allocated here, so no stage call allocates
  ctx->af_s = rp->adaptive_filtration_s > 0.0f ? std::min(rp->adaptive_filtration_s, 1.0f) : 0.0f;
  if (!ce && ctx->af_s > 0.0f)
    ce = alloc_copy((void**)&ctx->s_af, nullptr,
                    sizeof(float) * (size_t)ctx->n_readings * ctx->raw_rows * ctx->raw_ch);
  if (!ce) ce = cudaMemset(ctx->d_err, 0, sizeof(int));
  if (!ce && e.precision == WFBP_PRECISION_MIXED) {
    // Toeplitz operand T[n][k] = h[|n - k|] scaled by the power of two
    // tap_scale (the largest with tap_scale max|h| <= 16384), split into FP16
    // hi / lo planes (22 bits), zero-padded to [np][kp]
    const int nch = ctx->nch;
    ctx->tc_kp = (nch + 63) / 64 * 64;
    ctx->nrv = 1;
    while (ctx->nrv < ctx->nr) ctx->nrv <<= 1;
    ctx->tc_bn = tc_choose_bn(nch);
    ctx->tc_np = (nch + ctx->tc_bn - 1) / ctx->tc_bn * ctx->tc_bn;
    const size_t plane = (size_t)ctx->tc_np * ctx->tc_kp;
    std::vector<uint16_t> b(2 * plane, 0);
    double l1 = 0.0, hmax = 0.0;
    for (int d = 0; d < nch; d++) {
      l1 += (d ? 2.0 : 1.0) * fabs((double)ctx->taps[d]);
      hmax = std::max(hmax, fabs((double)ctx->taps[d]));
    }
    ctx->taps_l1 = (float)l1;
    ctx->tap_scale = hmax > 0.0 ? (float)exp2(floor(log2(16384.0 / hmax))) : 1.0f;
    // FP16 row pairs of the backprojection layout: one power of two >= the
    // taps' L1 norm divides every filtered row of the scan, so a stored value
    // is at most max|rebinned sample| (|y| <= max|x| sum|h|) and keeps FP16's
    // 11 significant bits; the backprojection multiplies it back once
    ctx->pair_scale = l1 > 0.0 ? (float)exp2(ceil(log2(l1))) : 1.0f;
    for (int n = 0; n < nch; n++)
      for (int k = 0; k < nch; k++) {
        const float h = ctx->taps[n > k ? n - k : k - n] * ctx->tap_scale;  // power of two: exact
        const __half hi = __float2half_rn(h);
        const __half lo = __float2half_rn(h - __half2float(hi));
        b[(size_t)n * ctx->tc_kp + k] = __half_as_ushort(hi);
        b[plane + (size_t)n * ctx->tc_kp + k] = __half_as_ushort(lo);
      }
    ce = alloc_copy(&ctx->d_bplanes, b.data(), sizeof(uint16_t) * b.size());
    // FP64 sample coordinates of the mixed form's rebin (rebin_kernel,
    // cuda_kernels.cuh:17-22, in double): per output channel the source
    // channel index (NaN off the detector) and beta / dtheta per reading
    const double c0 = cg->detector_central_col, dcol = cg->detector_pixel_size_col,
                 sdd = cg->distance_source_to_detector;
    const double dth = 2.0 * M_PI / (double)ctx->cg_read.projections_per_rotation;
    std::vector<double2> ch(nch);
    for (int c = 0; c < nch; c++) {
      const double beta = asin(((double)c - c0) * dcol / sdd);
      const double bidx = beta * sdd / dcol + c0;
      ch[c] = make_double2(bidx < 0.0 || bidx >= (double)nch || std::isnan(bidx) ? NAN : bidx, beta / dth);
    }
    if (!ce) ce = alloc_copy((void**)&ctx->d_chan64, ch.data(), sizeof(double2) * nch);
  }
  if (!ce) ce = launch_rebin_tables(ctx->d_chan_beta, ctx->d_chan_bidx, ctx->nch, cg->detector_central_col,
                                    cg->detector_pixel_size_col, cg->distance_source_to_detector, 0);
  if (!ce) ce = cudaDeviceSynchronize();
  if (ce) {
    int code = ce == cudaErrorMemoryAllocation ? WFBP_ERR_OOM : WFBP_ERR_CUDA;
    release(ctx);
    delete ctx;
    return code;
  }
  st = setup_slices(ctx);
  if (st) {
    release(ctx);
    delete ctx;
    return st;
  }
  *out = ctx;
  return WFBP_OK;
}

WFBP_API int wfbp_ctx_destroy(wfbp_ctx* ctx) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  release(ctx);
  delete ctx;
  return WFBP_OK;
}

WFBP_API int wfbp_query(const wfbp_ctx* ctx, wfbp_dims* d) {
  if (!ctx || !d) return WFBP_ERR_INVALID_ARG;
  memset(d, 0, sizeof(*d));
  d->n_views = ctx->V;
  d->n_rows = ctx->nr;
  d->n_channels = ctx->nch;
  d->n_readings = ctx->n_readings;
  d->raw_rows = ctx->raw_rows;
  d->raw_channels = ctx->raw_ch;
  d->nx = ctx->nx;
  d->ny = ctx->ny;
  d->n_slices_native = ctx->nz;
  d->n_slices_requested = ctx->nzr;
  d->precision = ctx->ext.precision;
  d->raw_bytes = sizeof(float) * (size_t)ctx->n_readings * ctx->raw_rows * ctx->raw_ch;
  stage_bytes(ctx, ctx->ext.filtered_layout, &d->rebinned_bytes, &d->filtered_bytes, &d->row_scale_bytes);
  d->native_volume_bytes = sizeof(float) * (size_t)ctx->nz * ctx->nx * ctx->ny;
  d->volume_bytes = sizeof(float) * (size_t)ctx->nzr * ctx->nx * ctx->ny;
  return WFBP_OK;
}

WFBP_API int wfbp_set_views(wfbp_ctx* ctx, const float* tube, const float* table) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!tube || !table) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_set_views: null array");
  for (int j = 0; j < ctx->n_readings; j++)
    if (!isfinite(tube[j]) || !isfinite(table[j]))
      return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_set_views: non-finite angle or table position at reading " +
                                                 std::to_string(j));
  // one view per G readings (flying focal spot), at the group's first reading
  std::vector<float> tv(ctx->V), zv(ctx->V);
  for (int v = 0; v < ctx->V; v++) {
    tv[v] = tube[(size_t)v * ctx->G];
    zv[v] = table[(size_t)v * ctx->G];
  }
  tube = tv.data();
  table = zv.data();
  DeviceGuard g(ctx->device);
  float *d_t = nullptr, *d_z = nullptr;
  CUDA_TRY(ctx, cudaMalloc(&d_t, sizeof(float) * ctx->V));
  cudaError_t e = cudaMalloc(&d_z, sizeof(float) * ctx->V);
  if (!e) e = cudaMemcpy(d_t, tube, sizeof(float) * ctx->V, cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(d_z, table, sizeof(float) * ctx->V, cudaMemcpyHostToDevice);
  if (!e) e = launch_view_tables(d_t, d_z, ctx->d_view_sc, ctx->d_view_z, ctx->V, 0);
  if (!e) {
    // FP64 per-view geometry: sin / cos of the tube angle and the table
    // position in double (the mixed form's backprojection records)
    std::vector<double2> sc64(ctx->V);
    std::vector<double> z64(ctx->V);
    for (int v = 0; v < ctx->V; v++) {
      sc64[v] = make_double2(sin((double)tube[v]), cos((double)tube[v]));
      z64[v] = (double)table[v];
    }
    e = cudaMemcpy(ctx->d_view_sc64, sc64.data(), sizeof(double2) * ctx->V, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(ctx->d_view_z64, z64.data(), sizeof(double) * ctx->V, cudaMemcpyHostToDevice);
  }
  if (!e) e = cudaDeviceSynchronize();
  cudaFree(d_t);
  cudaFree(d_z);
  CUDA_TRY(ctx, e);
  ctx->view_table.assign(table, table + ctx->V);
  ctx->adj_scale_valid = false;
  const int nrp = ctx->bpt.nrp;
  ctx->bp_tma_ok = choose_bp_tile(ctx, ctx->view_table);
  ctx->bpt.nrp = nrp;
  ctx->views_set = true;
  return WFBP_OK;
}

WFBP_API int wfbp_set_reading_offset(wfbp_ctx* ctx, int offset) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (offset < 0 || offset % ctx->G != 0)
    return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_set_reading_offset: need a non-negative multiple of the readings per view");
  ctx->reading_offset = offset;
  return WFBP_OK;
}

WFBP_API int wfbp_set_slices(wfbp_ctx* ctx, const float* native_z, int n_native, const float* requested_z,
                             int n_requested) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!native_z || !requested_z || n_native < 1 || n_requested < 1)
    return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_set_slices: need at least one native and one requested slice");
  for (int i = 0; i < n_native; i++)
    if (!isfinite(native_z[i])) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_set_slices: non-finite native z");
  for (int i = 0; i < n_requested; i++)
    if (!isfinite(requested_z[i])) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_set_slices: non-finite requested z");
  // monotone native list (the backprojection adjoint and the slab planning rely on it)
  if (n_native >= 2 && !(native_z[1] != native_z[0]))
    return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_set_slices: native slices must be strictly monotone");
  for (int i = 2; i < n_native; i++)
    if ((native_z[i] - native_z[i - 1]) * (native_z[1] - native_z[0]) <= 0.0f)
      return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_set_slices: native slices must be strictly monotone");
  ctx->z_native.assign(native_z, native_z + n_native);
  ctx->z_req.assign(requested_z, requested_z + n_requested);
  return setup_slices(ctx);
}

WFBP_API int wfbp_bp_configs(const wfbp_ctx* ctx, wfbp_bp_config* out, int cap, int* n) {
  if (!ctx || !n || cap < 0 || (cap > 0 && !out)) return WFBP_ERR_INVALID_ARG;
  if (!ctx->views_set) return WFBP_ERR_STATE;
  int k = 0;
  for (auto& c : kBpCandidates) {
    BPTile b;
    if (!slab_allowed(ctx, c[4]) || !size_bp_tile(ctx, c[0], c[1], c[2], c[3], c[4], &b)) continue;
    if (k < cap) {
      out[k].tile_x = c[0];
      out[k].tile_y = c[1];
      out[k].cols_per_step = c[2];
      out[k].consumer_warps = c[3];
      out[k].slab = c[4];
    }
    k++;
  }
  *n = k;
  return WFBP_OK;
}

WFBP_API int wfbp_get_bp_config(const wfbp_ctx* ctx, wfbp_bp_config* c) {
  if (!ctx || !c) return WFBP_ERR_INVALID_ARG;
  if (!ctx->views_set) return WFBP_ERR_STATE;
  if (!ctx->bp_tma_ok) return WFBP_ERR_UNSUPPORTED;
  c->tile_x = ctx->bpt.tx;
  c->tile_y = ctx->bpt.ty;
  c->cols_per_step = ctx->bpt.cu;
  c->consumer_warps = ctx->bpt.nw;
  c->slab = ctx->bpt.slab;
  return WFBP_OK;
}

WFBP_API int wfbp_set_bp_config(wfbp_ctx* ctx, const wfbp_bp_config* c) {
  if (!ctx || !c) return WFBP_ERR_INVALID_ARG;
  if (!ctx->views_set) return fail(ctx, WFBP_ERR_STATE, "wfbp_set_bp_config: call wfbp_set_views first");
  BPTile b;
  const int nw = c->consumer_warps ? c->consumer_warps : BT_CWARPS;
  const int slab = c->slab ? c->slab : (ctx->ext.bp_slab ? ctx->ext.bp_slab : 32);
  if (!slab_allowed(ctx, slab) || !size_bp_tile(ctx, c->tile_x, c->tile_y, c->cols_per_step, nw, slab, &b))
    return fail(ctx, WFBP_ERR_UNSUPPORTED, "wfbp_set_bp_config: configuration " + std::to_string(c->tile_x) + "x" +
                                               std::to_string(c->tile_y) + "/" + std::to_string(c->cols_per_step) + "w" +
                                               std::to_string(nw) + "s" + std::to_string(slab) +
                                               " is not supported for this geometry");
  ctx->bpt = b;
  ctx->bp_tma_ok = true;
  return WFBP_OK;
}

WFBP_API int wfbp_check_device_status(wfbp_ctx* ctx) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  DeviceGuard g(ctx->device);
  int h = 0;
  CUDA_TRY(ctx, cudaMemcpy(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) {
    cudaMemset(ctx->d_err, 0, sizeof(int));
    if (h == WFBP_ERR_TIMEOUT) return fail(ctx, WFBP_ERR_TIMEOUT, "a bounded device-side wait gave up");
    if (h & WFBP_ERRBIT_F16_RANGE)
      return fail(ctx, WFBP_ERR_UNSUPPORTED,
                  "mixed precision: a filtered row exceeds the FP16 row pairs' range (16384 x the scan's "
                  "power-of-two scale; rebinned samples above 16384)");
    return fail(ctx, WFBP_ERR_CUDA, "device-side sizing check failed (error word 0x" + hex_word(h) + ")");
  }
  return WFBP_OK;
}

WFBP_API int wfbp_selftest_bounded_wait(wfbp_ctx* ctx, int limit_ms, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (limit_ms < 1 || limit_ms > 10000) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_selftest_bounded_wait: limit 1-10000 ms");
  DeviceGuard g(ctx->device);
  CUDA_TRY(ctx, launch_selftest_wait(ctx->d_err, (unsigned long long)limit_ms * 1000000ull, (cudaStream_t)stream));
  return WFBP_OK;
}

WFBP_API int wfbp_get_geometry(const wfbp_ctx* ctx, CTGeometry* cg, GPUPrecompute* gp) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (cg) *cg = ctx->cg;
  if (gp) *gp = ctx->gp;
  return WFBP_OK;
}

WFBP_API int wfbp_get_slices(const wfbp_ctx* ctx, float* native_z, float* requested_z) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (native_z) std::copy(ctx->z_native.begin(), ctx->z_native.end(), native_z);
  if (requested_z) std::copy(ctx->z_req.begin(), ctx->z_req.end(), requested_z);
  return WFBP_OK;
}

// ---------------------------------------------------------------------------
// stages
// ---------------------------------------------------------------------------

namespace {
RebinParams rebin_params(const wfbp_ctx* ctx) {
  RebinParams p;
  p.V = ctx->V;
  p.nr = ctx->nr;
  p.nch = ctx->nch;
  p.dth = 2.0f * 3.14159265f / (float)ctx->cg_read.projections_per_rotation;  // cuda_kernels.cuh:15
  p.q8 = ctx->ext.tex_weights ? 1 : 0;
  p.G = ctx->G;
  p.phi = ctx->cg_read.ffs_phi ? 1 : 0;
  p.zf = ctx->cg_read.ffs_z ? 1 : 0;
  p.nch_raw = ctx->raw_ch;
  p.nr_raw = ctx->raw_rows;
  p.voff = ctx->reading_offset / ctx->G;
  return p;
}
}  // namespace

namespace {
// Rebin of views [vb, ve) (all: 0, V).
int do_rebin(wfbp_ctx* ctx, const float* raw, void* rebinned, int vb, int ve, void* stream) {
  const RebinParams p = rebin_params(ctx);
  if (ctx->ext.precision == WFBP_PRECISION_MIXED) {
    float *row_sc, *view_sc, *op_sc;
    mixed_scale_ptrs(ctx, rebinned, &row_sc, &view_sc, &op_sc);
    CUDA_TRY(ctx, launch_rebin_split(raw, rebinned, row_sc, view_sc, op_sc, ctx->d_chan_beta, ctx->d_chan_bidx,
                                     ctx->ext.tex_weights ? nullptr : ctx->d_chan64, p,
                                     ctx->tc_kp, ctx->nrv, ctx->taps_l1, (cudaStream_t)stream, vb, ve));
  } else {
    CUDA_TRY(ctx, launch_rebin_f32(raw, (float*)rebinned, ctx->d_chan_beta, ctx->d_chan_bidx, p, (cudaStream_t)stream,
                                   vb, ve));
  }
  return WFBP_OK;
}
}  // namespace

namespace {
// Adaptive filtration of readings [r0, r1) of `raw` into the context's
// filtered readings (context memory, allocated at creation).
int adaptive_filter(wfbp_ctx* ctx, const float* raw, long r0, long r1, void* stream) {
  CUDA_TRY(ctx, launch_adaptive_filter(raw, ctx->s_af, ctx->raw_rows, ctx->raw_ch, ctx->af_s, r0, r1,
                                       (cudaStream_t)stream));
  return WFBP_OK;
}
}  // namespace

WFBP_API int wfbp_rebin(wfbp_ctx* ctx, const float* raw, void* rebinned, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!raw || !rebinned) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_rebin: null buffer");
  DeviceGuard g(ctx->device);
  if (ctx->af_s > 0.0f) {
    const int st = adaptive_filter(ctx, raw, 0, ctx->n_readings, stream);
    if (st) return st;
    raw = ctx->s_af;
  }
  return do_rebin(ctx, raw, rebinned, 0, ctx->V, stream);
}

namespace {

// publish: write the FP16 pairs' scale into scales[vb..ve) (the stage API's
// contract); the context's own runs skip it, their backprojection applies
// the context's scale directly.
int do_filter(wfbp_ctx* ctx, const void* rebinned, void* filtered, float* scales, int layout, void* stream, int vb = 0,
              int ve = -1, bool publish = true) {
  const cudaStream_t s = (cudaStream_t)stream;
  if (ve < 0) ve = ctx->V;
  const bool bpl = layout == WFBP_LAYOUT_BACKPROJECTION;
  if (bpl && !ctx->bp_tma_ok)
    return fail(ctx, WFBP_ERR_UNSUPPORTED, "wfbp_filter: no backprojection-layout launch fits this geometry");
  if (ctx->ext.precision == WFBP_PRECISION_MIXED) {
    if (!scales) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_filter: mixed precision needs scales");
    float *row_sc, *view_sc, *op_sc;  // view_sc: the rebin's largest row scale per view (not read here)
    mixed_scale_ptrs(ctx, rebinned, &row_sc, &view_sc, &op_sc);
    (void)view_sc;
    TcOutArgs o;
    memset(&o, 0, sizeof(o));
    o.nr = ctx->nr;
    o.nrv = ctx->nrv;
    o.nrp = ctx->bpt.nrp;
    o.row_scale_in = row_sc;
    o.op_scale = op_sc;
    o.tap_scale = ctx->tap_scale;
    if (bpl) {
      o.mode = TC_OUT_PAIRS;
      o.pairs = static_cast<uint32_t*>(filtered);
      o.pair_scale = ctx->pair_scale;
      if (publish) CUDA_TRY(ctx, launch_fill(scales + vb, ctx->pair_scale, (size_t)(ve - vb), s));
    } else {
      o.mode = TC_OUT_F16_ROWS;
      o.y16 = static_cast<__half*>(filtered);
      o.row_scale_out = scales;
    }
    CUDA_TRY(ctx, launch_filter_tc(rebinned, ctx->d_bplanes, ctx->V * ctx->nrv, ctx->nch, ctx->tc_kp, ctx->tc_np,
                                   ctx->tc_bn, o, ctx->d_err, s, vb * ctx->nrv, ve * ctx->nrv));
    return WFBP_OK;
  }
  const float* x = (const float*)rebinned + (size_t)vb * ctx->nr * ctx->nch;
  const long rows = (long)(ve - vb) * ctx->nr;
  if (bpl)
    CUDA_TRY(ctx, launch_filter_f32_tr(x, (float*)filtered + (size_t)vb * ctx->nch * ctx->bpt.nrp, ctx->d_taps, rows,
                                       ctx->nch, ctx->nr, ctx->bpt.nrp, s));
  else
    CUDA_TRY(ctx, launch_filter_f32(x, (float*)filtered + (size_t)vb * ctx->nr * ctx->nch, ctx->d_taps, rows, ctx->nch,
                                    s));
  return WFBP_OK;
}

int do_backproject(wfbp_ctx* ctx, const void* filtered, const float* scales, float* vol,
                   unsigned long long* update_count, int layout, void* stream, const ThickFuse* tf = nullptr) {
  const cudaStream_t s = (cudaStream_t)stream;
  BPParams p = bp_params(ctx);
  const bool mixed = ctx->ext.precision == WFBP_PRECISION_MIXED;
  if (mixed && !scales) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_backproject: mixed precision needs scales");
  if (layout == WFBP_LAYOUT_BACKPROJECTION) {
    if (!ctx->bp_tma_ok)
      return fail(ctx, WFBP_ERR_UNSUPPORTED, "wfbp_backproject: no backprojection-layout launch fits this geometry");
    CUDA_TRY(ctx, launch_backproject_tma(filtered, mixed ? 1 : 0, ctx->pair_scale, vol, ctx->d_view_sc, ctx->d_view_z,
                                         ctx->d_z_native, p, ctx->bpt, update_count, ctx->d_err, s, tf));
    return WFBP_OK;
  }
  if (mixed)
    CUDA_TRY(ctx, launch_backproject_f16((const __half*)filtered, scales, vol, ctx->d_view_sc, ctx->d_view_z,
                                         ctx->d_z_native, p, update_count, s));
  else
    CUDA_TRY(ctx, launch_backproject_f32((const float*)filtered, vol, ctx->d_view_sc, ctx->d_view_z, ctx->d_z_native,
                                         p, update_count, s));
  return WFBP_OK;
}

}  // namespace

WFBP_API int wfbp_filter(wfbp_ctx* ctx, const void* rebinned, void* filtered, float* row_scales, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!rebinned || !filtered) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_filter: null buffer");
  DeviceGuard g(ctx->device);
  return do_filter(ctx, rebinned, filtered, row_scales, ctx->ext.filtered_layout, stream);
}

WFBP_API int wfbp_backproject(wfbp_ctx* ctx, const void* filtered, const float* row_scales, float* vol,
                              unsigned long long* update_count, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!filtered || !vol) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_backproject: null buffer");
  if (!ctx->views_set) return fail(ctx, WFBP_ERR_STATE, "wfbp_backproject: wfbp_set_views not called");
  DeviceGuard g(ctx->device);
  return do_backproject(ctx, filtered, row_scales, vol, update_count, ctx->ext.filtered_layout, stream);
}

WFBP_API int wfbp_thicken(wfbp_ctx* ctx, const float* vn, float* vol, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!vn || !vol) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_thicken: null buffer");
  DeviceGuard g(ctx->device);
  CUDA_TRY(ctx, launch_thicken(vn, vol, ctx->d_thick_off, ctx->d_thick_idx, ctx->d_thick_w, ctx->d_thick_ws,
                               ctx->nx * ctx->ny, ctx->nzr, (cudaStream_t)stream));
  return WFBP_OK;
}

// ---------------------------------------------------------------------------
// adjoints (FP32 form)
// ---------------------------------------------------------------------------

namespace {
constexpr size_t kAdjointTableBytes = size_t(6) << 30;  // backprojection adjoint scale table limit

int require_fp32_views(wfbp_ctx* ctx, const char* what) {
  if (!ctx->views_set) return fail(ctx, WFBP_ERR_STATE, std::string(what) + ": wfbp_set_views not called");
  if (ctx->ext.precision != WFBP_PRECISION_FP32)
    return fail(ctx, WFBP_ERR_UNSUPPORTED, std::string(what) + ": the adjoints are those of the FP32 form");
  return WFBP_OK;
}
}  // namespace

WFBP_API int wfbp_set_taps(wfbp_ctx* ctx, const float* taps, int n, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!taps || n < 1 || n > ctx->nch)
    return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_set_taps: need 1 <= n <= channels taps");
  if (ctx->ext.precision != WFBP_PRECISION_FP32)
    return fail(ctx, WFBP_ERR_UNSUPPORTED, "wfbp_set_taps: the mixed form bakes its taps into the operand planes");
  DeviceGuard g(ctx->device);
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_taps, taps, sizeof(float) * n, cudaMemcpyDefault, (cudaStream_t)stream));
  return WFBP_OK;
}

WFBP_API int wfbp_get_taps(wfbp_ctx* ctx, float* taps, void* stream) {
  if (!ctx || !taps) return WFBP_ERR_INVALID_ARG;
  DeviceGuard g(ctx->device);
  CUDA_TRY(ctx, cudaMemcpyAsync(taps, ctx->d_taps, sizeof(float) * ctx->nch, cudaMemcpyDefault, (cudaStream_t)stream));
  return WFBP_OK;
}

WFBP_API int wfbp_thicken_adjoint(wfbp_ctx* ctx, const float* g_volume, float* g_native, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!g_volume || !g_native) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_thicken_adjoint: null buffer");
  DeviceGuard g(ctx->device);
  CUDA_TRY(ctx, launch_thicken_adjoint(g_volume, g_native, ctx->d_thickT_off, ctx->d_thickT_idx, ctx->d_thickT_w,
                                       ctx->nx * ctx->ny, ctx->nz, (cudaStream_t)stream));
  return WFBP_OK;
}

WFBP_API int wfbp_backproject_adjoint(wfbp_ctx* ctx, const float* g_native, float* g_filtered, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!g_native || !g_filtered) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_backproject_adjoint: null buffer");
  int st = require_fp32_views(ctx, "wfbp_backproject_adjoint");
  if (st) return st;
  DeviceGuard g(ctx->device);
  const BPParams p = bp_params(ctx);
  const float z0 = ctx->z_native[0];
  // the gather finds a voxel's slice range from the spacing when the native
  // slices are evenly spaced (to a thousandth of a slice); otherwise (0) it
  // tests every slice
  float dzs = ctx->nz > 1 ? (ctx->z_native[ctx->nz - 1] - ctx->z_native[0]) / (float)(ctx->nz - 1) : 0.0f;
  for (int i = 0; i < ctx->nz && dzs != 0.0f; i++)
    if (fabsf(ctx->z_native[i] - (z0 + (float)i * dzs)) > 1e-3f * fabsf(dzs)) dzs = 0.0f;
  // the per-(voxel, theta~) scale table when it is small enough (a few GB);
  // otherwise the gather recomputes the weight sums
  const size_t n = (size_t)ctx->P2 * bp_adjoint_nzp(ctx->nz) * ctx->nx * ctx->ny;
  const bool want_table = ctx->ext.adjoint_scale_table == 0 && n * sizeof(float) <= kAdjointTableBytes;
  if (want_table && n > ctx->adj_scale_n) {
    free_dev(ctx->d_adj_scale);
    free_dev(ctx->d_adj_gvt);
    ctx->adj_scale_valid = false;
    const size_t ngt = (size_t)bp_adjoint_nzp(ctx->nz) * ctx->nx * ctx->ny;
    if (cudaMalloc(&ctx->d_adj_scale, n * sizeof(float)) == cudaSuccess &&
        cudaMalloc(&ctx->d_adj_gvt, ngt * sizeof(float)) == cudaSuccess) {
      ctx->adj_scale_n = n;
    } else {
      cudaGetLastError();  // too large for the free memory: recompute the sums instead
      free_dev(ctx->d_adj_scale);
      free_dev(ctx->d_adj_gvt);
      ctx->adj_scale_n = 0;
    }
  }
  float* table = want_table && ctx->d_adj_scale && ctx->d_adj_gvt && n <= ctx->adj_scale_n ? ctx->d_adj_scale
                                                                                              : nullptr;
  CUDA_TRY(ctx, launch_bp_adjoint(g_native, g_filtered, ctx->d_view_sc, ctx->d_view_z, ctx->d_z_native, p, z0, dzs,
                                  table, table && !ctx->adj_scale_valid, ctx->d_adj_gvt, (cudaStream_t)stream));
  if (table) ctx->adj_scale_valid = true;
  return WFBP_OK;
}

WFBP_API int wfbp_filter_adjoint(wfbp_ctx* ctx, const float* g_filtered, float* g_rebinned, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!g_filtered || !g_rebinned) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_filter_adjoint: null buffer");
  int st = require_fp32_views(ctx, "wfbp_filter_adjoint");
  if (st) return st;
  DeviceGuard g(ctx->device);
  // the Toeplitz operator h[|n - m|] is symmetric: its transpose is itself
  CUDA_TRY(ctx, launch_filter_f32(g_filtered, g_rebinned, ctx->d_taps, (long)ctx->V * ctx->nr, ctx->nch,
                                  (cudaStream_t)stream));
  return WFBP_OK;
}

WFBP_API int wfbp_rebin_adjoint(wfbp_ctx* ctx, const float* g_rebinned, float* g_raw, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!g_rebinned || !g_raw) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_rebin_adjoint: null buffer");
  int st = require_fp32_views(ctx, "wfbp_rebin_adjoint");
  if (st) return st;
  if (ctx->G != 1) return fail(ctx, WFBP_ERR_UNSUPPORTED, "wfbp_rebin_adjoint: flying focal spot scans");
  if (ctx->af_s > 0.0f) return fail(ctx, WFBP_ERR_UNSUPPORTED, "wfbp_rebin_adjoint: adaptive filtration");
  DeviceGuard g(ctx->device);
  constexpr int kMaxL = 8;
  if (!ctx->d_radj_cnt) {
    CUDA_TRY(ctx, cudaMalloc(&ctx->d_radj_cnt, sizeof(int) * ctx->nch));
    CUDA_TRY(ctx, cudaMalloc(&ctx->d_radj_idx, sizeof(int) * ctx->nch * kMaxL));
    CUDA_TRY(ctx, cudaMalloc(&ctx->d_radj_w, sizeof(float) * ctx->nch * kMaxL));
    CUDA_TRY(ctx, launch_rebin_adj_cols(ctx->d_chan_bidx, ctx->nch, ctx->ext.tex_weights ? 1 : 0, ctx->d_radj_cnt,
                                        ctx->d_radj_idx, ctx->d_radj_w, kMaxL, ctx->d_err, (cudaStream_t)stream));
  }
  CUDA_TRY(ctx, launch_rebin_adjoint(g_rebinned, g_raw, ctx->d_chan_beta, ctx->d_radj_cnt, ctx->d_radj_idx,
                                     ctx->d_radj_w, kMaxL, rebin_params(ctx), (cudaStream_t)stream));
  return WFBP_OK;
}

WFBP_API int wfbp_taps_gradient(wfbp_ctx* ctx, const float* raw, const float* g_filtered, float* g_taps, int n,
                                void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!raw || !g_filtered || !g_taps) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_taps_gradient: null buffer");
  if (n < 1 || n > ctx->nch) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_taps_gradient: need 1 <= n <= channels");
  int st = require_fp32_views(ctx, "wfbp_taps_gradient");
  if (st) return st;
  if (ctx->af_s > 0.0f) return fail(ctx, WFBP_ERR_UNSUPPORTED, "wfbp_taps_gradient: adaptive filtration");
  DeviceGuard g(ctx->device);
  const RebinParams p = rebin_params(ctx);
  const size_t need = (size_t)taps_grad_blocks(p) * n;
  if (need > ctx->tg_partial_n) {
    free_dev(ctx->d_tg_partial);
    CUDA_TRY(ctx, cudaMalloc(&ctx->d_tg_partial, sizeof(float) * need));
    ctx->tg_partial_n = need;
  }
  CUDA_TRY(ctx, launch_taps_gradient(raw, g_filtered, ctx->d_chan_beta, ctx->d_chan_bidx, p, n, ctx->d_tg_partial,
                                     g_taps, (cudaStream_t)stream));
  return WFBP_OK;
}

namespace {
// wfbp_run's own layout: the backprojection layout whenever a launch fits.
int run_layout(const wfbp_ctx* ctx) {
  return ctx->bp_tma_ok ? WFBP_LAYOUT_BACKPROJECTION : WFBP_LAYOUT_REFERENCE;
}

int ensure_scratch(wfbp_ctx* ctx) {
  size_t reb = 0, filt = 0, scal = 0;
  stage_bytes(ctx, run_layout(ctx), &reb, &filt, &scal);
  const size_t nat = sizeof(float) * (size_t)ctx->nz * ctx->nx * ctx->ny;
  if (!ctx->s_rebinned) CUDA_TRY(ctx, cudaMalloc(&ctx->s_rebinned, reb));
  if (!ctx->s_filtered) CUDA_TRY(ctx, cudaMalloc(&ctx->s_filtered, filt));
  if (!ctx->s_vol_native) CUDA_TRY(ctx, cudaMalloc(&ctx->s_vol_native, nat));
  if (!ctx->s_scales && scal) CUDA_TRY(ctx, cudaMalloc(&ctx->s_scales, scal));
  return WFBP_OK;
}

// Lists of the fused thickening for the current slab height: requested slices
// whose thickening CSR row lies in one slab (by slab), and the others.
int prepare_fuse(wfbp_ctx* ctx) {
  const int SL = ctx->bpt.slab;
  if (ctx->fuse_slab == SL) return WFBP_OK;
  const int nslab = (ctx->nz + SL - 1) / SL;
  std::vector<std::vector<int>> by(nslab);
  ctx->fuse_bnd_h.clear();
  for (int r = 0; r < ctx->nzr; r++) {
    const int a = ctx->thick_off[r], b = ctx->thick_off[r + 1];
    if (a < b && ctx->thick_idx[a] / SL == ctx->thick_idx[b - 1] / SL) by[ctx->thick_idx[a] / SL].push_back(r);
    else ctx->fuse_bnd_h.push_back(r);
  }
  ctx->fuse_slab_h.assign(nslab, make_int2(0, 0));
  ctx->fuse_req_h.clear();
  std::vector<int2> slab_tab(nslab, make_int2(0, 0));
  std::vector<int> tab;
  ctx->fuse_ok = true;
  for (int b = 0; b < nslab; b++) {
    ctx->fuse_slab_h[b].x = (int)ctx->fuse_req_h.size();
    ctx->fuse_req_h.insert(ctx->fuse_req_h.end(), by[b].begin(), by[b].end());
    ctx->fuse_slab_h[b].y = (int)ctx->fuse_req_h.size();
    slab_tab[b].x = (int)tab.size();
    for (int r : by[b]) {
      const int a = ctx->thick_off[r], e = ctx->thick_off[r + 1];
      float wsum = 0.0f;  // the sum k_thicken divides by, in the same order as setup_slices
      for (int t = a; t < e; t++) wsum += ctx->thick_w[t];
      int bits;
      tab.push_back(r);
      tab.push_back(e - a);
      memcpy(&bits, &wsum, 4);
      tab.push_back(bits);
      for (int t = a; t < e; t++) {
        tab.push_back(ctx->thick_idx[t] - b * SL);
        memcpy(&bits, &ctx->thick_w[t], 4);
        tab.push_back(bits);
      }
    }
    slab_tab[b].y = (int)tab.size();
    if (slab_tab[b].y - slab_tab[b].x > BT_FUSE_WORDS) ctx->fuse_ok = false;
  }
  free_dev(ctx->d_fuse_slab);
  free_dev(ctx->d_fuse_req);
  free_dev(ctx->d_fuse_bnd);
  free_dev(ctx->d_fuse_slab_tab);
  free_dev(ctx->d_fuse_tab);
  auto put = [&](auto** dst, const auto& v) -> cudaError_t {
    const size_t bytes = sizeof(v[0]) * std::max<size_t>(v.size(), 1);
    cudaError_t e = cudaMalloc(dst, bytes);
    if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(*dst, v.data(), sizeof(v[0]) * v.size(), cudaMemcpyHostToDevice);
    return e;
  };
  CUDA_TRY(ctx, put(&ctx->d_fuse_slab, ctx->fuse_slab_h));
  CUDA_TRY(ctx, put(&ctx->d_fuse_req, ctx->fuse_req_h));
  CUDA_TRY(ctx, put(&ctx->d_fuse_bnd, ctx->fuse_bnd_h));
  CUDA_TRY(ctx, put(&ctx->d_fuse_slab_tab, slab_tab));
  CUDA_TRY(ctx, put(&ctx->d_fuse_tab, tab));
  ctx->n_fuse_bnd = (int)ctx->fuse_bnd_h.size();
  ctx->fuse_slab = SL;
  return WFBP_OK;
}

ThickFuse make_fuse(const wfbp_ctx* ctx, float* out) {
  ThickFuse f;
  f.out = out;
  f.nzr = ctx->nzr;
  f.slab_req = ctx->d_fuse_slab;
  f.req = ctx->d_fuse_req;
  f.slab_tab = ctx->d_fuse_slab_tab;
  f.tab = ctx->d_fuse_tab;
  return f;
}

// The requested slices the fused write-back leaves out (they straddle slabs).
int thicken_boundary(wfbp_ctx* ctx, const float* vn, float* vol, cudaStream_t s) {
  CUDA_TRY(ctx, launch_thicken(vn, vol, ctx->d_thick_off, ctx->d_thick_idx, ctx->d_thick_w, ctx->d_thick_ws,
                               ctx->nx * ctx->ny, ctx->n_fuse_bnd, s, ctx->d_fuse_bnd));
  return WFBP_OK;
}
}  // namespace

namespace {
// The four stages on the context's scratch; `ev` (5 events or null) brackets
// them for the stage timers of the reference's GPUTimer (ReconstructionMachine
// .cu:239-293,345-361,391-426). NVTX ranges name the stages for profilers.
int run_stages(wfbp_ctx* ctx, const float* raw, float* vol, void* stream, cudaEvent_t* ev) {
  const cudaStream_t s = (cudaStream_t)stream;
  int st = ensure_scratch(ctx);
  if (st) return st;
  const int lay = run_layout(ctx);
  nvtxRangePushA("wfbp_run");
  if (ev) cudaEventRecord(ev[0], s);
  nvtxRangePushA("rebin");
  st = wfbp_rebin(ctx, raw, ctx->s_rebinned, stream);
  nvtxRangePop();
  if (ev) cudaEventRecord(ev[1], s);
  nvtxRangePushA("filter");
  if (!st) st = do_filter(ctx, ctx->s_rebinned, ctx->s_filtered, ctx->s_scales, lay, stream, 0, -1, false);
  nvtxRangePop();
  if (ev) cudaEventRecord(ev[2], s);
  // with the backprojection layout the thickening of the slices inside one
  // slab runs in the backprojection's write-back; the rest follow
  if (!st && lay == WFBP_LAYOUT_BACKPROJECTION) st = prepare_fuse(ctx);
  const bool fuse = !st && lay == WFBP_LAYOUT_BACKPROJECTION && ctx->fuse_ok;
  const ThickFuse tf = make_fuse(ctx, vol);
  nvtxRangePushA("backproject");
  if (!st)
    st = do_backproject(ctx, ctx->s_filtered, ctx->s_scales, ctx->s_vol_native, nullptr, lay, stream,
                        fuse ? &tf : nullptr);
  nvtxRangePop();
  if (ev) cudaEventRecord(ev[3], s);
  nvtxRangePushA("thicken");
  if (!st) st = fuse ? thicken_boundary(ctx, ctx->s_vol_native, vol, s) : wfbp_thicken(ctx, ctx->s_vol_native, vol, stream);
  nvtxRangePop();
  if (ev) cudaEventRecord(ev[4], s);
  nvtxRangePop();
  return st;
}
}  // namespace

WFBP_API int wfbp_run(wfbp_ctx* ctx, const float* raw, float* vol, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!raw || !vol) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_run: null buffer");
  if (!ctx->views_set) return fail(ctx, WFBP_ERR_STATE, "wfbp_run: wfbp_set_views not called");
  DeviceGuard g(ctx->device);
  return run_stages(ctx, raw, vol, stream, nullptr);
}

WFBP_API int wfbp_run_timed(wfbp_ctx* ctx, const float* raw, float* vol, void* stream, float* stage_ms) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!raw || !vol || !stage_ms) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_run_timed: null pointer");
  if (!ctx->views_set) return fail(ctx, WFBP_ERR_STATE, "wfbp_run_timed: wfbp_set_views not called");
  DeviceGuard g(ctx->device);
  cudaEvent_t ev[5] = {};
  for (auto& e : ev) CUDA_TRY(ctx, cudaEventCreate(&e));
  int st = run_stages(ctx, raw, vol, stream, ev);
  cudaError_t ce = cudaEventSynchronize(ev[4]);
  for (int i = 0; i < 4 && !st && !ce; i++) ce = cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
  for (auto& e : ev) cudaEventDestroy(e);
  if (st) return st;
  CUDA_TRY(ctx, ce);
  return WFBP_OK;
}

namespace {
// Views the rebin reads either side of a view (fan half-angle over the angular
// step, in views, plus the interpolation).
int rebin_reach_views(const wfbp_ctx* ctx) {
  const CTGeometry& cg = ctx->cg_read;
  const double sdd = cg.distance_source_to_detector, dcol = cg.detector_pixel_size_col, c0 = cg.detector_central_col;
  double beta = 0.0;
  for (double c : {0.0, (double)cg.num_detector_cols - 1.0})
    beta = std::max(beta, fabs(asin(std::max(-1.0, std::min(1.0, (c - c0) * dcol / sdd)))));
  const int reach_readings = (int)ceil(beta * cg.projections_per_rotation / (2 * M_PI)) + 2;
  return reach_readings / ctx->G + 2;
}

// wfbp_run_host as a pipeline over chunks of readings: the host-to-device
// copy of chunk c+1 (own stream) overlaps the rebin and filter of chunk c and
// the backprojection of every slab whose views are all filtered (the slab's
// table-position reach, the z cull of cuda_kernels.cuh:232). The
// backprojection thickens the requested slices inside its slabs as it writes
// them, and with a pinned destination those are copied back while later
// slabs run; the slices that straddle slabs are thickened and copied last.
// Same kernels, same per-voxel sums: the volume equals wfbp_run's.
int run_host_pipelined(wfbp_ctx* ctx, const float* raw_host, float* vol_host, cudaStream_t s) {
  int st = ensure_scratch(ctx);
  if (st) return st;
  const int lay = WFBP_LAYOUT_BACKPROJECTION;
  // chunks of about 64 MB of readings (8 to 64): the first backprojection
  // waits for the copies of the views its slabs reach, so smaller chunks
  // start it sooner (rows64, 2.24 GB: 8 chunks 261.5 ms, 35 chunks 256 ms)
  const size_t raw_bytes = sizeof(float) * (size_t)ctx->n_readings * ctx->raw_rows * ctx->raw_ch;
  const int kChunks = (int)std::max<size_t>(8, std::min<size_t>(64, (raw_bytes + (64u << 20) - 1) / (64u << 20)));
  if (!ctx->s_copy) CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->s_copy, cudaStreamNonBlocking));
  if (!ctx->s_back) CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->s_back, cudaStreamNonBlocking));
  for (auto& b : ctx->s_bp)
    if (!b) CUDA_TRY(ctx, cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
  if (ctx->ev_copy.size() != (size_t)kChunks + 4) {
    for (auto& e : ctx->ev_copy) cudaEventDestroy(e);
    // chunk copies, caller order, a launch's slices final, views filtered, streams joined
    ctx->ev_copy.resize(kChunks + 4);
    for (auto& e : ctx->ev_copy) CUDA_TRY(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const int V = ctx->V, G = ctx->G;
  const int cv = (V + kChunks - 1) / kChunks;
  const size_t frame = (size_t)ctx->raw_rows * ctx->raw_ch;
  const int reach = rebin_reach_views(ctx);
  // order the copies after the caller's earlier work on its stream
  CUDA_TRY(ctx, cudaEventRecord(ctx->ev_copy[kChunks], s));
  CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->s_copy, ctx->ev_copy[kChunks], 0));
  const int nchunk = (V + cv - 1) / cv;
  // From pinned memory every chunk copy is queued at once (the copy stream
  // then streams them back to back, ahead of the early copies of finished
  // slices). From pageable memory a copy holds the host until it is staged,
  // so each is issued just before the first work that needs it and the work
  // queued before it keeps the GPU busy meanwhile.
  int copies_issued = 0;
  auto issue_copies = [&](int upto) -> int {
    for (; copies_issued <= upto; copies_issued++) {
      const int c = copies_issued;
      const size_t r0 = (size_t)c * cv * G, r1 = (size_t)std::min(V, (c + 1) * cv) * G;
      CUDA_TRY(ctx, cudaMemcpyAsync(ctx->s_raw + r0 * frame, raw_host + r0 * frame,
                                    sizeof(float) * (r1 - r0) * frame, cudaMemcpyHostToDevice, ctx->s_copy));
      CUDA_TRY(ctx, cudaEventRecord(ctx->ev_copy[c], ctx->s_copy));
    }
    return WFBP_OK;
  };
  {
    cudaPointerAttributes ra;
    const bool raw_pinned = cudaPointerGetAttributes(&ra, raw_host) == cudaSuccess && ra.type == cudaMemoryTypeHost;
    cudaGetLastError();
    if (raw_pinned && (st = issue_copies(nchunk - 1))) return st;
  }
  // last view each slab needs: views j < K P/2 within the slab's reach in z
  const int SLB = ctx->bpt.slab;
  const int nslab = (ctx->nz + SLB - 1) / SLB;
  std::vector<int> need(nslab, -1);
  const int used = ctx->K * ctx->P2;
  for (int sl = 0; sl < nslab; sl++) {
    float zmn = 3e38f, zmx = -3e38f;
    for (int i = sl * SLB; i < std::min(ctx->nz, sl * SLB + SLB); i++) {
      zmn = std::min(zmn, ctx->z_native[i]);
      zmx = std::max(zmx, ctx->z_native[i]);
    }
    for (int j = 0; j < used; j++)
      if (!(ctx->view_table[j] < zmn - ctx->bp_reach || ctx->view_table[j] > zmx + ctx->bp_reach)) need[sl] = j;
  }
  std::vector<char> done(nslab, 0);
  const BPParams p = bp_params(ctx);
  const bool mixed = ctx->ext.precision == WFBP_PRECISION_MIXED;
  // fused thickening: the requested slices inside a slab are final when its
  // launch ends; with a pinned destination they are copied back right away
  // (on a stream of their own, behind the launch's event) while later slabs
  // run, so no later reading chunk's upload waits behind a copy-back
  if ((st = prepare_fuse(ctx))) return st;
  const bool fuse = ctx->fuse_ok;
  const ThickFuse tf = make_fuse(ctx, ctx->s_vol);
  cudaPointerAttributes pa;
  const bool pinned = fuse && cudaPointerGetAttributes(&pa, vol_host) == cudaSuccess && pa.type == cudaMemoryTypeHost;
  cudaGetLastError();
  const size_t plane = (size_t)ctx->nx * ctx->ny;
  auto copy_back = [&](const std::vector<int>& rs, cudaStream_t cs) -> int {
    // one copy per run of consecutive requested slices
    for (size_t a = 0; a < rs.size();) {
      size_t b = a + 1;
      while (b < rs.size() && rs[b] == rs[b - 1] + 1) b++;
      CUDA_TRY(ctx, cudaMemcpyAsync(vol_host + (size_t)rs[a] * plane, ctx->s_vol + (size_t)rs[a] * plane,
                                    sizeof(float) * plane * (b - a), cudaMemcpyDeviceToHost, cs));
      a = b;
    }
    return WFBP_OK;
  };
  std::vector<char> copied(ctx->nzr, 0);
  // Range launches alternate between two streams, so that one launch's last
  // partial wave of CTAs overlaps the next launch instead of idling the SMs;
  // each waits only for the views it reads (filtered on s).
  cudaEvent_t ev_done = ctx->ev_copy[kChunks + 1], ev_filt = ctx->ev_copy[kChunks + 2];
  int nlaunch = 0;
  // Once the readings are all on the device most slabs become ready at
  // once; a launch takes at most an eighth of them, so that the copy-back of
  // each launch's slices overlaps the next launches and only the last
  // launch's copy remains at the end.
  const int max_run = std::max(1, (nslab + 7) / 8);
  auto launch_ready = [&](int filtered_upto) -> int {
    for (int sl = 0; sl < nslab;) {
      if (done[sl] || need[sl] >= filtered_upto) {
        sl++;
        continue;
      }
      int e = sl;  // a run of ready slabs in one launch
      while (e < nslab && e - sl < max_run && !done[e] && need[e] < filtered_upto) e++;
      BPTile bt = ctx->bpt;
      bt.zb0 = sl;
      bt.nzb = e - sl;
      const cudaStream_t sb = ctx->s_bp[nlaunch++ % 2];
      CUDA_TRY(ctx, cudaEventRecord(ev_filt, s));
      CUDA_TRY(ctx, cudaStreamWaitEvent(sb, ev_filt, 0));
      CUDA_TRY(ctx, launch_backproject_tma(ctx->s_filtered, mixed ? 1 : 0, ctx->pair_scale, ctx->s_vol_native,
                                           ctx->d_view_sc, ctx->d_view_z, ctx->d_z_native, p, bt, nullptr,
                                           ctx->d_err, sb, fuse ? &tf : nullptr));
      for (int k = sl; k < e; k++) done[k] = 1;
      if (pinned) {
        std::vector<int> rs;
        for (int k = sl; k < e; k++)
          for (int i = ctx->fuse_slab_h[k].x; i < ctx->fuse_slab_h[k].y; i++) rs.push_back(ctx->fuse_req_h[i]);
        if (!rs.empty()) {
          CUDA_TRY(ctx, cudaEventRecord(ev_done, sb));
          CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->s_back, ev_done, 0));
          const int cst = copy_back(rs, ctx->s_back);
          if (cst) return cst;
          for (int r : rs) copied[r] = 1;
        }
      }
      sl = e;
    }
    return WFBP_OK;
  };
  long af_upto = 0;  // readings adaptively filtered so far
  for (int c = 0; c < nchunk; c++) {
    const int vb = c * cv, ve = std::min(V, (c + 1) * cv);
    const int last = std::min(nchunk - 1, (std::min(V, ve + reach) - 1) / cv);
    if ((st = issue_copies(last))) return st;
    CUDA_TRY(ctx, cudaStreamWaitEvent(s, ctx->ev_copy[last], 0));
    const float* rin = ctx->s_raw;
    if (ctx->af_s > 0.0f) {  // the readings copied so far, once each
      const long upto = std::min<long>(ctx->n_readings, (long)std::min(V, (last + 1) * cv) * G);
      if ((st = adaptive_filter(ctx, ctx->s_raw, af_upto, upto, s))) return st;
      af_upto = std::max(af_upto, upto);
      rin = ctx->s_af;
    }
    if ((st = do_rebin(ctx, rin, ctx->s_rebinned, vb, ve, s))) return st;
    if ((st = do_filter(ctx, ctx->s_rebinned, ctx->s_filtered, ctx->s_scales, lay, s, vb, ve, false))) return st;
    if ((st = launch_ready(ve))) return st;
  }
  if ((st = launch_ready(V + 1))) return st;
  for (auto& b : ctx->s_bp) {  // every backprojection launch before the rest of the thickening
    CUDA_TRY(ctx, cudaEventRecord(ctx->ev_copy[kChunks + 3], b));
    CUDA_TRY(ctx, cudaStreamWaitEvent(s, ctx->ev_copy[kChunks + 3], 0));
  }
  if ((st = fuse ? thicken_boundary(ctx, ctx->s_vol_native, ctx->s_vol, s)
                 : wfbp_thicken(ctx, ctx->s_vol_native, ctx->s_vol, s)))
    return st;
  std::vector<int> rest;
  for (int r = 0; r < ctx->nzr; r++)
    if (!copied[r]) rest.push_back(r);
  if ((st = copy_back(rest, s))) return st;
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->s_copy));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->s_back));
  CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return wfbp_check_device_status(ctx);
}
}  // namespace

WFBP_API int wfbp_run_host(wfbp_ctx* ctx, const float* raw_host, float* vol_host, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!raw_host || !vol_host) return fail(ctx, WFBP_ERR_INVALID_ARG, "wfbp_run_host: null buffer");
  if (!ctx->views_set) return fail(ctx, WFBP_ERR_STATE, "wfbp_run_host: wfbp_set_views not called");
  DeviceGuard g(ctx->device);
  wfbp_dims d;
  wfbp_query(ctx, &d);
  if (!ctx->s_raw) CUDA_TRY(ctx, cudaMalloc(&ctx->s_raw, d.raw_bytes));
  if (!ctx->s_vol) CUDA_TRY(ctx, cudaMalloc(&ctx->s_vol, d.volume_bytes));
  cudaStream_t s = (cudaStream_t)stream;
  if (run_layout(ctx) == WFBP_LAYOUT_BACKPROJECTION) return run_host_pipelined(ctx, raw_host, vol_host, s);
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->s_raw, raw_host, d.raw_bytes, cudaMemcpyHostToDevice, s));
  int st = wfbp_run(ctx, ctx->s_raw, ctx->s_vol, stream);
  if (st) return st;
  CUDA_TRY(ctx, cudaMemcpyAsync(vol_host, ctx->s_vol, d.volume_bytes, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return wfbp_check_device_status(ctx);
}

// ---------------------------------------------------------------------------
// synthetic scans
// ---------------------------------------------------------------------------

WFBP_API int wfbp_synth_project(const wfbp_synth_scan* scan, const wfbp_ellipsoid* ellipsoids, int n, float* out,
                                void* stream) {
  if (!scan || !out || n < 0 || (n > 0 && !ellipsoids) || scan->n_readings < 1 || scan->rows < 1 ||
      scan->channels < 1)
    return WFBP_ERR_INVALID_ARG;
  cudaError_t e = launch_synth(*scan, ellipsoids, n, out, (cudaStream_t)stream);
  if (e != cudaSuccess) return e == cudaErrorInvalidValue ? WFBP_ERR_INVALID_ARG : WFBP_ERR_CUDA;
  return WFBP_OK;
}

// ---------------------------------------------------------------------------
// internal entry points for the other host translation units
// ---------------------------------------------------------------------------

namespace wfbp_detail {
int set_error(wfbp_ctx* ctx, int code, const std::string& msg) { return fail(ctx, code, msg); }
BPParams backprojection_params(const wfbp_ctx* ctx) { return bp_params(ctx); }
void buffer_bytes(const wfbp_ctx* ctx, int layout, size_t* reb, size_t* filt, size_t* scal) {
  stage_bytes(ctx, layout, reb, filt, scal);
}
bool size_backprojection(const wfbp_ctx* ctx, int tx, int ty, int cu, int nw, int slab, BPTile* out) {
  return size_bp_tile(ctx, tx, ty, cu, nw, slab, out);
}
int filter_stage(wfbp_ctx* ctx, const void* rebinned, void* filtered, float* scales, int layout, void* stream) {
  return do_filter(ctx, rebinned, filtered, scales, layout, stream, 0, -1, false);
}
int backproject_stage(wfbp_ctx* ctx, const void* filtered, const float* scales, float* vol, int layout,
                      void* stream) {
  return do_backproject(ctx, filtered, scales, vol, nullptr, layout, stream);
}
int run_layout_of(const wfbp_ctx* ctx) { return run_layout(ctx); }
int n_bp_candidates() { return (int)(sizeof(kBpCandidates) / sizeof(kBpCandidates[0])); }
void bp_candidate(int i, int* tx, int* ty, int* cu, int* nw, int* slab) {
  *tx = kBpCandidates[i][0];
  *ty = kBpCandidates[i][1];
  *cu = kBpCandidates[i][2];
  *nw = kBpCandidates[i][3];
  *slab = kBpCandidates[i][4];
}
}  // namespace wfbp_detail
