// Internal declarations of the B200 WFBP library (not part of the ABI).
#pragma once

#include <cuda.h>
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
  const double2* sc64;       // [V] FP64 (sin, cos) of the tube angle (the mixed form's geometry)
  const double* z64;         // [V] FP64 table position
};

// Launch configuration of the TMA-staged backprojection (k_bp_tma.cu),
// sized on the host per geometry.
struct BPTile {
  int tx, ty;        // column tile (tx * ty = 16 consumer warps * columns per warp)
  int W;             // channels staged per view (TMA box)
  int nrp;           // rows per channel in the backprojection layout (multiple of 4)
  int nv_max;        // view slots per stage
  int slot_bytes;    // bytes per view slot (multiple of 128)
  float reach;       // slab-level half width of the table-position prefilter (mm)
  int smem_bytes;    // dynamic shared memory of the launch
  int cu;            // columns accumulated per step of the view loop (4 or 8)
  int nw;            // consumer warps per CTA (16, 20 or 24; one more warp produces)
  int slab;          // native slices per slab (32, or 16 with two column groups per warp)
  int zb0, nzb;      // slabs [zb0, zb0 + nzb) of this launch (nzb 0: all)
  int zc;            // 1: geometry records carry the table-position cull's row range (it can bind)
};

// Bits of the device-side error word besides WFBP_ERR_TIMEOUT (which a
// bounded wait that gave up stores whole): conditions the host's sizing rules
// out, and values outside the range of the mixed form's FP16 row pairs.
constexpr int WFBP_ERRBIT_BP_SLOTS = 0x100;   // backprojection: more views in a stage than slots
constexpr int WFBP_ERRBIT_BP_WINDOW = 0x200;  // backprojection: channel window too narrow
constexpr int WFBP_ERRBIT_ADJ_LIST = 0x400;   // rebin adjoint: per-channel source list full
constexpr int WFBP_ERRBIT_F16_RANGE = 0x800;  // filter: |filtered row / pair_scale| > 16384

// Byte offsets of the TMA backprojection's shared-memory regions; the same
// function sizes the launch on the host and carves the buffer on the device.
constexpr int BT_CWARPS = 16;  // default consumer warps of the TMA backprojection
constexpr int BT_STAGES = 2;   // view-window ring depth
constexpr int BT_FUSE_WORDS = 384;  // shared-memory words for one slab's fused-thickening records
constexpr int BP_GEO_BYTES_ZCULL = 48;  // column-pair record with the row range of the table-position cull
constexpr int BP_GEO_BYTES = 32;        // column-pair record when that cull never binds
struct BpSmem {
  unsigned slots, vinfo, vgeo, geo, fuse, total;
};
// Per staged view, the geometry the consumers' record pass reads (copied by
// the producer lane that selects the view): sin and cos of the tube angle and
// the table position, FP64 (mixed form) or FP32 (the first three floats).
struct __align__(16) BpViewGeo {
  double s, c, z, pad;
};
// Bytes 0..127 hold the ring's mbarriers and a few words (fixed across the
// tiles of a persistent launch); the per-scan regions follow.
__host__ __device__ inline BpSmem bp_smem_layout(const BPTile& bt, int cpw) {
  BpSmem L;
  unsigned o = 128;
  L.slots = o;  // [STAGES][nv_max][slot_bytes], 128-byte aligned TMA destinations
  o += (unsigned)(BT_STAGES * bt.nv_max * bt.slot_bytes);
  L.vinfo = o;
  o += (unsigned)(BT_STAGES * bt.nv_max * 8);
  o = (o + 15u) & ~15u;
  L.vgeo = o;
  o += (unsigned)(BT_STAGES * bt.nv_max * sizeof(BpViewGeo));
  L.geo = o;
  o += (unsigned)(bt.nw * bt.nv_max * (cpw / 2) * (bt.zc ? BP_GEO_BYTES_ZCULL : BP_GEO_BYTES));  // column-pair records
  L.fuse = o;
  o += (unsigned)(BT_FUSE_WORDS * 4);  // the slab's fused-thickening records (ThickFuse)
  L.total = o;
  return L;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn wfbp_encode_tiled_fn();

struct RebinParams {
  int V, nr, nch;            // output views, rows, channels (effective ones with FFS)
  float dth;                 // 2*3.14159265f / readings per rotation (cuda_kernels.cuh:15)
  int q8;                    // 8-bit fractional weights
  int G;                     // readings per view: 1, or 2 / 4 with a flying focal spot
  int phi, zf;               // FFS in channel / row direction
  int nch_raw, nr_raw;       // raw frame shape
  int voff;                  // index of the first view within the whole scan (wfbp_set_reading_offset / G)
};

// Chunk shape of the view-chunk rebin (k_rebin_vchunk): channels per CTA and
// consecutive views per thread.
constexpr int RV_CW = 128, RV_NY = 4;

struct wfbp_ctx {
  CTGeometry cg;                    // geometry of the views the stages work on (effective one with FFS)
  CTGeometry cg_read;               // geometry of the raw readings (== cg without FFS)
  int G = 1;                        // readings per view
  ReconConfig rp;
  GPUPrecompute gp;
  wfbp_ext ext;
  int device = 0;

  int V = 0, nr = 0, nch = 0, P = 0, P2 = 0, K = 0, nx = 0, ny = 0, nz = 0, nzr = 0;
  int n_readings = 0, raw_rows = 0, raw_ch = 0;
  int reading_offset = 0;           // first reading's index within the whole scan
  std::vector<float> z_native, z_req;
  std::vector<float> view_table;    // table position of each view (host copy)
  std::vector<float> taps;          // symmetric half taps h[0..nch-1]
  std::vector<int> thick_off;       // CSR over requested slices
  std::vector<int> thick_idx;
  std::vector<float> thick_w;

  // device tables
  float* d_taps = nullptr;          // [nch]
  float* d_chan_beta = nullptr;     // [nch]
  float* d_chan_bidx = nullptr;     // [nch], NaN where the rebin writes 0
  float2* d_view_sc = nullptr;      // [V] (sinf, cosf) of the tube angle
  double2* d_view_sc64 = nullptr;   // [V] FP64 (sin, cos) of the tube angle
  double* d_view_z64 = nullptr;     // [V] FP64 table position
  double2* d_chan64 = nullptr;      // [nch] mixed form: FP64 (source channel index or NaN, beta / dtheta)
  float* d_view_z = nullptr;        // [V] table position
  float* d_z_native = nullptr;      // [nz]
  int* d_thick_off = nullptr;
  int* d_thick_idx = nullptr;
  float* d_thick_w = nullptr;
  float* d_thick_ws = nullptr;      // [nzr] sum of weights
  // fused thickening lists for slabs of fuse_slab native slices (0: not built)
  int fuse_slab = 0;
  int2* d_fuse_slab = nullptr;      // [slabs] range into d_fuse_req
  int* d_fuse_req = nullptr;        // interior requested slices by slab
  int* d_fuse_bnd = nullptr;        // boundary requested slices
  int2* d_fuse_slab_tab = nullptr;  // [slabs] range into d_fuse_tab
  int* d_fuse_tab = nullptr;        // records (ThickFuse)
  int n_fuse_bnd = 0;
  bool fuse_ok = false;             // every slab's records fit in BT_FUSE_WORDS
  std::vector<int2> fuse_slab_h;    // host copies
  std::vector<int> fuse_req_h, fuse_bnd_h;
  int* d_thickT_off = nullptr;      // transposed CSR over native slices: (requested slice, w / sum w)
  int* d_thickT_idx = nullptr;
  float* d_thickT_w = nullptr;

  // adjoints
  int* d_radj_cnt = nullptr;        // rebin adjoint: per sheet column, the channels reaching it
  int* d_radj_idx = nullptr;
  float* d_radj_w = nullptr;
  float* d_tg_partial = nullptr;    // per-CTA partial tap gradients
  size_t tg_partial_n = 0;
  float* d_adj_scale = nullptr;     // backprojection adjoint: per-(voxel, theta~) weight dtheta / sum_k W_k
  size_t adj_scale_n = 0;
  float* d_adj_gvt = nullptr;       // backprojection adjoint: gradient as [ny][nx][nzp]
  bool adj_scale_valid = false;     // the table matches the current views and slices

  // mixed precision: Toeplitz operand planes for the tensor-core filter
  int tc_kp = 0, tc_np = 0, tc_bn = 0;
  int nrv = 0;                      // rows per view in the operand planes (power of two >= nr)
  float taps_l1 = 0.0f;             // sum over |d| < nch of |h[d]|
  float tap_scale = 1.0f;           // power of two applied to the taps in d_bplanes
  float pair_scale = 1.0f;          // power of two >= taps_l1 dividing the FP16 row pairs (backprojection layout)
  void* d_bplanes = nullptr;        // FP16 [2][tc_np][tc_kp] (hi, lo of tap_scale * T)
  int* d_err = nullptr;             // device-side error word (WFBP_ERR_TIMEOUT, or WFBP_ERRBIT_* bits)

  // TMA-staged backprojection (backprojection layout [V][nch][nrp])
  bool bp_tma_ok = false;
  BPTile bpt;
  float bp_reach = 0.0f;            // slab-level view prefilter half width (mm)
  int bp_nv_max = 1;                // most views of one theta~ reaching a slab
  int bp_zcull = 1;                 // 0: the table-position cull (|z - z_j| > z_rot) never removes a
                                    // sample whose row lies in [0, nr - 2] (cone shorter than z_rot)

  // context-owned scratch for wfbp_run / wfbp_run_host
  void* s_rebinned = nullptr;
  void* s_filtered = nullptr;
  float* s_scales = nullptr;
  float* s_vol_native = nullptr;
  float* s_raw = nullptr;
  float* s_vol = nullptr;
  cudaStream_t s_copy = nullptr;    // wfbp_run_host: host-to-device copies of the reading chunks
  cudaStream_t s_back = nullptr;    // wfbp_run_host: device-to-host copies of finished slices
  float af_s = 0.0f;                // adaptive filtration strength (ReconConfig.adaptive_filtration_s, <= 1; 0: off)
  float* s_af = nullptr;            // adaptively filtered readings [n_readings][raw_rows][raw_ch] (af_s > 0)
  cudaStream_t s_bp[2] = {nullptr, nullptr};  // wfbp_run_host: backprojection launches (alternating)
  std::vector<cudaEvent_t> ev_copy; // one per chunk, plus the caller-stream fence

  bool views_set = false;
  std::string err;
};

// kernels (launchers return cudaError_t of the launch)
cudaError_t launch_view_tables(const float* d_tube, const float* d_table, float2* d_sc, float* d_z, int V,
                               cudaStream_t s);
cudaError_t launch_rebin_tables(float* d_beta, float* d_bidx, int nch, float c0, float dcol, float sdd,
                                cudaStream_t s);
// Stage launchers take an optional range: views [vb, ve) for the rebins,
// rows [mb, me) for the tensor-core filter (-1: all).
cudaError_t launch_rebin_f32(const float* raw, float* out, const float* d_beta, const float* d_bidx,
                             const RebinParams& p, cudaStream_t s, int vb = 0, int ve = -1);
cudaError_t launch_filter_f32(const float* x, float* y, const float* d_taps, long rows, int nch, cudaStream_t s);
cudaError_t launch_backproject_f32(const float* D, float* vol, const float2* sc, const float* vz,
                                   const float* zs, const BPParams& p, unsigned long long* count,
                                   cudaStream_t s);
cudaError_t launch_backproject_f16(const __half* D, const float* scales, float* vol, const float2* sc,
                                   const float* vz, const float* zs, const BPParams& p, unsigned long long* count,
                                   cudaStream_t s);
cudaError_t launch_rebin_split(const float* raw, void* planes, float* row_scale, float* view_scale,
                               float* op_scale, const float* d_beta, const float* d_bidx, const double2* d_chan64,
                               const RebinParams& p, int kp, int nrv, float taps_l1, cudaStream_t s, int vb = 0,
                               int ve = -1);
// Output modes of the tensor-core filter epilogue.
enum TcOut { TC_OUT_F32 = 0, TC_OUT_F16_ROWS = 1, TC_OUT_PAIRS = 2 };
struct TcOutArgs {
  int mode;
  int nr, nrv, nrp;             // valid rows per view, rows per view in the planes, rows in the pairs layout
  float* y32;                   // TC_OUT_F32: [V*nrv][nch]
  __half* y16;                  // TC_OUT_F16_ROWS: [V][nr][nch]
  uint32_t* pairs;              // TC_OUT_PAIRS: [V][nch][nrp] half2 (row i, row i+1)
  const float* row_scale_in;    // [V*nrv]
  float* row_scale_out;         // [V][nr]
  float pair_scale;             // TC_OUT_PAIRS: power of two dividing every stored row of the scan
  const float* op_scale;        // [V] power-of-two scale of the view's FP16 operand rows
  float tap_scale;              // power-of-two scale of the FP16 Toeplitz operand
};
// dst[0..n) = value
cudaError_t launch_fill(float* dst, float value, size_t n, cudaStream_t s);
cudaError_t launch_filter_tc(const void* a_planes, const void* b_planes, int M, int nch, int kp, int np, int bn,
                             const TcOutArgs& out, int* err, cudaStream_t s, int mb = 0, int me = -1);
cudaError_t launch_filter_f32_tr(const float* x, float* yt, const float* d_taps, long rows, int nch, int nr, int nrp,
                                 cudaStream_t s);
// Thickening fused into the TMA backprojection's write-back: a requested
// slice whose native slices (the thickening CSR row) all lie in one slab is
// formed from that slab's registers and written to `out`; the other
// ("boundary") requested slices are thickened afterwards from the native
// volume. out == nullptr: no fusion.
// Records of slab b, words tab[slab_tab[b].x .. slab_tab[b].y) (at most
// BT_FUSE_WORDS), one per interior requested slice r:
//   r, n, bits(sum of weights), then n pairs (native slice - slab start, bits(w))
// in the thickening CSR's order.
struct ThickFuse {
  float* out;            // requested volume [nzr][ny][nx]
  int nzr;
  const int2* slab_req;  // per slab: [begin, end) into req
  const int* req;        // interior requested slices, grouped by slab, ascending
  const int2* slab_tab;  // per slab: [begin, end) into tab
  const int* tab;
};

// One scan of a persistent (batched) backprojection launch, in device memory.
struct alignas(64) BpScan {
  CUtensorMap map;              // filtered rows [V][nch][nrp], box {nrp, W, 1}
  BPParams p;
  BPTile bt;
  float* vol;                   // native volume
  const float2* view_sc;
  const float* view_z;
  const float* zslices;
  ThickFuse tf;                 // fused thickening (tf.out == nullptr: none)
};
cudaError_t bp_tma_encode_map(const void* D, int elem_half2, const BPParams& p, const BPTile& bt, CUtensorMap* map);
cudaError_t launch_backproject_tma_batch(int elem_half2, int cpw, int cu, int nw, int slab, int zc, const BpScan* scans,
                                         const int4* items, int n_items, unsigned* next, int* err, int smem_bytes,
                                         int grid, cudaStream_t s);
size_t bp_tma_smem_bytes(const BPTile& bt, int elem_bytes);
bool bp_tma_supported(const BPTile& bt);
cudaError_t launch_backproject_tma(const void* D, int elem_half2, float row_scale, float* vol,
                                   const float2* sc, const float* vz, const float* zs, const BPParams& p,
                                   const BPTile& bt, unsigned long long* count, int* err, cudaStream_t s,
                                   const ThickFuse* tf = nullptr);
int tc_choose_bn(int nch);
// requested slices list[0..nzr) (list == nullptr: 0..nzr-1)
cudaError_t launch_thicken(const float* vn, float* out, const int* off, const int* idx, const float* w,
                           const float* ws, int nxy, int nzr, cudaStream_t s, const int* list = nullptr);
// slice stride of the backprojection adjoint's scale table [P/2][ny][nx][nzp]
inline int bp_adjoint_nzp(int nz) { return (nz + 3) / 4 * 4; }
// scale_table: [P/2][ny][nx][nzp] weights dtheta / sum_k W_k, filled first
// when fill_table is set; nullptr: the gather recomputes the weight sums.
// gvol_t: [ny][nx][nzp] scratch for the transposed gradient (table path).
cudaError_t launch_bp_adjoint(const float* gvol, float* gD, const float2* sc, const float* vz, const float* zs,
                              const BPParams& p, float z0, float dzs, float* scale_table, bool fill_table,
                              float* gvol_t, cudaStream_t s);
cudaError_t launch_thicken_adjoint(const float* gvol, float* gvn, const int* off, const int* ridx, const float* w,
                                   int nxy, int nz, cudaStream_t s);
cudaError_t launch_rebin_adj_cols(const float* bidx, int nch, int q8, int* cnt, int* cidx, float* cw, int maxl,
                                  int* err, cudaStream_t s);
cudaError_t launch_rebin_adjoint(const float* gR, float* graw, const float* beta, const int* cnt, const int* cidx,
                                 const float* cw, int maxl, const RebinParams& p, cudaStream_t s);
int taps_grad_blocks(const RebinParams& p);
cudaError_t launch_selftest_wait(int* err, unsigned long long limit_ns, cudaStream_t s);
cudaError_t launch_taps_gradient(const float* raw, const float* gY, const float* beta, const float* bidx,
                                 const RebinParams& p, int ntaps, float* partial, float* out, cudaStream_t s);
cudaError_t launch_adaptive_filter(const float* raw, float* out, int nr, int nch, float s, long r0, long r1,
                                   cudaStream_t st);
cudaError_t launch_synth(const wfbp_synth_scan& scan, const wfbp_ellipsoid* d_e, int ne, float* out,
                         cudaStream_t s);

// Host helpers of wfbp_host.cu used by the other host translation units.
namespace wfbp_detail {
int set_error(wfbp_ctx* ctx, int code, const std::string& msg);
BPParams backprojection_params(const wfbp_ctx* ctx);
void buffer_bytes(const wfbp_ctx* ctx, int layout, size_t* reb, size_t* filt, size_t* scal);
bool size_backprojection(const wfbp_ctx* ctx, int tx, int ty, int cu, int nw, int slab, BPTile* out);
// wfbp_filter without writing the FP16 pairs' scale into `scales` (the
// context's backprojection applies the scale itself)
int filter_stage(wfbp_ctx* ctx, const void* rebinned, void* filtered, float* scales, int layout, void* stream);
int backproject_stage(wfbp_ctx* ctx, const void* filtered, const float* scales, float* vol, int layout,
                      void* stream);
int run_layout_of(const wfbp_ctx* ctx);  // the layout wfbp_run uses
int n_bp_candidates();
void bp_candidate(int i, int* tx, int* ty, int* cu, int* nw, int* slab);
}  // namespace wfbp_detail
