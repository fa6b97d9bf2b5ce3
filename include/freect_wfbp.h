/*
 * freect_wfbp.h — C ABI of the B200 (sm_100a) helical WFBP path.
 *
 * This is the drop-in boundary for FreeCT fct_wfbp's reconstruction path:
 *   rebin (fan -> parallel, optional flying focal spot merge)
 *   -> ramp filter (Toeplitz contraction along the channel axis)
 *   -> helical Q-weighted backprojection
 *   -> final slice thickening.
 *
 * The reference has no plugin or FFI layer; its boundary is the C++ class
 * fct::ReconstructionMachine (applications/fct_wfbp/include/ReconstructionMachine.h:8-50)
 * whose stage methods RebinAndFilter / Backproject / ApplyFinalSliceThicknessing
 * (ReconstructionMachine.h:25-28) exchange device buffers with fixed layouts.
 * Every entry point below replaces one of those methods (cited per function)
 * and keeps its buffer layout, but:
 *   - buffers are caller-owned device pointers (scratch is context-owned),
 *   - every call takes an explicit CUDA stream (passed as void*),
 *   - errors are returned as status codes instead of exit() (the reference's
 *     gpuErrChk/cufftErrChk call exit(), gpu_error_check.h:38-58),
 *   - no call synchronises the device unless documented,
 *   - a context's own scratch (wfbp_run's intermediates, the adjoint's weight
 *     table, the fused-thickening lists) is shared by the calls on it: call a
 *     context from one host thread at a time, and do not let wfbp_run /
 *     wfbp_run_host / the backprojection adjoint of one context overlap on
 *     the GPU (stage calls into caller buffers on different streams may).
 *
 * All structs keep the reference's field order and types, so host code that
 * fills the reference's structs can pass them unchanged.
 */
#ifndef FREECT_WFBP_H
#define FREECT_WFBP_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Reference structs (byte-identical to applications/fct_wfbp/include/       */
/* recon_structs.h:6-31, 33-50, 52-67)                                        */
/* ------------------------------------------------------------------------ */

/* recon_structs.h:6-31 */
typedef struct CTGeometry {
  size_t total_number_of_projections;
  size_t projections_per_rotation;
  float detector_pixel_size_col;     /* transverse spacing at the detector (mm) */
  float detector_pixel_size_row;     /* axial spacing at the detector (mm) */
  size_t num_detector_cols;
  size_t num_detector_cols_padded;
  size_t num_detector_cols_padded_fft;
  size_t num_detector_rows;
  size_t num_detector_rows_padded;
  float detector_central_col;
  float detector_central_row;
  float distance_source_to_detector;
  float distance_source_to_isocenter;
  float collimated_slice_width;
  float theta_cone;
  float acquisition_field_of_view;
  float z_rot;
  float anode_angle;
  bool ffs_phi;
  bool ffs_z;
  bool ffs_diag;
} CTGeometry;

/* recon_structs.h:33-50 */
typedef struct ReconConfig {
  char raw_data_dir[4096];
  char output_dir[4096];
  char output_file[255];
  float start_pos;
  float end_pos;
  float recon_fov;
  float slice_thickness;
  float slice_pitch;
  size_t nx;
  size_t ny;
  int recon_kernel;
  float x_origin;
  float y_origin;
  float tube_angle_offset;
  float adaptive_filtration_s;
} ReconConfig;

/* recon_structs.h:52-67 (the data members; InitFromCTGeometry is
 * wfbp_configure_geometry below) */
typedef struct GPUPrecompute {
  float half_acquisition_fov;
  float half_acquisition_fov_squared;
  int projections_per_half_turn;
  int n_half_turns;
  float distance_source_to_isocenter_squared;
  float z_rot_over_2_pi;
  float recip_distance_source_to_detector;
  float recip_distance_source_to_isocenter;
  float tanf_theta_cone;
  float pixel_scale;
  float two_pi_over_projections_per_rotation;
  int n_slices_native;
  int n_slices_requested;
} GPUPrecompute;

/* ------------------------------------------------------------------------ */
/* Scan metadata: the RawDataSet getters that ConfigureCTGeometry reads      */
/* (modules/fct_read/include/fct/RawDataSet.h:90-106)                        */
/* ------------------------------------------------------------------------ */
typedef struct wfbp_scan_meta {
  int total_num_projections;         /* readings in the file (after FFS: readings, not views) */
  int projections_per_rotation;      /* readings per rotation */
  int detector_channels;
  int detector_rows;
  float detector_transverse_spacing; /* mm at the detector */
  float detector_axial_spacing;      /* mm at the detector */
  float detector_central_channel;
  float detector_central_row;
  float dist_source_to_isocenter;
  float dist_source_to_detector;
  int ffs_mode;                      /* wfbp_ffs_mode */
  float anode_angle;                 /* rad, used by z-FFS */
} wfbp_scan_meta;

/* ------------------------------------------------------------------------ */
/* Status codes and options                                                 */
/* ------------------------------------------------------------------------ */
enum wfbp_status {
  WFBP_OK = 0,
  WFBP_ERR_INVALID_ARG = 1,   /* bad pointer, size, or struct field */
  WFBP_ERR_OOM = 2,           /* a context allocation failed */
  WFBP_ERR_CUDA = 3,          /* a CUDA runtime call or kernel launch failed */
  WFBP_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up */
  WFBP_ERR_UNSUPPORTED = 5,   /* option not supported for this geometry */
  WFBP_ERR_STATE = 6          /* call out of order (e.g. views not set) */
};

enum wfbp_precision {
  WFBP_PRECISION_FP32 = 0,    /* FP32 rebin, FP32 SIMT Toeplitz filter, FP32 rows, FP32 backprojection */
  WFBP_PRECISION_MIXED = 1    /* rebin with FP64 sample coordinates into split hi+lo FP16 operand
                                 planes, tcgen05 filter (FP32 accumulate in TMEM), FP16 filtered
                                 rows with power-of-two scales, backprojection with FP64 per-view
                                 geometry and FP32 accumulation */
};

enum wfbp_filter_window {
  WFBP_FILTER_REFERENCE = 0,  /* generate_filter(cg, c, a): ReconstructionMachine.cu:478-513 */
  WFBP_FILTER_SHEPP_LOGAN = 1,/* discrete Shepp-Logan kernel h[n] = -2/(pi^2 ds (4n^2-1)) */
  WFBP_FILTER_USER = 2        /* caller-provided symmetric taps h[0..n-1] */
};

/* Values of ReconConfig.recon_kernel. fct_wfbp parses the field
 * (parse_config.cpp:53) but always filters with generate_filter's ramp
 * (ReconstructionMachine.cu:204); here it selects the window whenever the
 * wfbp_ext is NULL or leaves filter_window at WFBP_FILTER_REFERENCE with
 * filter_c = filter_a = 1 (or both 0). 0 reproduces fct_wfbp; other values
 * are rejected (WFBP_ERR_INVALID_ARG). The Hann and Hamming windows are
 * generate_filter's `a` parameter (resources/ramp.m: 0.5, 0.54). */
enum wfbp_recon_kernel {
  WFBP_RECON_KERNEL_RAMLAK = 0,      /* generate_filter(c = 1, a = 1) */
  WFBP_RECON_KERNEL_SHEPP_LOGAN = 1, /* WFBP_FILTER_SHEPP_LOGAN */
  WFBP_RECON_KERNEL_HANN = 2,        /* generate_filter(c = 1, a = 0.5) */
  WFBP_RECON_KERNEL_HAMMING = 3      /* generate_filter(c = 1, a = 0.54) */
};

/* Layout of the filtered projections at the wfbp_filter / wfbp_backproject
 * boundary. REFERENCE keeps the reference's [view][row][channel] FP32 (or
 * FP16 + per-row scales); BACKPROJECTION is the channel-major layout the
 * TMA-staged backprojection reads: [view][channel][nrp] FP32, or half2 pairs
 * (row r, row r+1) of the rows divided by one power of two for the whole
 * scan (the smallest >= the taps' L1 norm sum|h|, so a stored value is at
 * most the largest rebinned sample); nrp = nr rounded up to a multiple of 4.
 * wfbp_filter writes that scale into every view's entry of row_scales [V]
 * and wfbp_backproject applies it. wfbp_run always uses BACKPROJECTION
 * internally when the geometry allows it. */
enum wfbp_layout {
  WFBP_LAYOUT_REFERENCE = 0,
  WFBP_LAYOUT_BACKPROJECTION = 1
};

enum wfbp_ffs_mode {
  WFBP_FFS_NONE = 0,
  WFBP_FFS_PHI = 1,
  WFBP_FFS_Z = 2,
  WFBP_FFS_PHIZ = 3
};

/* Extension options that the reference has no field for. */
#define WFBP_EXT_VERSION 1
typedef struct wfbp_ext {
  int version;                /* must be WFBP_EXT_VERSION */
  int precision;              /* wfbp_precision */
  int filter_window;          /* wfbp_filter_window */
  float filter_c;             /* generate_filter's c (reference default 1) */
  float filter_a;             /* generate_filter's a (reference default 1) */
  const float* user_taps;     /* WFBP_FILTER_USER: h[0..n_user_taps-1], h[-n]=h[n] */
  int n_user_taps;
  int tex_weights;            /* 1: rebin uses 8-bit fractional bilinear weights like the
                                 texture unit the reference samples through (cuda_kernels.cuh:36) */
  int bp_slab;                /* 0 = any; 16 or 32: only backprojection configurations whose
                                 slabs hold that many native slices (wfbp_bp_config.slab) */
  int filtered_layout;        /* wfbp_layout of the stage API (default REFERENCE) */
  int adjoint_scale_table;    /* 0: the backprojection adjoint keeps a per-(voxel, half-turn angle)
                                 weight table dtheta / sum_k W_k when it fits in 6 GB, computed on
                                 the first adjoint call after the views or slices change;
                                 -1: never (the adjoint recomputes the weight sums) */
  int reserved[5];
} wfbp_ext;

/* Sizes of every stage buffer a context expects (bytes unless noted). */
typedef struct wfbp_dims {
  int n_views;                /* V after FFS merge */
  int n_rows;                 /* rows after FFS merge */
  int n_channels;             /* channels after FFS merge */
  int n_readings;             /* raw readings (V * readings_per_view) */
  int raw_rows, raw_channels; /* raw frame shape */
  int nx, ny;
  int n_slices_native;
  int n_slices_requested;
  int precision;
  size_t raw_bytes;           /* float [n_readings][raw_rows][raw_channels] */
  size_t rebinned_bytes;      /* stage-1 output (FP32 [V][nr][nch], or the split FP16 operand planes) */
  size_t filtered_bytes;      /* stage-2 output (FP32 or FP16 [V][nr][nch]) */
  size_t row_scale_bytes;     /* FP32 scales: [V][nr] (MIXED, REFERENCE layout) or [V]
                                 (MIXED, BACKPROJECTION layout), else 0 */
  size_t native_volume_bytes; /* FP32 [nz_native][ny][nx] */
  size_t volume_bytes;        /* FP32 [nz_requested][ny][nx] */
} wfbp_dims;

typedef struct wfbp_ctx wfbp_ctx;

/* ------------------------------------------------------------------------ */
/* Geometry (host-only, no device needed)                                   */
/* ------------------------------------------------------------------------ */

/* ReconstructionMachine::ConfigureCTGeometry (ReconstructionMachine.cu:44-74)
 * followed by GPUPrecompute::InitFromCTGeometry (recon_structs.h:69-83).
 * table_positions: n = meta->total_num_projections floats (needs n > P). */
int wfbp_configure_geometry(const wfbp_scan_meta* meta, const float* table_positions,
                            CTGeometry* cg, GPUPrecompute* gp);

/* The geometry the stages of a context created from `cg` work on (host
 * only): `cg` itself, or with a flying focal spot the effective geometry of
 * wfbp_get_geometry (one view per focal-state cycle, 2x channels / rows at
 * half the spacing). Slice lists of a context follow this geometry. */
int wfbp_effective_geometry(const CTGeometry* cg, CTGeometry* eff);

/* Slice lists of ReconstructionMachine::AllocateKeyArrays
 * (ReconstructionMachine.cu:107-137), float accumulation included.
 * Either output pointer may be NULL to query counts. */
int wfbp_slice_locations(const CTGeometry* cg, const ReconConfig* rp,
                         float* native_z, int native_cap, int* n_native,
                         float* requested_z, int requested_cap, int* n_requested);

/* The filter window, c and a that a ReconConfig.recon_kernel value selects
 * (wfbp_recon_kernel; host only). WFBP_ERR_INVALID_ARG for other values. */
int wfbp_recon_kernel_filter(int recon_kernel, int* window, float* c, float* a);

/* Filter taps: the spatial-domain kernel of generate_filter
 * (ReconstructionMachine.cu:478-513) before its FFT, as the symmetric half
 * h[0..n-1] (h[-k] = h[k]) in FP32. */
int wfbp_filter_taps(const CTGeometry* cg, int window, float c, float a, float* taps, int n);

/* ------------------------------------------------------------------------ */
/* Context                                                                   */
/* ------------------------------------------------------------------------ */

/* Creates a context on `device` for one scan geometry and recon config.
 * Replaces the state the reference keeps in ReconstructionMachine
 * (ReconstructionMachine.h:30-48) plus its __constant__ copies
 * (cuda_kernels.cuh:5-7). `ext` may be NULL (FP32; the filter of rp->recon_kernel,
 * wfbp_recon_kernel).
 * rp->adaptive_filtration_s, which fct_wfbp parses (parse_config.cpp:57) but
 * never applies, turns on adaptive filtration of the raw readings before the
 * rebin when > 0 (values above 1 act as 1): with p_max the largest line
 * integral of a reading and p_t = (1 - s) p_max, each sample p becomes
 * p + w (pbar - p), pbar = (p[c-1] + 2 p[c] + p[c+1]) / 4 along its detector
 * row (edge channels repeated), w = clamp((p - p_t) / (p_max - p_t), 0, 1):
 * attenuation-adaptive smoothing after Kachelriess, Watzke and Kalender,
 * Med. Phys. 28 (2001) 475-490. The filtered readings live in context memory
 * (the raw frames' size, allocated here); the rebin adjoint and the tap
 * gradient refuse such a context (WFBP_ERR_UNSUPPORTED). */
int wfbp_ctx_create(const CTGeometry* cg, const ReconConfig* rp, const wfbp_ext* ext,
                    int device, wfbp_ctx** out);
int wfbp_ctx_destroy(wfbp_ctx* ctx);
int wfbp_query(const wfbp_ctx* ctx, wfbp_dims* dims);

/* Per-view tube angles and table positions, host arrays of n_readings floats
 * (ReconstructionMachine.cu:96-102). Builds the per-view tables: sinf / cosf
 * and the table position in FP32, as the reference evaluates them per voxel
 * (cuda_kernels.cuh:235-238), for the FP32 form, and sin / cos / table
 * position in FP64 for the mixed form's backprojection geometry. */
int wfbp_set_views(wfbp_ctx* ctx, const float* tube_angles, const float* table_positions);

/* The geometry the stages work on: the caller's CTGeometry, or for a flying
 * focal spot scan its effective geometry (one view per focal-state cycle,
 * 2x channels / rows at half the spacing, central channel 2 c0 + 1/2), and
 * the GPUPrecompute derived from it (recon_structs.h:69-83). No counterpart
 * in the reference, whose fct_wfbp ignores the FFS fields
 * (recon_structs.h:26-29). */
int wfbp_get_geometry(const wfbp_ctx* ctx, CTGeometry* cg, GPUPrecompute* gp);

/* Copies the native / requested slice z lists (as wfbp_slice_locations). */
int wfbp_get_slices(const wfbp_ctx* ctx, float* native_z, float* requested_z);

/* Index of the context's first reading within the whole scan (default 0),
 * for a context that holds a window of a scan's readings: the rebin samples
 * reading v at the whole scan's index angle (v + offset) 2 pi / P
 * (rebin_kernel, cuda_kernels.cuh:15-20), so the window rebins exactly like
 * the whole scan. A multiple of the readings per view. No counterpart in
 * the reference. */
int wfbp_set_reading_offset(wfbp_ctx* ctx, int offset);

/* Replaces the slice lists that wfbp_ctx_create derived from ReconConfig
 * (ReconstructionMachine.cu:107-137) with explicit ones: native z (strictly
 * monotone) and requested z. Used to reconstruct a z-slab of a scan with
 * exactly the slice positions of the whole scan's lists (sharding across
 * GPUs); the thickening weights and the backprojection launch are rebuilt.
 * No counterpart in the reference. */
int wfbp_set_slices(wfbp_ctx* ctx, const float* native_z, int n_native, const float* requested_z,
                    int n_requested);

/* Launch configuration of the backprojection in the backprojection layout
 * (no counterpart in the reference, whose backproject_kernel launch is a
 * fixed 16x16-thread block per voxel tile, ReconstructionMachine.cu:347-351).
 * A CTA covers tile_x * tile_y voxel columns and `slab` native slices (32,
 * or 16 with two column groups per warp; 0 = 32) with consumer_warps warps
 * (0 = 16) plus one TMA producer warp; cols_per_step columns are
 * accumulated per pass over a view window.
 * wfbp_set_views picks a default; an autotuner lists the configurations that
 * fit this geometry, times them and sets the fastest. All need set_views. */
typedef struct wfbp_bp_config {
  int tile_x, tile_y;
  int cols_per_step;
  int consumer_warps;
  int slab;
} wfbp_bp_config;
int wfbp_bp_configs(const wfbp_ctx* ctx, wfbp_bp_config* out, int cap, int* n);
int wfbp_get_bp_config(const wfbp_ctx* ctx, wfbp_bp_config* config);
int wfbp_set_bp_config(wfbp_ctx* ctx, const wfbp_bp_config* config);

/* Reads and clears the context's device-side error word, which kernels
 * with bounded waits set instead of hanging (synchronous). Returns
 * WFBP_ERR_TIMEOUT if a wait gave up since the last check,
 * WFBP_ERR_UNSUPPORTED if the mixed form's filter met a filtered value
 * beyond the range of its FP16 row pairs (16384 x the scan's scale, which
 * takes rebinned samples above 16384), WFBP_ERR_CUDA if a device-side sizing
 * check failed. No counterpart in the reference, which has no device-side
 * waits. */
int wfbp_check_device_status(wfbp_ctx* ctx);

/* Failure-detection self-test: launches a kernel whose mbarrier wait can
 * never complete (nothing arrives) with a wall-clock limit of limit_ms
 * (1-10000); the wait gives up, the kernel sets the context's error word
 * and returns, so the next wfbp_check_device_status reports
 * WFBP_ERR_TIMEOUT and the context stays usable. Every production wait
 * (TMA rings, tensor-core pipeline) is bounded the same way (4 s). */
int wfbp_selftest_bounded_wait(wfbp_ctx* ctx, int limit_ms, void* stream);

/* Last error message of this context (never NULL). */
const char* wfbp_last_error(const wfbp_ctx* ctx);
const char* wfbp_status_string(int status);

/* ------------------------------------------------------------------------ */
/* Stages (device pointers, asynchronous on `stream`)                       */
/* ------------------------------------------------------------------------ */

/* Stage 1 of RebinAndFilter (ReconstructionMachine.cu:141-256 and
 * rebin_kernel, cuda_kernels.cuh:11-39): host reshape/flip + rebin of every
 * row in one launch. raw: FP32 [n_readings][raw_rows][raw_channels].
 * rebinned: FP32 [V][nr][nch] (row index = flipped row sheet index), or for
 * WFBP_PRECISION_MIXED the split FP16 operand planes of the filter with
 * their scales. */
int wfbp_rebin(wfbp_ctx* ctx, const float* raw, void* rebinned, void* stream);

/* Stage 2 of RebinAndFilter (ReconstructionMachine.cu:262-290: R2C,
 * multiply_filter, C2R, reshape_rebin_into_final_array) as a Toeplitz
 * contraction. filtered: FP32 [V][nr][nch] (FP32) or FP16 [V][nr][nch]
 * plus row_scales FP32 [V][nr] (MIXED; row_scales may be NULL for FP32), in
 * the reference layout; in the backprojection layout see wfbp_layout. */
int wfbp_filter(wfbp_ctx* ctx, const void* rebinned, void* filtered, float* row_scales,
                void* stream);

/* ReconstructionMachine::Backproject (ReconstructionMachine.cu:308-385,
 * backproject_kernel cuda_kernels.cuh:198-287). volume_native: FP32
 * [nz_native][ny][nx], overwritten. update_count: optional device uint64
 * that receives the number of contributing voxel-view updates (adds to it). */
int wfbp_backproject(wfbp_ctx* ctx, const void* filtered, const float* row_scales,
                     float* volume_native, unsigned long long* update_count, void* stream);

/* ReconstructionMachine::ApplyFinalSliceThicknessing (ReconstructionMachine.cu:387-434,
 * thicken_slices cuda_kernels.cuh:289-320), without the D2H copy. */
int wfbp_thicken(wfbp_ctx* ctx, const float* volume_native, float* volume, void* stream);

/* RunReconstruction (ReconstructionMachine.cu:76-82) on device buffers:
 * raw (device) -> volume (device), with context-owned intermediates. */
int wfbp_run(wfbp_ctx* ctx, const float* raw, float* volume, void* stream);

/* wfbp_run without any device allocation. No counterpart in the reference.
 *
 * wfbp_run allocates its intermediates (rebinned rows, filtered rows, row
 * scales, native-thickness volume) with cudaMalloc on first use. Callers that
 * must not allocate -- an application whose device memory all belongs to its
 * own pool or caching allocator, a scanner pipeline held to a fixed memory
 * budget fixed at start-up, a latency-critical loop that cannot take
 * cudaMalloc's implicit synchronisation -- call this instead: the
 * intermediates live in one static device array of WFBP_STATIC_SCRATCH_BYTES
 * that every GPU which loads the library holds until the process exits.
 *   - Geometries whose intermediates exceed WFBP_STATIC_SCRATCH_BYTES are
 *     rejected with WFBP_ERR_INVALID_ARG and a message (wfbp_last_error).
 *   - The first call on a device looks up the array's device address on that
 *     device (cudaGetSymbolAddress); make that first call before any stream
 *     capture begins.
 *   - All calls on one device share the array: calls that overlap on the GPU
 *     (other streams, other contexts, other threads) race; serialise them.
 *   - Each stage overwrites its whole region, so no state carries over from
 *     the previous call.
 * The context itself is created (and allocates its tables) beforehand with
 * wfbp_ctx_create; this call allocates nothing. */
#define WFBP_STATIC_SCRATCH_BYTES (32u << 20)
int wfbp_run_static(wfbp_ctx* ctx, const float* raw, float* volume, void* stream);

/* wfbp_run, synchronous, with the device time of each stage in ms
 * (stage_ms[0..3] = rebin, filter, backprojection, thickening), the
 * reference's per-stage GPUTimer output (ReconstructionMachine.cu:239-293,
 * 345-361, 391-426). Stages are also marked as NVTX ranges. */
int wfbp_run_timed(wfbp_ctx* ctx, const float* raw, float* volume, void* stream, float* stage_ms);

/* RunReconstruction from host memory: H2D of the raw readings, the four
 * stages, D2H of the final volume (ReconstructionMachine.cu:246,423),
 * synchronous on return. Pinned host buffers overlap the copies with the
 * stages. */
int wfbp_run_host(wfbp_ctx* ctx, const float* raw_host, float* volume_host, void* stream);

/* ------------------------------------------------------------------------ */
/* Batched scans (no counterpart in the reference, which reconstructs one   */
/* scan per run, main.cpp:60-66)                                            */
/* ------------------------------------------------------------------------ */

/* A batch of scans of any shapes, one context each (same device, same
 * precision, views set, backprojection layout supported). wfbp_batch_run
 * rebins and filters every scan with its own launches, backprojects ALL
 * scans in one persistent launch whose CTAs take (scan, column tile, slab)
 * work items from a list sorted by estimated cost, and thickens per scan.
 * The chain is captured into a CUDA graph on the first call and replayed
 * while the raw / volume pointers stay the same (new pointers: recaptured).
 * The batch owns the intermediates; the contexts must outlive it.
 * stream NULL: runs on an internal stream, synchronous on return. */
typedef struct wfbp_batch wfbp_batch;
int wfbp_batch_create(wfbp_ctx* const* ctxs, int n, wfbp_batch** out);
int wfbp_batch_destroy(wfbp_batch* batch);
int wfbp_batch_run(wfbp_batch* batch, const float* const* raws, float* const* volumes, void* stream);
/* wfbp_batch_run from HOST buffers (pinned for overlap): the readings are
 * copied scan by scan on a second stream; the leading scans holding a quarter
 * of the readings' bytes are reconstructed (one persistent backprojection
 * launch) while the remaining copies land, and their volumes are copied back
 * while the rest of the batch runs (a second launch). The volumes equal
 * wfbp_batch_run's. Synchronous. The batch keeps device copies of the
 * readings and volumes after the first call. Like wfbp_run_host for one scan
 * (ReconstructionMachine's host-in / host-out RunReconstruction,
 * ReconstructionMachine.cu:141-434, over several scans). */
int wfbp_batch_run_host(wfbp_batch* batch, const float* const* raws_host, float* const* volumes_host,
                        void* stream);
int wfbp_batch_size(const wfbp_batch* batch, int* n_scans, int* n_items);
/* Backprojection configurations that fit every scan of the batch, and the
 * one in use (the autotuner times them and sets the fastest; setting one
 * drops the captured graph). */
int wfbp_batch_bp_configs(const wfbp_batch* batch, wfbp_bp_config* out, int cap, int* n);
int wfbp_batch_get_bp_config(const wfbp_batch* batch, wfbp_bp_config* config);
int wfbp_batch_set_bp_config(wfbp_batch* batch, const wfbp_bp_config* config);
/* Reads and clears the batch's device-side error word and those of its
 * scans' contexts (synchronous); statuses as wfbp_check_device_status. */
int wfbp_batch_check_device_status(wfbp_batch* batch);
const char* wfbp_batch_last_error(const wfbp_batch* batch);

/* ------------------------------------------------------------------------ */
/* Adjoints of the FP32 form (no counterpart in the reference, which has no */
/* backward pass). Each is the exact transpose of its forward stage, with   */
/* every output element owned by one thread (no atomics, deterministic).    */
/* Buffers are FP32 device arrays in the reference layout; all need         */
/* wfbp_set_views and a context with WFBP_PRECISION_FP32.                   */
/* ------------------------------------------------------------------------ */

/* Overwrites taps h[0..n-1] of the context's symmetric half taps (device or
 * host pointer, stream-ordered copy) -- the learnable part of the filter.
 * The taps start as generate_filter's (ReconstructionMachine.cu:478-513)
 * or the ext's window; wfbp_get_taps reads all n_channels of them. */
int wfbp_set_taps(wfbp_ctx* ctx, const float* taps, int n, void* stream);
int wfbp_get_taps(wfbp_ctx* ctx, float* taps, void* stream);

/* Transpose of wfbp_thicken: g_volume [nz_requested][ny][nx] ->
 * g_native [nz_native][ny][nx]. */
int wfbp_thicken_adjoint(wfbp_ctx* ctx, const float* g_volume, float* g_native, void* stream);

/* Transpose of wfbp_backproject (reference layout, FP32):
 * g_native [nz_native][ny][nx] -> g_filtered [V][nr][nch]. Voxels the
 * forward leaves NaN (no contributing view) contribute nothing. */
int wfbp_backproject_adjoint(wfbp_ctx* ctx, const float* g_native, float* g_filtered, void* stream);

/* Transpose of wfbp_filter (FP32): the Toeplitz operator is symmetric, so
 * this filters g_filtered [V][nr][nch] with the same taps. */
int wfbp_filter_adjoint(wfbp_ctx* ctx, const float* g_filtered, float* g_rebinned, void* stream);

/* Transpose of wfbp_rebin: g_rebinned [V][nr][nch] -> g_raw
 * [n_readings][raw_rows][raw_channels], with the context's texel weights.
 * Not for flying-focal-spot scans (WFBP_ERR_UNSUPPORTED). */
int wfbp_rebin_adjoint(wfbp_ctx* ctx, const float* g_rebinned, float* g_raw, void* stream);

/* Gradient of the filter taps: g_taps[d] = sum over rows of
 * sum_n g[n] (x[n-d] + x[n+d]) (d > 0; sum_n g[n] x[n] for d = 0), d < n,
 * where x are the rebinned rows, recomputed from `raw` inside the kernel
 * (nothing of the rebinned array is stored) and g = g_filtered. */
int wfbp_taps_gradient(wfbp_ctx* ctx, const float* raw, const float* g_filtered, float* g_taps, int n,
                       void* stream);

/* ------------------------------------------------------------------------ */
/* Input files (host only)                                                   */
/* ------------------------------------------------------------------------ */

/* The recon-parameter YAML file of fct_wfbp (parse_config,
 * applications/fct_wfbp/src/parse_config.cpp:31-63): keys raw_data_dir,
 * output_dir, start_pos, end_pos, recon_fov, slice_thickness, slice_pitch,
 * nx, ny, recon_kernel, x_origin, y_origin, tube_angle_offset,
 * adaptive_filtration_s; absent keys stay 0, slice_pitch 0 becomes
 * slice_thickness, output_file is "<path>_recon.dat". Flat `key: value`
 * YAML only (WFBP_ERR_INVALID_ARG otherwise). */
int wfbp_parse_recon_config(const char* path, ReconConfig* rp);

/* FreeCT 2-file scan format (fct_read: RawDataSet::writeAll,
 * modules/fct_read/src/RawDataSet.cpp:84-104; FreeCTFrame::readFromFile,
 * FreeCTDataSet.cpp:8-21): <dir>/meta.yaml and <dir>/projections.dat, one
 * frame per reading = {float angle, axial, radial; float [rows][channels]}.
 * wfbp_read_meta fills the scan metadata (flying_focal_spot_mode FFSNONE /
 * FFSZ / FFSXY / FFSXYZ); wfbp_read_frames reads readings [first,
 * first+count) into host arrays (tube_angles / table_positions may be
 * NULL), one seek for the whole window; wfbp_write_scan writes a scan. */
int wfbp_read_meta(const char* dir, wfbp_scan_meta* meta);
int wfbp_read_frames(const char* dir, const wfbp_scan_meta* meta, int first, int count, float* tube_angles,
                     float* table_positions, float* raw);
int wfbp_write_scan(const char* dir, const wfbp_scan_meta* meta, const float* tube_angles,
                    const float* table_positions, const float* raw);

/* DICOM-CT-PD projection data, one reading per file (the TCIA LDCT format),
 * as fct_read's DicomDataSet reads it with DCMTK
 * (modules/fct_read/src/DicomDataSet.cpp): the directory's regular files in
 * name order (:156-162); wfbp_dicom_read_meta fills the scan metadata from the
 * first file (readMetadata, :232-316: detector rows (7029,1010), channels
 * (7029,1011), transverse / axial spacing (7029,1002) / (7029,1006), source to
 * isocentre (7031,1003) and to detector (7031,1031), readings per rotation
 * (7033,1013), central channel and row (7031,1033), flying-focal-spot mode
 * (7033,100E)); wfbp_dicom_read_frames reads readings [first, first+count):
 * tube angle (7031,1001), table position (7031,1002) and the uint16 pixel
 * data times the rescale slope plus intercept ((0028,1053), (0028,1052)) as
 * float [count][rows][channels], from a [rows][channels] or a
 * [channels][rows] image (DicomFrame::readFromFile, :56-155).
 * tube_angles / table_positions may be NULL. Implicit and explicit VR little
 * endian only; WFBP_ERR_INVALID_ARG for a missing element, another transfer
 * syntax or a size that does not match. Host only. */
int wfbp_dicom_read_meta(const char* dir, wfbp_scan_meta* meta);
int wfbp_dicom_read_frames(const char* dir, const wfbp_scan_meta* meta, int first, int count, float* tube_angles,
                           float* table_positions, float* raw);

/* ------------------------------------------------------------------------ */
/* Synthetic scans (test-data generator; no counterpart in the reference)    */
/* ------------------------------------------------------------------------ */

typedef struct wfbp_ellipsoid {
  double cx, cy, cz;          /* centre (mm) */
  double ax, ay, az;          /* semi-axes (mm) */
  double phi;                 /* rotation about z (rad) */
  double mu;                  /* additive attenuation (1/mm) */
} wfbp_ellipsoid;

typedef struct wfbp_synth_scan {
  int n_readings, rows, channels, readings_per_rotation;
  double sid, sdd;            /* mm */
  double dcol, drow;          /* detector spacing at the detector (mm) */
  double central_channel;
  double angle0, dangle;      /* tube angle of reading 0, signed step per reading (rad) */
  double z0, dz;              /* table position of reading 0, signed step per reading (mm) */
  double i0;                  /* incident photons (0 = noiseless line integrals) */
  unsigned long long seed;
  int ffs_mode;               /* wfbp_ffs_mode: reading n has focal state n % G (G = 4 for
                                 PHIZ: phi bit = state & 1, z bit = state >> 1; G = 2 otherwise)
                                 and samples the effective channels 2b + phi bit and rows
                                 2r + z bit of a detector with twice the channels / rows at
                                 half the spacing and central channel 2 c0 + 1/2 */
} wfbp_synth_scan;

/* Line integrals (and Poisson noise, log transform) through the ellipsoid
 * phantom in the geometry conventions that the reference's rebin and
 * backprojection invert. out: device FP32 [n_readings][rows][channels]. */
int wfbp_synth_project(const wfbp_synth_scan* scan, const wfbp_ellipsoid* ellipsoids,
                       int n_ellipsoids, float* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FREECT_WFBP_H */
