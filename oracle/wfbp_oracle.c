/*
 * wfbp_oracle.c -- CPU oracle for the helical WFBP path.
 *
 * TEST INFRASTRUCTURE ONLY. tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py use it as the checker; the product library
 * (freect_b200/lib/libfreect_wfbp.so) never links or calls it.
 *
 * Two forms of the same algorithm:
 *
 *  "ref32"  A single-precision restatement of the reference's own arithmetic,
 *           following applications/fct_wfbp/src/ReconstructionMachine.cu (RM)
 *           and applications/fct_wfbp/include/cuda_kernels.cuh (CK) line by
 *           line, including the behaviour of its implementation:
 *             - host reshape with channel and row flips (RM:147-162),
 *             - rebin with the index angle v*2pi/P, texel-centre offsets and
 *               clamp addressing of the 2-D texture (CK:11-39, RM:176-180),
 *               optionally with 8-bit fractional bilinear weights,
 *             - the zero-padded circular FFT filter, including the left pad
 *               of view 0 that the rebin never rewrites (it keeps the previous
 *               row's filtered output) and views beyond 8*floor(V/8) that the
 *               rebin grid skips (RM:184-292),
 *             - the p-flip kluge, the q index computed in double, the bounds
 *               tests, NaN where no half turn contributes (CK:198-287),
 *             - float-accumulated slice lists (RM:107-137),
 *             - thickening over every native slice (CK:289-320).
 *           The FFT convolution itself is evaluated in double and rounded to
 *           float (cuFFT's FP32 rounding is not reproduced).
 *
 *  "f64"    The same algorithm in double precision, without the
 *           implementation quirks: exact bilinear weights, linear
 *           convolution over the detector row, every view rebinned.
 *
 * Parity pin: the reference ships no golden vectors or known-answer tests
 * for this path. The ref32 form is pinned by (a) the filter-tap known
 * answers of resources/ramp.m:1-15, (b) the FFT/Toeplitz identity, and
 * (c) fixtures produced by the reference's own cuda_kernels.cuh compiled
 * from its source tree with a texture-object shim (oracle/ref_shim/) and
 * run on a B200; tests/golden/ holds those fixtures and the script that
 * made them.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "../include/freect_wfbp.h"

#define ORC_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* threads                                                                   */
/* ------------------------------------------------------------------------ */
static int g_threads = 0;

ORC_EXPORT void orc_set_threads(int n) { g_threads = n; }
ORC_EXPORT int orc_get_threads(void) {
  if (g_threads > 0) return g_threads;
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}

typedef void (*orc_body)(void* arg, long i0, long i1);
typedef struct { orc_body f; void* arg; long n; long chunk; long next; pthread_mutex_t mu; } orc_pool;

static void* orc_worker(void* p) {
  orc_pool* pool = (orc_pool*)p;
  for (;;) {
    pthread_mutex_lock(&pool->mu);
    long i0 = pool->next;
    pool->next += pool->chunk;
    pthread_mutex_unlock(&pool->mu);
    if (i0 >= pool->n) break;
    long i1 = i0 + pool->chunk;
    if (i1 > pool->n) i1 = pool->n;
    pool->f(pool->arg, i0, i1);
  }
  return NULL;
}

static void orc_parallel_for(long n, long chunk, orc_body f, void* arg) {
  int nt = orc_get_threads();
  if (chunk < 1) chunk = 1;
  if (nt <= 1 || n <= chunk) { f(arg, 0, n); return; }
  orc_pool pool = {f, arg, n, chunk, 0, PTHREAD_MUTEX_INITIALIZER};
  pthread_t th[256];
  if (nt > 256) nt = 256;
  int started = 0;
  for (int t = 0; t < nt; t++)
    if (pthread_create(&th[t], NULL, orc_worker, &pool) == 0) started++;
  if (started == 0) { f(arg, 0, n); return; }
  for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------ */
/* geometry: RM:44-74 + recon_structs.h:69-83, float host arithmetic          */
/* ------------------------------------------------------------------------ */
static const float PI_F = 3.1415926535897f; /* recon_structs.h:76,81 */

static size_t next_pow2_at_least(size_t n) {
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

ORC_EXPORT int orc_configure_geometry(const wfbp_scan_meta* m, const float* table, CTGeometry* cg,
                                      GPUPrecompute* gp) {
  if (!m || !table || !cg || !gp) return WFBP_ERR_INVALID_ARG;
  if (m->total_num_projections <= m->projections_per_rotation || m->projections_per_rotation < 2)
    return WFBP_ERR_INVALID_ARG;
  memset(cg, 0, sizeof(*cg));
  memset(gp, 0, sizeof(*gp));
  cg->total_number_of_projections = (size_t)m->total_num_projections;
  cg->projections_per_rotation = (size_t)m->projections_per_rotation;
  cg->detector_pixel_size_col = m->detector_transverse_spacing;
  cg->detector_pixel_size_row = m->detector_axial_spacing;
  cg->num_detector_cols = (size_t)m->detector_channels;
  cg->num_detector_cols_padded = 2 * (size_t)m->detector_channels;
  /* RM:54 pow(2, ceil(log(2 nch)/log 2)); equal to the next power of two for
   * every 2*nch that is not itself a power of two */
  cg->num_detector_cols_padded_fft = next_pow2_at_least(2 * (size_t)m->detector_channels);
  cg->num_detector_rows = (size_t)m->detector_rows;
  cg->num_detector_rows_padded = 2 * (size_t)m->detector_rows;
  cg->detector_central_col = m->detector_central_channel;
  cg->detector_central_row = m->detector_central_row;
  cg->distance_source_to_isocenter = m->dist_source_to_isocenter;
  cg->distance_source_to_detector = m->dist_source_to_detector;
  cg->collimated_slice_width =
      m->dist_source_to_isocenter * (m->detector_axial_spacing / m->dist_source_to_detector); /* RM:62 */
  cg->z_rot = fabsf(table[m->projections_per_rotation] - table[0]);                          /* RM:64 */
  float cone_offset = ((float)(cg->num_detector_rows - 1)) / 2.0f;                             /* RM:66 */
  cg->theta_cone = 2.0f * (float)atan((double)(cone_offset * cg->collimated_slice_width /
                                               cg->distance_source_to_isocenter)); /* RM:67 */
  cg->acquisition_field_of_view =
      2.0f * cg->distance_source_to_isocenter *
      (float)sin((double)((((float)cg->num_detector_cols - 1.0f) / 2.0f) * m->detector_transverse_spacing *
                          (1.0f / cg->distance_source_to_detector))); /* RM:69 */
  cg->anode_angle = m->anode_angle;
  cg->ffs_phi = (m->ffs_mode & WFBP_FFS_PHI) != 0;
  cg->ffs_z = (m->ffs_mode & WFBP_FFS_Z) != 0;
  cg->ffs_diag = 0;

  /* recon_structs.h:69-83 */
  gp->half_acquisition_fov = 0.5f * cg->acquisition_field_of_view;
  gp->half_acquisition_fov_squared = gp->half_acquisition_fov * gp->half_acquisition_fov;
  gp->projections_per_half_turn = (int)(cg->projections_per_rotation / 2);
  gp->n_half_turns = (int)(cg->total_number_of_projections / (size_t)gp->projections_per_half_turn);
  gp->distance_source_to_isocenter_squared = cg->distance_source_to_isocenter * cg->distance_source_to_isocenter;
  gp->z_rot_over_2_pi = cg->z_rot / (2.0f * PI_F);
  gp->recip_distance_source_to_detector = 1.0f / cg->distance_source_to_detector;
  gp->recip_distance_source_to_isocenter = 1.0f / cg->distance_source_to_isocenter;
  gp->tanf_theta_cone = (float)tan((double)(cg->theta_cone / 2.0f));
  gp->pixel_scale = cg->distance_source_to_detector / (cg->distance_source_to_isocenter * cg->detector_pixel_size_col);
  gp->two_pi_over_projections_per_rotation = 2.0f * PI_F / (float)cg->projections_per_rotation;
  return WFBP_OK;
}

/* RM:107-137. Either output may be NULL (count only). Returns counts. */
ORC_EXPORT int orc_slice_locations(const CTGeometry* cg, const ReconConfig* rp, float* native, int native_cap,
                                   int* n_native, float* req, int req_cap, int* n_req) {
  int nn = 0, nr = 0;
  if (rp->start_pos != rp->end_pos) {
    float span = rp->end_pos - rp->start_pos;
    float d_native = cg->collimated_slice_width * fabsf(span) / span;
    float d_req = rp->slice_pitch * fabsf(span) / span;
    if (d_req > 0) {
      for (float loc = rp->start_pos; loc < rp->end_pos; loc += d_native) {
        if (native && nn < native_cap) native[nn] = loc;
        nn++;
        if (nn > 10000000) return WFBP_ERR_INVALID_ARG;
      }
      for (float loc = rp->start_pos; loc < rp->end_pos; loc += d_req) {
        if (req && nr < req_cap) req[nr] = loc;
        nr++;
        if (nr > 10000000) return WFBP_ERR_INVALID_ARG;
      }
    } else {
      for (float loc = rp->start_pos; loc > rp->end_pos; loc += d_native) {
        if (native && nn < native_cap) native[nn] = loc;
        nn++;
        if (nn > 10000000) return WFBP_ERR_INVALID_ARG;
      }
      for (float loc = rp->start_pos; loc > rp->end_pos; loc += d_req) {
        if (req && nr < req_cap) req[nr] = loc;
        nr++;
        if (nr > 10000000) return WFBP_ERR_INVALID_ARG;
      }
    }
  } else {
    if (native && native_cap > 0) native[0] = rp->start_pos;
    if (req && req_cap > 0) req[0] = rp->start_pos;
    nn = nr = 1;
  }
  if (n_native) *n_native = nn;
  if (n_req) *n_req = nr;
  return WFBP_OK;
}

/* ------------------------------------------------------------------------ */
/* filter taps                                                               */
/* ------------------------------------------------------------------------ */

/* The lambda r(t) of RM:493-498, evaluated like the reference's host code:
 * sin/cos of a float argument in double, stored as float. */
static float ramp_r_f(float t) {
  float v = (float)(sin((double)t) / (double)t + (cos((double)t) - 1.0f) / (double)(t * t));
  if (t == 0) v = 0.5f;
  return v;
}

/* generate_filter (RM:478-513): N taps for i in [-N/2, N/2), then fftshift.
 * out[j] = f(i) with i = j for j < N/2 and i = j - N for j >= N/2. */
ORC_EXPORT void orc_filter_taps_ref_fft(const CTGeometry* cg, float c, float a, float* out) {
  int N = (int)cg->num_detector_cols_padded_fft;
  const float pi_f = 3.141592653589f; /* RM:490 */
  float ds = cg->detector_pixel_size_col * cg->distance_source_to_isocenter / cg->distance_source_to_detector;
  float* h = (float*)malloc(sizeof(float) * N);
  for (int i = -N / 2; i < N / 2; i++) {
    h[i + N / 2] = (c * c / (2.0f * ds)) *
                   (a * ramp_r_f(c * pi_f * i) + (((1.0f - a) / 2.0f) * ramp_r_f(pi_f * c * i + pi_f)) +
                    (((1.0f - a) / 2.0f) * ramp_r_f(pi_f * c * i - pi_f)));
  }
  for (int i = 0; i < N / 2; i++) { /* RM:509-513 */
    float tmp = h[i];
    h[i] = h[i + N / 2];
    h[i + N / 2] = tmp;
  }
  memcpy(out, h, sizeof(float) * N);
  free(h);
}

/* Discrete Shepp-Logan kernel in the reference's scaling (one factor of ds
 * folded into the taps like generate_filter): h[n] = -2 / (pi^2 ds (4n^2-1)). */
ORC_EXPORT void orc_filter_taps_f64(const CTGeometry* cg, int window, double c, double a, double* half, int n) {
  double ds = (double)cg->detector_pixel_size_col * (double)cg->distance_source_to_isocenter /
              (double)cg->distance_source_to_detector;
  for (int k = 0; k < n; k++) {
    double v;
    if (window == WFBP_FILTER_SHEPP_LOGAN) {
      v = -2.0 / (M_PI * M_PI * ds * (4.0 * k * k - 1.0));
    } else {
      double t0 = c * M_PI * k, tp = M_PI * c * k + M_PI, tm = M_PI * c * k - M_PI;
#define RR(t) ((t) == 0 ? 0.5 : sin(t) / (t) + (cos(t) - 1.0) / ((t) * (t)))
      v = (c * c / (2.0 * ds)) * (a * RR(t0) + ((1.0 - a) / 2.0) * RR(tp) + ((1.0 - a) / 2.0) * RR(tm));
#undef RR
    }
    half[k] = v;
  }
}

/* ------------------------------------------------------------------------ */
/* FFT (iterative radix-2, double, complex)                                  */
/* ------------------------------------------------------------------------ */
typedef struct { int n; int logn; double* c; double* s; int* rev; } fft_plan;

static int fft_init(fft_plan* p, int n) {
  int logn = 0;
  while ((1 << logn) < n) logn++;
  if ((1 << logn) != n) return -1;
  p->n = n; p->logn = logn;
  p->c = (double*)malloc(sizeof(double) * (n / 2 + 1));
  p->s = (double*)malloc(sizeof(double) * (n / 2 + 1));
  p->rev = (int*)malloc(sizeof(int) * n);
  for (int k = 0; k <= n / 2; k++) { p->c[k] = cos(2 * M_PI * k / n); p->s[k] = sin(2 * M_PI * k / n); }
  for (int i = 0; i < n; i++) {
    int r = 0;
    for (int b = 0; b < logn; b++) if (i & (1 << b)) r |= 1 << (logn - 1 - b);
    p->rev[i] = r;
  }
  return 0;
}
static void fft_free(fft_plan* p) { free(p->c); free(p->s); free(p->rev); }

/* forward: X[k] = sum x[j] e^{-2 pi i jk/n}; inverse without 1/n */
static void fft_run(const fft_plan* p, double* re, double* im, int inverse) {
  int n = p->n;
  for (int i = 0; i < n; i++) {
    int r = p->rev[i];
    if (r > i) { double t = re[i]; re[i] = re[r]; re[r] = t; t = im[i]; im[i] = im[r]; im[r] = t; }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1, step = n / len;
    for (int i = 0; i < n; i += len) {
      for (int k = 0; k < half; k++) {
        double wr = p->c[k * step], wi = inverse ? p->s[k * step] : -p->s[k * step];
        int a = i + k, b = a + half;
        double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
        re[b] = re[a] - xr; im[b] = im[a] - xi;
        re[a] += xr; im[a] += xi;
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* rebin                                                                     */
/* ------------------------------------------------------------------------ */

/* Texel (b, view) of row sheet i: the reshape of RM:153-162 places
 * raw[view][r][k] at sheet[nr-1-r][view][nch-1-k]. */
static inline float sheet_texel(const float* raw, int nr, int nch, int r_raw, int b, int view) {
  return raw[((size_t)view * nr + r_raw) * nch + (nch - 1 - b)];
}

/* tex2D with cudaFilterModeLinear, cudaAddressModeClamp, unnormalised
 * coordinates: xB = x - 0.5, i = floor(xB), alpha = frac(xB) (same in y);
 * q8 rounds the fractions to 8 bits like the texture unit's 9-bit
 * fixed-point weights. */
static float tex2d_ref(const float* raw, int nr, int nch, int V, int r_raw, float x, float y, int q8) {
  float xb = x - 0.5f, yb = y - 0.5f;
  float fx = floorf(xb), fy = floorf(yb);
  float ax = xb - fx, ay = yb - fy;
  if (q8) { ax = rintf(ax * 256.0f) / 256.0f; ay = rintf(ay * 256.0f) / 256.0f; }
  long i0 = (long)fx, j0 = (long)fy, i1 = i0 + 1, j1 = j0 + 1;
  if (i0 < 0) i0 = 0; if (i0 > nch - 1) i0 = nch - 1;
  if (i1 < 0) i1 = 0; if (i1 > nch - 1) i1 = nch - 1;
  if (j0 < 0) j0 = 0; if (j0 > V - 1) j0 = V - 1;
  if (j1 < 0) j1 = 0; if (j1 > V - 1) j1 = V - 1;
  float t00 = sheet_texel(raw, nr, nch, r_raw, (int)i0, (int)j0);
  float t10 = sheet_texel(raw, nr, nch, r_raw, (int)i1, (int)j0);
  float t01 = sheet_texel(raw, nr, nch, r_raw, (int)i0, (int)j1);
  float t11 = sheet_texel(raw, nr, nch, r_raw, (int)i1, (int)j1);
  return (1.0f - ax) * (1.0f - ay) * t00 + ax * (1.0f - ay) * t10 + (1.0f - ax) * ay * t01 + ax * ay * t11;
}

/* rebin_kernel (CK:11-39) value at output channel c (< nch) of view v */
static float rebin_value_ref(const CTGeometry* cg, const float* raw, int r_raw, int c, int v, int q8) {
  int nch = (int)cg->num_detector_cols, nr = (int)cg->num_detector_rows, V = (int)cg->total_number_of_projections;
  float delta_theta = 2.0f * 3.14159265f / (float)cg->projections_per_rotation;
  float p = ((float)c - cg->detector_central_col) * (float)cg->detector_pixel_size_col;
  float beta = asinf(p / cg->distance_source_to_detector);
  float theta = (float)v * delta_theta;
  float alpha = theta - beta;
  float beta_idx = (beta * cg->distance_source_to_detector / cg->detector_pixel_size_col) + cg->detector_central_col;
  float alpha_idx = alpha / delta_theta;
  if (beta_idx < 0 || beta_idx >= (float)cg->num_detector_cols || isnan(beta_idx)) return 0.0f;
  return tex2d_ref(raw, nr, nch, V, r_raw, beta_idx + 0.5f, (float)(alpha_idx + 0.5), q8);
}

/* Clean FP32 rebin (stage boundary of the product): out[v][i][c], every view. */
typedef struct { const CTGeometry* cg; const float* raw; float* out; int q8; } rb32_args;
static void rb32_body(void* a_, long i0, long i1) {
  rb32_args* a = (rb32_args*)a_;
  int nr = (int)a->cg->num_detector_rows, nch = (int)a->cg->num_detector_cols;
  for (long row = i0; row < i1; row++) {
    int v = (int)(row / nr), i = (int)(row % nr);
    int r_raw = nr - 1 - i;
    for (int c = 0; c < nch; c++) a->out[row * nch + c] = rebin_value_ref(a->cg, a->raw, r_raw, c, v, a->q8);
  }
}
ORC_EXPORT void orc_rebin_ref32(const CTGeometry* cg, const float* raw, int q8, float* out) {
  rb32_args a = {cg, raw, out, q8};
  long rows = (long)cg->total_number_of_projections * (long)cg->num_detector_rows;
  orc_parallel_for(rows, 64, rb32_body, &a);
}

/* FP64 rebin: exact bilinear weights, clamp addressing, all views. `off`:
 * index of the first reading within the whole scan (a window of readings is
 * rebinned with the whole scan's index angles, rebin_kernel CK:15-20). */
typedef struct { const CTGeometry* cg; const float* raw; double* out; long off; } rb64_args;
static void rb64_body(void* a_, long i0, long i1) {
  rb64_args* a = (rb64_args*)a_;
  const CTGeometry* cg = a->cg;
  int nr = (int)cg->num_detector_rows, nch = (int)cg->num_detector_cols, V = (int)cg->total_number_of_projections;
  double dth = 2.0 * M_PI / (double)cg->projections_per_rotation;
  double c0 = cg->detector_central_col, dcol = cg->detector_pixel_size_col, sdd = cg->distance_source_to_detector;
  for (long row = i0; row < i1; row++) {
    int v = (int)(row / nr), i = (int)(row % nr);
    int r_raw = nr - 1 - i;
    for (int c = 0; c < nch; c++) {
      double p = ((double)c - c0) * dcol;
      double beta = asin(p / sdd);
      double bidx = beta * sdd / dcol + c0;
      double aidx = (double)(v + a->off) - beta / dth;
      double val = 0.0;
      if (!(bidx < 0 || bidx >= (double)nch || isnan(bidx))) {
        double fx = floor(bidx), fy = floor(aidx);
        double ax = bidx - fx, ay = aidx - fy;
        long x0 = (long)fx, y0 = (long)fy - a->off, x1 = x0 + 1, y1 = y0 + 1;
        if (x0 < 0) x0 = 0; if (x0 > nch - 1) x0 = nch - 1;
        if (x1 < 0) x1 = 0; if (x1 > nch - 1) x1 = nch - 1;
        if (y0 < 0) y0 = 0; if (y0 > V - 1) y0 = V - 1;
        if (y1 < 0) y1 = 0; if (y1 > V - 1) y1 = V - 1;
        double t00 = sheet_texel(a->raw, nr, nch, r_raw, (int)x0, (int)y0);
        double t10 = sheet_texel(a->raw, nr, nch, r_raw, (int)x1, (int)y0);
        double t01 = sheet_texel(a->raw, nr, nch, r_raw, (int)x0, (int)y1);
        double t11 = sheet_texel(a->raw, nr, nch, r_raw, (int)x1, (int)y1);
        val = (1 - ax) * (1 - ay) * t00 + ax * (1 - ay) * t10 + (1 - ax) * ay * t01 + ax * ay * t11;
      }
      a->out[row * nch + c] = val;
    }
  }
}
ORC_EXPORT void orc_rebin_f64_off(const CTGeometry* cg, const float* raw, long off, double* out) {
  rb64_args a = {cg, raw, out, off};
  long rows = (long)cg->total_number_of_projections * (long)cg->num_detector_rows;
  orc_parallel_for(rows, 64, rb64_body, &a);
}
ORC_EXPORT void orc_rebin_f64(const CTGeometry* cg, const float* raw, double* out) { orc_rebin_f64_off(cg, raw, 0, out); }

/* ------------------------------------------------------------------------ */
/* filter                                                                    */
/* ------------------------------------------------------------------------ */

/* Linear convolution along channels with symmetric taps h[0..nch-1] (FP64):
 * y[m] = sum_{k<nch} h[|m-k|] x[k]. in/out may be float or double rows. */
typedef struct {
  int nch, L; const double* H_re; const double* H_im; long rows;
  const double* in64; const float* in32; double* out64; float* out32;
} lconv_args;

static void lconv_body(void* a_, long i0, long i1) {
  lconv_args* a = (lconv_args*)a_;
  fft_plan p;
  fft_init(&p, a->L);
  double* re = (double*)malloc(sizeof(double) * a->L);
  double* im = (double*)malloc(sizeof(double) * a->L);
  for (long pr = i0; pr < i1; pr++) {
    long r0 = 2 * pr, r1 = 2 * pr + 1;
    memset(re, 0, sizeof(double) * a->L);
    memset(im, 0, sizeof(double) * a->L);
    for (int k = 0; k < a->nch; k++) {
      re[k] = a->in64 ? a->in64[r0 * a->nch + k] : a->in32[r0 * a->nch + k];
      if (r1 < a->rows) im[k] = a->in64 ? a->in64[r1 * a->nch + k] : a->in32[r1 * a->nch + k];
    }
    fft_run(&p, re, im, 0);
    for (int k = 0; k < a->L; k++) {
      double xr = re[k] * a->H_re[k] - im[k] * a->H_im[k];
      double xi = re[k] * a->H_im[k] + im[k] * a->H_re[k];
      re[k] = xr; im[k] = xi;
    }
    fft_run(&p, re, im, 1);
    for (int k = 0; k < a->nch; k++) {
      double y0 = re[k] / a->L, y1 = im[k] / a->L;
      if (a->out64) {
        a->out64[r0 * a->nch + k] = y0;
        if (r1 < a->rows) a->out64[r1 * a->nch + k] = y1;
      } else {
        a->out32[r0 * a->nch + k] = (float)y0;
        if (r1 < a->rows) a->out32[r1 * a->nch + k] = (float)y1;
      }
    }
  }
  free(re); free(im);
  fft_free(&p);
}

static void lconv_rows(int nch, long rows, const double* half, const double* in64, const float* in32,
                       double* out64, float* out32) {
  int L = (int)next_pow2_at_least(2 * (size_t)nch);
  double* hr = (double*)calloc(L, sizeof(double));
  double* hi = (double*)calloc(L, sizeof(double));
  for (int d = 0; d < nch; d++) { hr[d] = half[d]; if (d) hr[L - d] = half[d]; }
  fft_plan p;
  fft_init(&p, L);
  fft_run(&p, hr, hi, 0);
  fft_free(&p);
  lconv_args a = {nch, L, hr, hi, rows, in64, in32, out64, out32};
  orc_parallel_for((rows + 1) / 2, 16, lconv_body, &a);
  free(hr); free(hi);
}

/* FP64 filter of rebinned rows [rows][nch]. */
ORC_EXPORT void orc_filter_f64(int nch, long rows, const double* half, const double* in, double* out) {
  lconv_rows(nch, rows, half, in, NULL, out, NULL);
}
/* FP32 rows, FP64 arithmetic, rounded to float (ideal FP32 filter). */
ORC_EXPORT void orc_filter_f32(int nch, long rows, const double* half, const float* in, float* out) {
  lconv_rows(nch, rows, half, NULL, in, NULL, out);
}

/* The reference's rebin + filter + reshape, faithful to its padded sheet
 * state (RM:141-306): sheet i is rebinned into a zero-initialised
 * [V][N_fft] buffer that persists across rows; the circular FFT convolution
 * with the fftshifted taps (cuFFT R2C, multiply_filter's 1/N, C2R) runs on
 * every view; reshape copies the data window. taps_fft: N_fft taps as
 * orc_filter_taps_ref_fft returns them. flags bit0: 8-bit texture weights. */
typedef struct {
  const CTGeometry* cg; const float* raw; float* sheet; int r_raw; int q8; int Vr;
  int N; int off; const double* H_re; const double* H_im;
} rf_args;

static void rf_rebin_body(void* a_, long v0, long v1) {
  rf_args* a = (rf_args*)a_;
  int nch = (int)a->cg->num_detector_cols;
  for (long v = v0; v < v1; v++) {
    for (int c = 0; c < a->N; c++) {
      size_t out_idx = (size_t)(c + a->off) + (size_t)v * a->N;
      float val = (c < nch) ? rebin_value_ref(a->cg, a->raw, a->r_raw, c, (int)v, a->q8) : 0.0f;
      a->sheet[out_idx] = val;
    }
  }
}

static void rf_fft_body(void* a_, long p0, long p1) {
  rf_args* a = (rf_args*)a_;
  int N = a->N;
  long V = (long)a->cg->total_number_of_projections;
  fft_plan p;
  fft_init(&p, N);
  double* re = (double*)malloc(sizeof(double) * N);
  double* im = (double*)malloc(sizeof(double) * N);
  for (long pr = p0; pr < p1; pr++) {
    long v0 = 2 * pr, v1 = 2 * pr + 1;
    for (int k = 0; k < N; k++) {
      re[k] = a->sheet[(size_t)v0 * N + k];
      im[k] = v1 < V ? a->sheet[(size_t)v1 * N + k] : 0.0;
    }
    fft_run(&p, re, im, 0);
    for (int k = 0; k < N; k++) {
      double xr = re[k] * a->H_re[k] - im[k] * a->H_im[k];
      double xi = re[k] * a->H_im[k] + im[k] * a->H_re[k];
      re[k] = xr; im[k] = xi;
    }
    fft_run(&p, re, im, 1);
    for (int k = 0; k < N; k++) {
      a->sheet[(size_t)v0 * N + k] = (float)(re[k] / N);
      if (v1 < V) a->sheet[(size_t)v1 * N + k] = (float)(im[k] / N);
    }
  }
  free(re); free(im);
  fft_free(&p);
}

ORC_EXPORT int orc_rebin_filter_ref32(const CTGeometry* cg, const float* raw, const float* taps_fft, int flags,
                                      float* filtered) {
  int N = (int)cg->num_detector_cols_padded_fft;
  int nch = (int)cg->num_detector_cols, nr = (int)cg->num_detector_rows;
  long V = (long)cg->total_number_of_projections;
  int off = (N - nch) / 2;
  /* + N floats of slack: the rebin grid of the last view writes up to
   * off floats past the [V][N] sheet (CK:29-37 with RM:255) */
  float* sheet = (float*)calloc((size_t)V * N + N, sizeof(float));
  if (!sheet) return WFBP_ERR_OOM;
  double* hr = (double*)malloc(sizeof(double) * N);
  double* hi = (double*)calloc(N, sizeof(double));
  for (int k = 0; k < N; k++) hr[k] = taps_fft[k];
  fft_plan p;
  fft_init(&p, N);
  fft_run(&p, hr, hi, 0);
  fft_free(&p);
  int Vr = (int)(V / 8) * 8; /* rebin grid covers 8*floor(V/8) views (RM:255) */
  for (int i = 0; i < nr; i++) {
    rf_args a = {cg, raw, sheet, nr - 1 - i, flags & 1, Vr, N, off, hr, hi};
    orc_parallel_for(Vr, 32, rf_rebin_body, &a);
    orc_parallel_for((V + 1) / 2, 16, rf_fft_body, &a);
    for (long v = 0; v < V; v++) /* CK:60-77 */
      memcpy(&filtered[((size_t)v * nr + i) * nch], &sheet[(size_t)v * N + off], sizeof(float) * nch);
  }
  free(sheet); free(hr); free(hi);
  return WFBP_OK;
}

/* ------------------------------------------------------------------------ */
/* backprojection                                                            */
/* ------------------------------------------------------------------------ */

/* W() of CK:79-93 */
static inline float w_ref(float q) {
  const float Q = 0.6f;
  float wq;
  q = fabsf(q);
  if (q < Q) wq = 1.0f;
  else if (Q <= q && q < 1.0f) {
    wq = cosf((0.5f * 3.14159265f) * (q - Q) / (1.0f - Q));
    wq = wq * wq;
  } else wq = 0.0f;
  return wq;
}
static inline double w_f64(double q) {
  const double Q = 0.6;
  q = fabs(q);
  if (q < Q) return 1.0;
  if (q < 1.0) { double w = cos(0.5 * M_PI * (q - Q) / (1.0 - Q)); return w * w; }
  return 0.0;
}

typedef struct {
  const CTGeometry* cg; const ReconConfig* rp; const GPUPrecompute* gp;
  const float* D; const float* tube; const float* table; const float* slices; int nz; float* vol;
} bp32_args;

/* backproject_kernel (CK:198-287), one (slice, y) row of voxels per item */
static void bp32_body(void* a_, long i0, long i1) {
  bp32_args* a = (bp32_args*)a_;
  const CTGeometry* cg = a->cg; const ReconConfig* rp = a->rp; const GPUPrecompute* gp = a->gp;
  int nx = (int)rp->nx, ny = (int)rp->ny;
  size_t nch = cg->num_detector_cols, nr = cg->num_detector_rows;
  for (long item = i0; item < i1; item++) {
    int s = (int)(item / ny), iy = (int)(item % ny);
    float y_loc = ((float)iy - 0.5f * ((float)rp->ny - 1.0f)) * rp->recon_fov / (float)rp->ny + rp->y_origin;
    float z_loc = a->slices[s];
    for (int ix = 0; ix < nx; ix++) {
      float x_loc = ((float)ix - 0.5f * ((float)rp->nx - 1.0f)) * rp->recon_fov / (float)rp->nx + rp->x_origin;
      float* out = &a->vol[((size_t)s * ny + iy) * nx + ix];
      if (x_loc * x_loc + y_loc * y_loc > gp->half_acquisition_fov_squared) continue;
      for (int t = 0; t < gp->projections_per_half_turn; t++) {
        float bp = 0.0f, nf = 0.0f;
        for (int k = 0; k < gp->n_half_turns; k++) {
          int j = t + k * gp->projections_per_half_turn;
          float zt = a->table[j];
          if (fabsf(zt - z_loc) > cg->z_rot) continue;
          float th = a->tube[j];
          float p_hat = x_loc * sinf(th) - y_loc * cosf(th);
          float l_hat = sqrtf(gp->distance_source_to_isocenter_squared - powf(p_hat, 2.0f)) - x_loc * cosf(th) -
                        y_loc * sinf(th);
          float q_hat = (z_loc - zt + (gp->z_rot_over_2_pi) * asinf(gp->recip_distance_source_to_isocenter * p_hat)) /
                        (l_hat * gp->tanf_theta_cone);
          if (q_hat > 1.0f || q_hat < -1.0f) continue;
          float p_idx = p_hat * gp->pixel_scale + cg->detector_central_col;
          float q_idx = (float)(0.5 * (double)(q_hat + 1.0f) * (double)((float)nr - 1.0f));
          p_idx = (float)(((double)nch + 1.75) - (double)p_idx);
          int q_floor = (int)floorf(q_idx), q_ceil = (int)ceilf(q_idx);
          int p_floor = (int)floorf(p_idx), p_ceil = (int)ceilf(p_idx);
          if (p_floor < 0 || q_floor < 0) continue;
          if ((size_t)p_ceil >= nch - 1 || (size_t)q_ceil >= nr - 1) continue;
          float w_q = q_idx - (float)q_floor, w_p = p_idx - (float)p_floor;
          size_t lo = (size_t)p_floor + (size_t)q_floor * nch + (size_t)j * nr * nch;
          size_t hi = (size_t)p_floor + (size_t)(q_floor + 1) * nch + (size_t)j * nr * nch;
          float g = (1.0f - w_q) * (1.0f - w_p) * a->D[lo] + (1.0f - w_q) * (w_p)*a->D[lo + 1] +
                    (w_q) * (1.0f - w_p) * a->D[hi] + (w_q) * (w_p)*a->D[hi + 1];
          float W = w_ref(q_hat);
          bp += W * g;
          nf += W;
        }
        *out += gp->two_pi_over_projections_per_rotation * (1.0f / nf) * bp;
      }
    }
  }
}

/* vol: [nz][ny][nx], zeroed here (RM:341) */
ORC_EXPORT void orc_backproject_ref32(const CTGeometry* cg, const ReconConfig* rp, const GPUPrecompute* gp,
                                      const float* filtered, const float* tube, const float* table,
                                      const float* slices, int nz, float* vol) {
  memset(vol, 0, sizeof(float) * (size_t)nz * rp->nx * rp->ny);
  bp32_args a = {cg, rp, gp, filtered, tube, table, slices, nz, vol};
  orc_parallel_for((long)nz * (long)rp->ny, 1, bp32_body, &a);
}

/* FP64 form. Geometry derived in double from the float base geometry. */
typedef struct {
  double sid, sid2, sdd, dcol, c0, afov_half2, z_rot, zr2pi, tanc, pixel_scale, dtheta;
  int P2, K, nch, nr, nx, ny; double fov, x0, y0;
} bp64_geo;

typedef struct {
  bp64_geo g; const double* D; const double* tube; const double* table; const double* slices; int nz;
  double* vol; unsigned long long* counts; /* per item */
} bp64_args;

static void bp64_geo_init(bp64_geo* g, const CTGeometry* cg, const ReconConfig* rp, const double* table) {
  g->sid = cg->distance_source_to_isocenter; g->sid2 = g->sid * g->sid;
  g->sdd = cg->distance_source_to_detector; g->dcol = cg->detector_pixel_size_col;
  g->c0 = cg->detector_central_col;
  g->nch = (int)cg->num_detector_cols; g->nr = (int)cg->num_detector_rows;
  double drow = cg->detector_pixel_size_row;
  double csw = g->sid * drow / g->sdd;
  double theta_cone = 2.0 * atan(((g->nr - 1) / 2.0) * csw / g->sid);
  double afov = 2.0 * g->sid * sin(((g->nch - 1.0) / 2.0) * g->dcol / g->sdd);
  g->afov_half2 = 0.25 * afov * afov;
  int P = (int)cg->projections_per_rotation;
  (void)table;
  g->z_rot = (double)cg->z_rot;  /* ConfigureCTGeometry's |z[P] - z[0]| (RM.cu:64) */
  g->zr2pi = g->z_rot / (2.0 * M_PI);
  g->tanc = tan(theta_cone / 2.0);
  g->pixel_scale = g->sdd / (g->sid * g->dcol);
  g->dtheta = 2.0 * M_PI / P;
  g->P2 = P / 2;
  g->K = (int)(cg->total_number_of_projections / (size_t)g->P2);
  g->nx = (int)rp->nx; g->ny = (int)rp->ny;
  g->fov = rp->recon_fov; g->x0 = rp->x_origin; g->y0 = rp->y_origin;
}

static void bp64_body(void* a_, long i0, long i1) {
  bp64_args* a = (bp64_args*)a_;
  const bp64_geo* g = &a->g;
  size_t nch = (size_t)g->nch, nr = (size_t)g->nr;
  for (long item = i0; item < i1; item++) {
    int s = (int)(item / g->ny), iy = (int)(item % g->ny);
    double y = (iy - 0.5 * (g->ny - 1.0)) * g->fov / g->ny + g->y0;
    double z = a->slices[s];
    unsigned long long cnt = 0;
    for (int ix = 0; ix < g->nx; ix++) {
      double x = (ix - 0.5 * (g->nx - 1.0)) * g->fov / g->nx + g->x0;
      double* out = &a->vol[((size_t)s * g->ny + iy) * g->nx + ix];
      *out = 0.0;
      if (x * x + y * y > g->afov_half2) continue;
      double acc = 0.0;
      for (int t = 0; t < g->P2; t++) {
        double bp = 0.0, nf = 0.0;
        for (int k = 0; k < g->K; k++) {
          int j = t + k * g->P2;
          double zt = a->table[j];
          if (fabs(zt - z) > g->z_rot) continue;
          double th = a->tube[j], sn = sin(th), cs = cos(th);
          double p_hat = x * sn - y * cs;
          double l_hat = sqrt(g->sid2 - p_hat * p_hat) - x * cs - y * sn;
          double q_hat = (z - zt + g->zr2pi * asin(p_hat / g->sid)) / (l_hat * g->tanc);
          if (q_hat > 1.0 || q_hat < -1.0) continue;
          double p_idx = (g->nch + 1.75) - (p_hat * g->pixel_scale + g->c0);
          double q_idx = 0.5 * (q_hat + 1.0) * (g->nr - 1.0);
          double pf = floor(p_idx), qf = floor(q_idx);
          if (pf < 0 || qf < 0) continue;
          if (ceil(p_idx) >= g->nch - 1 || ceil(q_idx) >= g->nr - 1) continue;
          double wq = q_idx - qf, wp = p_idx - pf;
          size_t lo = (size_t)pf + (size_t)qf * nch + (size_t)j * nr * nch;
          size_t hi = lo + nch;
          double gv = (1 - wq) * (1 - wp) * a->D[lo] + (1 - wq) * wp * a->D[lo + 1] + wq * (1 - wp) * a->D[hi] +
                      wq * wp * a->D[hi + 1];
          double W = w_f64(q_hat);
          bp += W * gv;
          nf += W;
          cnt++;
        }
        acc += g->dtheta * (1.0 / nf) * bp;
      }
      *out = acc;
    }
    if (a->counts) a->counts[item] = cnt;
  }
}

/* FP64 backprojection; returns the number of contributing voxel-view
 * updates (voxels inside the acquisition FOV, views passing every test). */
ORC_EXPORT unsigned long long orc_backproject_f64(const CTGeometry* cg, const ReconConfig* rp,
                                                  const double* filtered, const double* tube,
                                                  const double* table, const double* slices, int nz,
                                                  double* vol) {
  bp64_args a;
  bp64_geo_init(&a.g, cg, rp, table);
  a.D = filtered; a.tube = tube; a.table = table; a.slices = slices; a.nz = nz; a.vol = vol;
  long items = (long)nz * (long)rp->ny;
  a.counts = (unsigned long long*)calloc(items, sizeof(unsigned long long));
  orc_parallel_for(items, 1, bp64_body, &a);
  unsigned long long total = 0;
  for (long i = 0; i < items; i++) total += a.counts[i];
  free(a.counts);
  return total;
}

/* ------------------------------------------------------------------------ */
/* thickening (CK:289-320)                                                   */
/* ------------------------------------------------------------------------ */
ORC_EXPORT void orc_thicken_ref32(const ReconConfig* rp, const float* vol_native, const float* z_native, int nz,
                                  const float* z_req, int nzr, float* out) {
  size_t plane = rp->nx * rp->ny;
  for (int r = 0; r < nzr; r++) {
    for (size_t px = 0; px < plane; px++) {
      float val = 0.0f, ws = 0.0f;
      for (int i = 0; i < nz; i++) {
        float w = fmaxf(0.0f, 1.0f - fabsf(z_native[i] - z_req[r]) / rp->slice_thickness);
        if (w == 0.0f) continue;
        ws += w;
        val += w * vol_native[(size_t)i * plane + px];
      }
      out[(size_t)r * plane + px] = val / ws;
    }
  }
}
ORC_EXPORT void orc_thicken_f64(const ReconConfig* rp, const double* vol_native, const double* z_native, int nz,
                                const double* z_req, int nzr, double* out) {
  size_t plane = rp->nx * rp->ny;
  for (int r = 0; r < nzr; r++) {
    for (size_t px = 0; px < plane; px++) {
      double val = 0.0, ws = 0.0;
      for (int i = 0; i < nz; i++) {
        double w = 1.0 - fabs(z_native[i] - z_req[r]) / rp->slice_thickness;
        if (w <= 0.0) continue;
        ws += w;
        val += w * vol_native[(size_t)i * plane + px];
      }
      out[(size_t)r * plane + px] = val / ws;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* synthetic scans: ellipsoid line integrals + Poisson noise (FP64)          */
/* ------------------------------------------------------------------------ */

/* Philox4x32-10 (Salmon et al., SC'11) */
static void philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                       uint32_t out[4]) {
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
static inline double u01(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

static double poisson_draw(double lam, const uint32_t r[4]) {
  if (lam <= 0) return 0.0;
  if (lam < 64.0) {
    double u = u01(r[0]), p = exp(-lam), F = p;
    int k = 0;
    while (u > F && k < 4096) { k++; p *= lam / k; F += p; }
    return (double)k;
  }
  double z = sqrt(-2.0 * log(u01(r[0]))) * cos(2.0 * M_PI * u01(r[1]));
  double n = floor(lam + sqrt(lam) * z + 0.5);
  return n < 0 ? 0.0 : n;
}

static double chord_sum(const wfbp_ellipsoid* e, int ne, const double S[3], const double U[3]) {
  double unorm = sqrt(U[0] * U[0] + U[1] * U[1] + U[2] * U[2]);
  double total = 0.0;
  for (int n = 0; n < ne; n++) {
    double cp = cos(e[n].phi), sp = sin(e[n].phi);
    double dx = S[0] - e[n].cx, dy = S[1] - e[n].cy, dz = S[2] - e[n].cz;
    double px = (dx * cp + dy * sp) / e[n].ax, py = (-dx * sp + dy * cp) / e[n].ay, pz = dz / e[n].az;
    double ux = (U[0] * cp + U[1] * sp) / e[n].ax, uy = (-U[0] * sp + U[1] * cp) / e[n].ay, uz = U[2] / e[n].az;
    double A = ux * ux + uy * uy + uz * uz, B = px * ux + py * uy + pz * uz, C = px * px + py * py + pz * pz - 1.0;
    double disc = B * B - A * C;
    if (disc > 0) total += e[n].mu * (2.0 * sqrt(disc) / A) * unorm;
  }
  return total;
}

/* Ray of reading v, raw row r, raw channel k. The reference's rebin and
 * backprojection (CK:11-39, 198-287) invert this geometry exactly when the
 * tube angle decreases and the table position decreases with the reading
 * index: flipped channel b = nch-1-k has fan angle beta = (b-c0)*dcol/sdd,
 * the parallel direction is theta = angle_v - beta, the in-plane ray is
 * x sin(theta) - y cos(theta) = (nch + 1.75 - 2 c0) ds - R sin(beta), the
 * source sits on it at radius R, and flipped row rr = nr-1-r rises with
 * slope (rr - (nr-1)/2) drow/sdd per mm of in-plane distance. With a flying
 * focal spot the same holds on the effective detector (2x channels / rows at
 * half the spacing, central channel 2 c0 + 1/2), where reading v of focal
 * state (sp, sz) samples effective channel 2b + sp and effective row
 * 2 rr + sz (see orc_ffs_effective). */
static void synth_ray(const wfbp_synth_scan* s, long v, int r, int k, double S[3], double U[3]) {
  int nch = s->channels, nr = s->rows;
  const int phi = (s->ffs_mode & WFBP_FFS_PHI) != 0, zf = (s->ffs_mode & WFBP_FFS_Z) != 0;
  const int G = (phi ? 2 : 1) * (zf ? 2 : 1);
  const int rho = (int)(v % G);
  const int sp = phi ? (G == 4 ? (rho & 1) : rho) : 0, sz = zf ? (G == 4 ? (rho >> 1) : rho) : 0;
  const int nche = phi ? 2 * nch : nch, nre = zf ? 2 * nr : nr;
  const double c0e = phi ? 2.0 * s->central_channel + 0.5 : s->central_channel;
  const double dcole = phi ? 0.5 * s->dcol : s->dcol, drowe = zf ? 0.5 * s->drow : s->drow;
  double R = s->sid;
  double ds = dcole * R / s->sdd;
  double delta = nche + 1.75 - 2.0 * c0e;
  int b = nch - 1 - k, rr = nr - 1 - r;
  int be = phi ? 2 * b + sp : b, rre = zf ? 2 * rr + sz : rr;
  double beta = (be - c0e) * dcole / s->sdd;
  double ang = s->angle0 + v * s->dangle;
  double zs = s->z0 + v * s->dz;
  double theta = ang - beta;
  double sn = sin(theta), cs = cos(theta);
  double pstar = delta * ds - R * sin(beta);
  double t = sqrt(R * R - pstar * pstar);
  S[0] = pstar * sn + t * cs;
  S[1] = -pstar * cs + t * sn;
  S[2] = zs;
  double slope = (rre - (nre - 1) / 2.0) * drowe / s->sdd;
  U[0] = -cs; U[1] = -sn; U[2] = slope;
}

typedef struct { const wfbp_synth_scan* s; const wfbp_ellipsoid* e; int ne; float* out; } syn_args;
static void syn_body(void* a_, long i0, long i1) {
  syn_args* a = (syn_args*)a_;
  const wfbp_synth_scan* s = a->s;
  int nr = s->rows, nch = s->channels;
  for (long row = i0; row < i1; row++) {
    long v = row / nr;
    int r = (int)(row % nr);
    for (int k = 0; k < nch; k++) {
      double S[3], U[3];
      synth_ray(s, v, r, k, S, U);
      double p = chord_sum(a->e, a->ne, S, U);
      if (s->i0 > 0) {
        uint64_t idx = (uint64_t)row * nch + k;
        uint32_t rnd[4];
        philox4x32((uint32_t)idx, (uint32_t)(idx >> 32), 0u, 0u, (uint32_t)s->seed, (uint32_t)(s->seed >> 32), rnd);
        double n = poisson_draw(s->i0 * exp(-p), rnd);
        if (n < 1.0) n = 1.0;
        p = -log(n / s->i0);
      }
      a->out[row * nch + k] = (float)p;
    }
  }
}

ORC_EXPORT int orc_synth_project(const wfbp_synth_scan* s, const wfbp_ellipsoid* e, int ne, float* out) {
  if (!s || !out || (ne > 0 && !e)) return WFBP_ERR_INVALID_ARG;
  syn_args a = {s, e, ne, out};
  orc_parallel_for((long)s->n_readings * s->rows, 16, syn_body, &a);
  return WFBP_OK;
}

/* Voxelised phantom: mean attenuation over ss^3 sub-samples per voxel. */
typedef struct { const wfbp_ellipsoid* e; int ne; const ReconConfig* rp; const double* z; double dz; int ss; double* out; } vox_args;
static void vox_body(void* a_, long i0, long i1) {
  vox_args* a = (vox_args*)a_;
  int nx = (int)a->rp->nx, ny = (int)a->rp->ny, ss = a->ss;
  double vx = a->rp->recon_fov / nx, vy = a->rp->recon_fov / ny;
  for (long item = i0; item < i1; item++) {
    int s = (int)(item / ny), iy = (int)(item % ny);
    for (int ix = 0; ix < nx; ix++) {
      double xc = (ix - 0.5 * (nx - 1.0)) * vx + a->rp->x_origin, yc = (iy - 0.5 * (ny - 1.0)) * vy + a->rp->y_origin;
      double acc = 0.0;
      for (int sz = 0; sz < ss; sz++)
        for (int sy = 0; sy < ss; sy++)
          for (int sx = 0; sx < ss; sx++) {
            double px = xc + ((sx + 0.5) / ss - 0.5) * vx, py = yc + ((sy + 0.5) / ss - 0.5) * vy;
            double pz = a->z[s] + ((sz + 0.5) / ss - 0.5) * a->dz;
            for (int n = 0; n < a->ne; n++) {
              const wfbp_ellipsoid* e = &a->e[n];
              double cp = cos(e->phi), sp = sin(e->phi);
              double dx = px - e->cx, dy = py - e->cy, dzz = pz - e->cz;
              double lx = (dx * cp + dy * sp) / e->ax, ly = (-dx * sp + dy * cp) / e->ay, lz = dzz / e->az;
              if (lx * lx + ly * ly + lz * lz <= 1.0) acc += e->mu;
            }
          }
      a->out[((size_t)s * ny + iy) * nx + ix] = acc / (ss * ss * ss);
    }
  }
}
ORC_EXPORT void orc_voxelize(const wfbp_ellipsoid* e, int ne, const ReconConfig* rp, const double* z, int nz,
                             double dz, int ss, double* out) {
  vox_args a = {e, ne, rp, z, dz, ss, out};
  orc_parallel_for((long)nz * (long)rp->ny, 1, vox_body, &a);
}

/* ------------------------------------------------------------------------ */
/* flying focal spot (no counterpart in the reference's WFBP)               */
/* ------------------------------------------------------------------------ */
/* Readings cycle through the focal states of fct_icd's generate_ffs_offset
 * (applications/fct_icd/src/generate_system_matrix_ffs.cpp:242-290): with
 * phi and z FFS, state = reading % 4, phi bit = state & 1, z bit = state >> 1;
 * with one of them, state = reading % 2. A reading of phi state sp samples
 * the effective channels 2b + sp (fan angle offset by (sp - 1/2) dbeta/2), a
 * reading of z state sz the effective rows 2r + sz (half a row). The
 * effective detector has 2x channels / rows at half the spacing, central
 * channel 2 c0 + 1/2, and one effective view per G readings (G = number of
 * states), at the angle and table position of the group's first reading. */
static int ffs_groups(const CTGeometry* cg) { return (cg->ffs_phi ? 2 : 1) * (cg->ffs_z ? 2 : 1); }

ORC_EXPORT int orc_ffs_effective(const CTGeometry* in, CTGeometry* out) {
  *out = *in;
  int G = ffs_groups(in);
  if (in->total_number_of_projections % G || in->projections_per_rotation % G) return WFBP_ERR_INVALID_ARG;
  int fp = in->ffs_phi ? 2 : 1, fz = in->ffs_z ? 2 : 1;
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
  float cone_offset = ((float)(out->num_detector_rows - 1)) / 2.0f;
  out->theta_cone = 2.0f * (float)atan((double)(cone_offset * out->collimated_slice_width /
                                                out->distance_source_to_isocenter));
  out->acquisition_field_of_view =
      2.0f * out->distance_source_to_isocenter *
      (float)sin((double)((((float)out->num_detector_cols - 1.0f) / 2.0f) * out->detector_pixel_size_col *
                          (1.0f / out->distance_source_to_detector)));
  return WFBP_OK;
}

/* FP64 rebin of FFS readings onto the effective parallel grid: the fan
 * sample at fractional effective channel bidx and reading index
 * G v - beta/dtheta_reading is interpolated between the two effective
 * channels around bidx, each from its own focal state's readings (linear in
 * reading angle between that state's neighbouring readings). out:
 * [V/G][nr_eff][nch_eff]. */
typedef struct { const CTGeometry* cg; const CTGeometry* ce; const float* raw; double* out; long off; } rbf_args;
static void rbf_body(void* a_, long i0, long i1) {
  rbf_args* a = (rbf_args*)a_;
  const CTGeometry* cg = a->cg; const CTGeometry* ce = a->ce;
  const int G = ffs_groups(cg), phi = cg->ffs_phi, zf = cg->ffs_z;
  const int nch = (int)cg->num_detector_cols, nr = (int)cg->num_detector_rows;
  const int nche = (int)ce->num_detector_cols, nre = (int)ce->num_detector_rows, Ve = (int)ce->total_number_of_projections;
  const double dth = 2.0 * M_PI / (double)cg->projections_per_rotation;
  const double c0e = ce->detector_central_col, dcole = ce->detector_pixel_size_col, sdd = cg->distance_source_to_detector;
  for (long row = i0; row < i1; row++) {
    int v = (int)(row / nre), ie = (int)(row % nre);
    int zs = zf ? (ie & 1) : 0, iraw = zf ? ie >> 1 : ie, rraw = nr - 1 - iraw;
    for (int c = 0; c < nche; c++) {
      double p = ((double)c - c0e) * dcole;
      double beta = asin(p / sdd);
      double bidx = beta * sdd / dcole + c0e;
      double val = 0.0;
      if (!(bidx < 0 || bidx >= (double)nche || isnan(bidx))) {
        double fx = floor(bidx), ax = bidx - fx;
        double nf = (double)G * (v + a->off) - beta / dth;  /* whole-scan reading index */
        for (int t = 0; t < 2; t++) {
          long e = (long)fx + t;
          if (e < 0) e = 0;
          if (e > nche - 1) e = nche - 1;
          double we = t ? ax : 1.0 - ax;
          int sp = phi ? (int)(e & 1) : 0;
          int b = phi ? (int)(e >> 1) : (int)e;
          int rho = (G == 4) ? sp + 2 * zs : (phi ? sp : zs);
          double mf = (nf - rho) / G, m0 = floor(mf), ay = mf - m0;
          for (int u = 0; u < 2; u++) {
            long m = (long)m0 + u - a->off;
            if (m < 0) m = 0;
            if (m > Ve - 1) m = Ve - 1;
            double wy = u ? ay : 1.0 - ay;
            long n = (long)G * m + rho;
            val += we * wy * a->raw[((size_t)n * nr + rraw) * nch + (nch - 1 - b)];
          }
        }
      }
      a->out[row * nche + c] = val;
    }
  }
}
/* off: index of the first view (focal-state cycle) of raw within the whole scan */
ORC_EXPORT int orc_rebin_ffs_f64_off(const CTGeometry* cg, const float* raw, long off, double* out) {
  CTGeometry ce;
  int st = orc_ffs_effective(cg, &ce);
  if (st) return st;
  rbf_args a = {cg, &ce, raw, out, off};
  orc_parallel_for((long)ce.total_number_of_projections * (long)ce.num_detector_rows, 16, rbf_body, &a);
  return WFBP_OK;
}
ORC_EXPORT int orc_rebin_ffs_f64(const CTGeometry* cg, const float* raw, double* out) {
  return orc_rebin_ffs_f64_off(cg, raw, 0, out);
}

/* ------------------------------------------------------------------------ */
/* adjoints (FP64), the transposes of the forward loops above               */
/* ------------------------------------------------------------------------ */

/* thickening: g_native[n] += w_n / sum(w) * g_vol[r] */
ORC_EXPORT void orc_thicken_adjoint_f64(const ReconConfig* rp, const double* g_vol, const double* z_native, int nz,
                                        const double* z_req, int nzr, double* g_native) {
  size_t plane = rp->nx * rp->ny;
  memset(g_native, 0, sizeof(double) * plane * nz);
  for (int r = 0; r < nzr; r++) {
    double ws = 0.0;
    for (int i = 0; i < nz; i++) {
      double w = 1.0 - fabs(z_native[i] - z_req[r]) / rp->slice_thickness;
      if (w > 0.0) ws += w;
    }
    if (!(ws > 0.0)) continue;
    for (int i = 0; i < nz; i++) {
      double w = 1.0 - fabs(z_native[i] - z_req[r]) / rp->slice_thickness;
      if (w <= 0.0) continue;
      for (size_t px = 0; px < plane; px++) g_native[(size_t)i * plane + px] += w / ws * g_vol[(size_t)r * plane + px];
    }
  }
}

/* backprojection: for every voxel and theta~, the weights W_k/sum(W) of the
 * forward's normalised average, times dtheta, scatter the voxel's gradient
 * through each view's bilinear weights. Views are owned by threads (each
 * thread loops over all voxels for its views), so no two threads write the
 * same sample. g_filtered: [V][nr][nch]. */
typedef struct { bp64_geo g; const double* gv; const double* tube; const double* table; const double* slices; int nz;
                 double* gf; } bpa_args;
static void bpa_body(void* a_, long t0, long t1) {
  bpa_args* a = (bpa_args*)a_;
  const bp64_geo* g = &a->g;
  size_t nch = (size_t)g->nch, nr = (size_t)g->nr;
  double* Wk = (double*)malloc(sizeof(double) * g->K);
  double* pidx = (double*)malloc(sizeof(double) * g->K);
  double* qidx = (double*)malloc(sizeof(double) * g->K);
  for (long t = t0; t < t1; t++) { /* theta~ */
    for (int s = 0; s < a->nz; s++) {
      double z = a->slices[s];
      for (int iy = 0; iy < g->ny; iy++) {
        double y = (iy - 0.5 * (g->ny - 1.0)) * g->fov / g->ny + g->y0;
        for (int ix = 0; ix < g->nx; ix++) {
          double x = (ix - 0.5 * (g->nx - 1.0)) * g->fov / g->nx + g->x0;
          if (x * x + y * y > g->afov_half2) continue;
          double gvox = a->gv[((size_t)s * g->ny + iy) * g->nx + ix];
          if (gvox == 0.0) continue;
          double nf = 0.0;
          for (int k = 0; k < g->K; k++) {
            Wk[k] = 0.0;
            int j = (int)t + k * g->P2;
            double zt = a->table[j];
            if (fabs(zt - z) > g->z_rot) continue;
            double th = a->tube[j], sn = sin(th), cs = cos(th);
            double p_hat = x * sn - y * cs;
            double l_hat = sqrt(g->sid2 - p_hat * p_hat) - x * cs - y * sn;
            double q_hat = (z - zt + g->zr2pi * asin(p_hat / g->sid)) / (l_hat * g->tanc);
            if (q_hat > 1.0 || q_hat < -1.0) continue;
            double pi_ = (g->nch + 1.75) - (p_hat * g->pixel_scale + g->c0);
            double qi = 0.5 * (q_hat + 1.0) * (g->nr - 1.0);
            if (floor(pi_) < 0 || floor(qi) < 0) continue;
            if (ceil(pi_) >= g->nch - 1 || ceil(qi) >= g->nr - 1) continue;
            Wk[k] = w_f64(q_hat);
            pidx[k] = pi_;
            qidx[k] = qi;
            nf += Wk[k];
          }
          if (!(nf > 0.0)) continue;
          for (int k = 0; k < g->K; k++) {
            if (Wk[k] == 0.0) continue;
            int j = (int)t + k * g->P2;
            double c = gvox * g->dtheta * Wk[k] / nf;
            double pf = floor(pidx[k]), qf = floor(qidx[k]);
            double wp = pidx[k] - pf, wq = qidx[k] - qf;
            size_t lo = (size_t)pf + (size_t)qf * nch + (size_t)j * nr * nch, hi = lo + nch;
            a->gf[lo] += c * (1 - wq) * (1 - wp);
            a->gf[lo + 1] += c * (1 - wq) * wp;
            a->gf[hi] += c * wq * (1 - wp);
            a->gf[hi + 1] += c * wq * wp;
          }
        }
      }
    }
  }
  free(Wk); free(pidx); free(qidx);
}
ORC_EXPORT void orc_backproject_adjoint_f64(const CTGeometry* cg, const ReconConfig* rp, const double* g_native,
                                            const double* tube, const double* table, const double* slices, int nz,
                                            double* g_filtered) {
  bpa_args a;
  bp64_geo_init(&a.g, cg, rp, table);
  a.gv = g_native; a.tube = tube; a.table = table; a.slices = slices; a.nz = nz; a.gf = g_filtered;
  memset(g_filtered, 0, sizeof(double) * cg->total_number_of_projections * cg->num_detector_rows * cg->num_detector_cols);
  /* threads own theta~ values: views theta~ + k P/2 belong to exactly one thread */
  orc_parallel_for(a.g.P2, 4, bpa_body, &a);
}

/* tap gradient: dL/dh[d] = sum_rows sum_n g[n] (x[n-d] + x[n+d]) (d > 0), sum g[n] x[n] (d = 0) */
ORC_EXPORT void orc_taps_gradient_f64(int nch, long rows, const double* g, const double* x, int ntaps, double* out) {
  for (int d = 0; d < ntaps; d++) {
    double acc = 0.0;
    for (long r = 0; r < rows; r++) {
      const double* gr = g + r * nch;
      const double* xr = x + r * nch;
      for (int n = 0; n < nch; n++) {
        if (d == 0) acc += gr[n] * xr[n];
        else {
          if (n - d >= 0) acc += gr[n] * xr[n - d];
          if (n + d < nch) acc += gr[n] * xr[n + d];
        }
      }
    }
    out[d] = acc;
  }
}

/* rebin (FP64, exact weights, clamp addressing): transpose of rb64_body */
typedef struct { const CTGeometry* cg; const double* gx; double* graw; } rba_args;
static void rba_body(void* a_, long i0, long i1) {
  rba_args* a = (rba_args*)a_;
  const CTGeometry* cg = a->cg;
  int nr = (int)cg->num_detector_rows, nch = (int)cg->num_detector_cols, V = (int)cg->total_number_of_projections;
  double dth = 2.0 * M_PI / (double)cg->projections_per_rotation;
  double c0 = cg->detector_central_col, dcol = cg->detector_pixel_size_col, sdd = cg->distance_source_to_detector;
  for (long i = i0; i < i1; i++) { /* rows are independent: raw row nr-1-i */
    int r_raw = nr - 1 - (int)i;
    for (int v = 0; v < V; v++) {
      for (int c = 0; c < nch; c++) {
        double gval = a->gx[((size_t)v * nr + i) * nch + c];
        if (gval == 0.0) continue;
        double p = ((double)c - c0) * dcol;
        double beta = asin(p / sdd);
        double bidx = beta * sdd / dcol + c0;
        if (bidx < 0 || bidx >= (double)nch || isnan(bidx)) continue;
        double aidx = (double)v - beta / dth;
        double fx = floor(bidx), fy = floor(aidx);
        double ax = bidx - fx, ay = aidx - fy;
        long xs[2] = {(long)fx, (long)fx + 1}, ys[2] = {(long)fy, (long)fy + 1};
        double wx[2] = {1 - ax, ax}, wy[2] = {1 - ay, ay};
        for (int u = 0; u < 2; u++) {
          long xx = xs[u] < 0 ? 0 : (xs[u] > nch - 1 ? nch - 1 : xs[u]);
          for (int t = 0; t < 2; t++) {
            long yy = ys[t] < 0 ? 0 : (ys[t] > V - 1 ? V - 1 : ys[t]);
            a->graw[((size_t)yy * nr + r_raw) * nch + (nch - 1 - xx)] += gval * wx[u] * wy[t];
          }
        }
      }
    }
  }
}
ORC_EXPORT void orc_rebin_adjoint_f64(const CTGeometry* cg, const double* g_rebinned, double* g_raw) {
  rba_args a = {cg, g_rebinned, g_raw};
  memset(g_raw, 0, sizeof(double) * cg->total_number_of_projections * cg->num_detector_rows * cg->num_detector_cols);
  orc_parallel_for((long)cg->num_detector_rows, 1, rba_body, &a);
}

/* ------------------------------------------------------------------------ */
/* adaptive filtration of the raw readings (FP64)                            */
/* ------------------------------------------------------------------------ */
/* fct_wfbp parses ReconConfig.adaptive_filtration_s (parse_config.cpp:57)
 * but never applies it (README: "Need to add adaptive filtration back into
 * the toolbox"). The product defines it as attenuation-adaptive smoothing of
 * the raw line integrals, after Kachelriess, Watzke and Kalender, Med. Phys.
 * 28 (2001) 475-490: with s = min(s, 1) > 0 and p_max the largest line
 * integral of a reading, each sample p of the reading becomes
 * p + w (pbar - p), pbar = (p[c-1] + 2 p[c] + p[c+1]) / 4 along its detector
 * row (edge channels repeated), w = clamp((p - p_t) / (p_max - p_t), 0, 1),
 * p_t = (1 - s) p_max: the most attenuated (photon-starved) rays are
 * smoothed most, rays below p_t pass unchanged. s <= 0, or a reading with
 * p_max <= 0, leaves the samples unchanged. This is the FP64 statement of
 * that definition; out: [readings][rows][channels]. */
typedef struct { const float* raw; int nr, nch; double s; double* out; } af_args;
static void af_body(void* a_, long i0, long i1) {
  af_args* a = (af_args*)a_;
  const long fr = (long)a->nr * a->nch;
  const double s = a->s < 1.0 ? a->s : 1.0;
  for (long n = i0; n < i1; n++) {
    const float* x = a->raw + n * fr;
    double* y = a->out + n * fr;
    double pmax = -INFINITY;
    for (long k = 0; k < fr; k++)
      if (x[k] > pmax) pmax = x[k];
    if (!(s > 0.0) || !(pmax > 0.0)) {
      for (long k = 0; k < fr; k++) y[k] = x[k];
      continue;
    }
    const double pt = (1.0 - s) * pmax;
    for (int r = 0; r < a->nr; r++)
      for (int c = 0; c < a->nch; c++) {
        const float* row = x + (long)r * a->nch;
        const double p = row[c];
        const double pb = 0.25 * ((double)row[c > 0 ? c - 1 : 0] + 2.0 * p + (double)row[c < a->nch - 1 ? c + 1 : c]);
        double w = (p - pt) / (pmax - pt);
        w = w < 0.0 ? 0.0 : (w > 1.0 ? 1.0 : w);
        y[(long)r * a->nch + c] = p + w * (pb - p);
      }
  }
}
ORC_EXPORT void orc_adaptive_filter_f64(const float* raw, long n_readings, int nr, int nch, double s, double* out) {
  af_args a = {raw, nr, nch, s, out};
  orc_parallel_for(n_readings, 4, af_body, &a);
}
