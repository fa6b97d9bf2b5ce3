// Rebin sample arithmetic shared by the forward rebin (k_stages.cu) and the
// kernels that recompute or transpose it (k_adjoint.cu).
#pragma once

#include "wfbp_internal.h"

// One output sample (v, i, c) of the reference's rebin of row sheet i
// (cuda_kernels.cuh:11-39) read straight from the raw [reading][row][channel]
// frames: the host reshape of ReconstructionMachine.cu:153-162 is folded into
// the index math (sheet row i <- raw row nr-1-i, sheet column b <- raw
// channel nch-1-b). The bilinear sample follows the texture unit's linear
// filter with clamp addressing and texel centres at +0.5 (RM.cu:176-180).
// voff: index of the first view within the whole scan. The sample angle is
// the whole scan's index angle (v + voff) 2 pi / P, so a window of a scan
// rebins exactly like the whole scan; texel rows are then taken relative to
// the window (and clamped to it).
// The part of a sample that depends on the view and the output channel only
// (not on the detector row): the clamped texel views and raw channels and the
// two fractional weights. raw0/raw1 point at the two views' last raw row
// (sheet row 0); sheet row i is nch floats earlier per row.
struct RebinTaps {
  const float* raw0;
  const float* raw1;
  int c0, c1;  // raw channels of the two texel columns
  float ax, ay;
  bool ok;     // false: the fan sample is outside the detector (bidx NaN), value 0
};

// The channel part of rebin_taps: the clamped raw channels of the two texel
// columns, the channel weight and whether the fan sample lies on the detector.
struct RebinTapsX {
  int c0, c1;
  float ax;
  bool ok;
};
__device__ __forceinline__ RebinTapsX rebin_taps_x(int nch, float bidx, int q8) {
  RebinTapsX t;
  t.ok = !isnan(bidx);
  float xb = (bidx + 0.5f) - 0.5f;
  float fx = floorf(xb);
  float ax = xb - fx;
  if (q8) ax = rintf(ax * 256.0f) * (1.0f / 256.0f);
  int x0 = t.ok ? (int)fx : 0;
  int x1 = min(max(x0 + 1, 0), nch - 1);
  x0 = min(max(x0, 0), nch - 1);
  t.c0 = nch - 1 - x0;
  t.c1 = nch - 1 - x1;
  t.ax = ax;
  return t;
}
// The reading part: the clamped window-relative readings of the two texel
// rows and the reading weight of output view v.
struct RebinTapsY {
  int y0, y1;
  float ay;
};
__device__ __forceinline__ RebinTapsY rebin_taps_y(int V, float beta, int v, float dth, int q8, int voff) {
  RebinTapsY t;
  float theta = (float)(v + voff) * dth;
  float alpha = theta - beta;
  float aidx = alpha / dth;
  float yb = (aidx + 0.5f) - 0.5f;
  float fy = floorf(yb);
  float ay = yb - fy;
  if (q8) ay = rintf(ay * 256.0f) * (1.0f / 256.0f);
  int y0 = (int)fy - voff;
  t.y1 = min(max(y0 + 1, 0), V - 1);
  t.y0 = min(max(y0, 0), V - 1);
  t.ay = ay;
  return t;
}

__device__ __forceinline__ RebinTaps rebin_taps(const float* __restrict__ raw, size_t view_stride, int V, int nr,
                                                int nch, float bidx, float beta, int v, float dth, int q8, int voff) {
  const RebinTapsX x = rebin_taps_x(nch, bidx, q8);
  const RebinTapsY y = rebin_taps_y(V, beta, v, dth, q8, voff);
  RebinTaps t;
  t.ok = x.ok;
  const float* last = raw + (size_t)(nr - 1) * nch;
  t.raw0 = last + (size_t)y.y0 * view_stride;
  t.raw1 = last + (size_t)y.y1 * view_stride;
  t.c0 = x.c0;
  t.c1 = x.c1;
  t.ax = x.ax;
  t.ay = y.ay;
  return t;
}

// rebin_taps with FP64 sample coordinates (the mixed form): the source
// channel index bidx and beta / dtheta come from the context's FP64
// per-channel table, the fractional view index (v + voff) - beta / dtheta and
// both fractional weights are formed in double (the FP64 oracle's
// arithmetic, oracle/wfbp_oracle.c rb64_body) and only the weights rounded to
// FP32. Exact weights (no 8-bit texture fractions).
__device__ __forceinline__ RebinTapsX rebin_taps64_x(int nch, double2 ch) {
  RebinTapsX t;
  t.ok = !isnan(ch.x);
  const double fx = t.ok ? floor(ch.x) : 0.0;
  int x0 = (int)fx;
  int x1 = min(max(x0 + 1, 0), nch - 1);
  x0 = min(max(x0, 0), nch - 1);
  t.c0 = nch - 1 - x0;
  t.c1 = nch - 1 - x1;
  t.ax = t.ok ? (float)(ch.x - fx) : 0.0f;
  return t;
}
__device__ __forceinline__ RebinTapsY rebin_taps64_y(int V, double2 ch, int v, int voff) {
  RebinTapsY t;
  const double aidx = (double)(v + voff) - ch.y;
  const double fy = floor(aidx);
  int y0 = (int)fy - voff;
  t.y1 = min(max(y0 + 1, 0), V - 1);
  t.y0 = min(max(y0, 0), V - 1);
  t.ay = (float)(aidx - fy);
  return t;
}
__device__ __forceinline__ RebinTaps rebin_taps64(const float* __restrict__ raw, size_t view_stride, int V, int nr,
                                                  int nch, double2 ch, int v, int voff) {
  const RebinTapsX x = rebin_taps64_x(nch, ch);
  const RebinTapsY y = rebin_taps64_y(V, ch, v, voff);
  RebinTaps t;
  t.ok = x.ok;
  const float* last = raw + (size_t)(nr - 1) * nch;
  t.raw0 = last + (size_t)y.y0 * view_stride;
  t.raw1 = last + (size_t)y.y1 * view_stride;
  t.c0 = x.c0;
  t.c1 = x.c1;
  t.ax = x.ax;
  t.ay = y.ay;
  return t;
}

// The bilinear texel blend of rebin_kernel's linear texture filter.
__device__ __forceinline__ float rebin_bilinear(float t00, float t10, float t01, float t11, float ax, float ay) {
  return (1.0f - ax) * (1.0f - ay) * t00 + ax * (1.0f - ay) * t10 + (1.0f - ax) * ay * t01 + ax * ay * t11;
}

// The bilinear sample of sheet row i (raw row nr-1-i) at the taps.
__device__ __forceinline__ float rebin_taps_sample(const RebinTaps& t, int i, int nch) {
  if (!t.ok) return 0.0f;
  const float* r0 = t.raw0 - (size_t)i * nch;
  const float* r1 = t.raw1 - (size_t)i * nch;
  float t00 = __ldg(r0 + t.c0), t10 = __ldg(r0 + t.c1);
  float t01 = __ldg(r1 + t.c0), t11 = __ldg(r1 + t.c1);
  return rebin_bilinear(t00, t10, t01, t11, t.ax, t.ay);
}

// Flying focal spot (no counterpart in the reference's WFBP): readings cycle
// through G focal states (the state order of fct_icd's generate_ffs_offset,
// applications/fct_icd/src/generate_system_matrix_ffs.cpp:242-290: phi bit =
// state & 1, z bit = state >> 1 when both are on). A reading of phi state sp
// samples effective channels 2b + sp, of z state sz effective rows 2r + sz.
// The effective fan sample at fractional effective channel bidx is
// interpolated between the two effective channels around it, each from its
// own state's readings, linearly in reading angle between that state's
// neighbouring readings (so no reading is assigned another reading's angle).
__device__ __forceinline__ float rebin_sample_ffs(const float* __restrict__ raw, const RebinParams& p, float bidx,
                                                  float beta, int v, int ie) {
  if (isnan(bidx)) return 0.0f;
  const int zs = p.zf ? (ie & 1) : 0, iraw = p.zf ? (ie >> 1) : ie;
  const float* rawrow = raw + (size_t)(p.nr_raw - 1 - iraw) * p.nch_raw;
  const size_t vs = (size_t)p.nr_raw * p.nch_raw;
  const float nf = ((float)(p.G * (v + p.voff)) * p.dth - beta) / p.dth;  // fractional reading index (whole scan)
  const float fx = floorf(bidx);
  float ax = bidx - fx;
  if (p.q8) ax = rintf(ax * 256.0f) * (1.0f / 256.0f);
  float val = 0.0f;
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int e = min(max((int)fx + t, 0), p.nch - 1);
    const float we = t ? ax : 1.0f - ax;
    const int sp = p.phi ? (e & 1) : 0, b = p.phi ? (e >> 1) : e;
    const int rho = (p.G == 4) ? sp + 2 * zs : (p.phi ? sp : zs);
    const float mf = (nf - (float)rho) / (float)p.G, m0 = floorf(mf);
    float ay = mf - m0;
    if (p.q8) ay = rintf(ay * 256.0f) * (1.0f / 256.0f);
    const int ma = min(max((int)m0 - p.voff, 0), p.V - 1), mb = min(max((int)m0 + 1 - p.voff, 0), p.V - 1);
    const float t0 = __ldg(rawrow + (size_t)(p.G * ma + rho) * vs + (p.nch_raw - 1 - b));
    const float t1 = __ldg(rawrow + (size_t)(p.G * mb + rho) * vs + (p.nch_raw - 1 - b));
    val += we * ((1.0f - ay) * t0 + ay * t1);
  }
  return val;
}

// rebin_sample_ffs split like RebinTaps: for output channel (bidx, beta) of
// view v, the two focal-state row parities (zs) each have two effective
// channel taps (weight we, reading weight ay, the two readings' offsets from
// the raw row); only the raw row depends on the detector row. The sum runs
// in rebin_sample_ffs's order.
struct RebinTapsFfs {
  float we[2][2], ay[2][2];
  size_t oa[2][2], ob[2][2];
  bool ok;
};

__device__ __forceinline__ RebinTapsFfs rebin_taps_ffs(const RebinParams& p, float bidx, float beta, int v) {
  RebinTapsFfs T;
  T.ok = !isnan(bidx);
  const size_t vs = (size_t)p.nr_raw * p.nch_raw;
  const float nf = ((float)(p.G * (v + p.voff)) * p.dth - beta) / p.dth;
  const float fx = T.ok ? floorf(bidx) : 0.0f;
  float ax = T.ok ? bidx - fx : 0.0f;
  if (p.q8) ax = rintf(ax * 256.0f) * (1.0f / 256.0f);
#pragma unroll
  for (int zs = 0; zs < 2; zs++)
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const int e = min(max((int)fx + t, 0), p.nch - 1);
      T.we[zs][t] = t ? ax : 1.0f - ax;
      const int sp = p.phi ? (e & 1) : 0, b = p.phi ? (e >> 1) : e;
      const int z = p.zf ? zs : 0;
      const int rho = (p.G == 4) ? sp + 2 * z : (p.phi ? sp : z);
      const float mf = (nf - (float)rho) / (float)p.G, m0 = floorf(mf);
      float ay = mf - m0;
      if (p.q8) ay = rintf(ay * 256.0f) * (1.0f / 256.0f);
      T.ay[zs][t] = ay;
      const int ma = min(max((int)m0 - p.voff, 0), p.V - 1), mb = min(max((int)m0 + 1 - p.voff, 0), p.V - 1);
      T.oa[zs][t] = (size_t)(p.G * ma + rho) * vs + (size_t)(p.nch_raw - 1 - b);
      T.ob[zs][t] = (size_t)(p.G * mb + rho) * vs + (size_t)(p.nch_raw - 1 - b);
    }
  return T;
}

// rebin_taps_ffs with FP64 sample coordinates (the mixed form; exact
// weights): reading index G (v + voff) - beta / dtheta_reading and the
// per-state fractional readings in double, as the FP64 oracle's rbf_body.
__device__ __forceinline__ RebinTapsFfs rebin_taps_ffs64(const RebinParams& p, double2 ch, int v) {
  RebinTapsFfs T;
  T.ok = !isnan(ch.x);
  const size_t vs = (size_t)p.nr_raw * p.nch_raw;
  const double nf = (double)(p.G * (v + p.voff)) - ch.y;
  const double fx = T.ok ? floor(ch.x) : 0.0;
  const float ax = T.ok ? (float)(ch.x - fx) : 0.0f;
#pragma unroll
  for (int zs = 0; zs < 2; zs++)
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const int e = min(max((int)fx + t, 0), p.nch - 1);
      T.we[zs][t] = t ? ax : 1.0f - ax;
      const int sp = p.phi ? (e & 1) : 0, b = p.phi ? (e >> 1) : e;
      const int z = p.zf ? zs : 0;
      const int rho = (p.G == 4) ? sp + 2 * z : (p.phi ? sp : z);
      const double mf = (nf - (double)rho) / (double)p.G, m0 = floor(mf);
      T.ay[zs][t] = (float)(mf - m0);
      const int ma = min(max((int)m0 - p.voff, 0), p.V - 1), mb = min(max((int)m0 + 1 - p.voff, 0), p.V - 1);
      T.oa[zs][t] = (size_t)(p.G * ma + rho) * vs + (size_t)(p.nch_raw - 1 - b);
      T.ob[zs][t] = (size_t)(p.G * mb + rho) * vs + (size_t)(p.nch_raw - 1 - b);
    }
  return T;
}

// Sample of effective row ie at the taps (rebin_sample_ffs's value).
__device__ __forceinline__ float rebin_taps_ffs_sample(const float* __restrict__ raw, const RebinParams& p,
                                                       const RebinTapsFfs& T, int ie) {
  if (!T.ok) return 0.0f;
  const int zs = p.zf ? (ie & 1) : 0, iraw = p.zf ? (ie >> 1) : ie;
  const float* rawrow = raw + (size_t)(p.nr_raw - 1 - iraw) * p.nch_raw;
  float val = 0.0f;
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const float we = zs ? T.we[1][t] : T.we[0][t];
    const float ay = zs ? T.ay[1][t] : T.ay[0][t];
    const float t0 = __ldg(rawrow + (zs ? T.oa[1][t] : T.oa[0][t]));
    const float t1 = __ldg(rawrow + (zs ? T.ob[1][t] : T.ob[0][t]));
    val += we * ((1.0f - ay) * t0 + ay * t1);
  }
  return val;
}

// One rebinned sample of output view v, row i (flipped row-sheet index),
// output channel with table entries (bidx, beta).
__device__ __forceinline__ float wfbp_rebin_sample(const float* __restrict__ raw, const RebinParams& p, float bidx, float beta,
                                           int v, int i) {
  if (p.G > 1) return rebin_sample_ffs(raw, p, bidx, beta, v, i);
  const RebinTaps t = rebin_taps(raw, (size_t)p.nr * p.nch, p.V, p.nr, p.nch, bidx, beta, v, p.dth, p.q8, p.voff);
  return rebin_taps_sample(t, i, p.nch);
}

// The taps of output channel (bidx, beta) of view v without a flying focal
// spot (p.G == 1).
__device__ __forceinline__ RebinTaps wfbp_rebin_taps(const float* __restrict__ raw, const RebinParams& p, float bidx,
                                                     float beta, int v) {
  return rebin_taps(raw, (size_t)p.nr * p.nch, p.V, p.nr, p.nch, bidx, beta, v, p.dth, p.q8, p.voff);
}

