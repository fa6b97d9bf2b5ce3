// Rebin, FP32 Toeplitz filter, thickening and table kernels (sm_100a).
#include "wfbp_internal.h"

#include <algorithm>

#include <math.h>

// ---------------------------------------------------------------------------
// tables
// ---------------------------------------------------------------------------

// Per-view sin/cos of the tube angle, evaluated with the accurate sinf/cosf
// the reference calls per voxel (cuda_kernels.cuh:235-238).
__global__ void k_view_tables(const float* __restrict__ tube, const float* __restrict__ table,
                              float2* __restrict__ sc, float* __restrict__ z, int V) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= V) return;
  float th = tube[j];
  sc[j] = make_float2(sinf(th), cosf(th));
  z[j] = table[j];
}

cudaError_t launch_view_tables(const float* d_tube, const float* d_table, float2* d_sc, float* d_z, int V,
                               cudaStream_t s) {
  k_view_tables<<<(V + 255) / 256, 256, 0, s>>>(d_tube, d_table, d_sc, d_z, V);
  return cudaGetLastError();
}

// Per-channel rebin geometry of rebin_kernel (cuda_kernels.cuh:17-22): the
// fan angle beta of output channel c and the source channel index; NaN marks
// channels the reference writes as zero (cuda_kernels.cuh:32-34).
__global__ void k_rebin_tables(float* __restrict__ beta_t, float* __restrict__ bidx_t, int nch, float c0,
                               float dcol, float sdd) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nch) return;
  float p = ((float)c - c0) * dcol;
  float beta = asinf(p / sdd);
  float bidx = (beta * sdd / dcol) + c0;
  if (bidx < 0 || bidx >= (float)nch || isnan(bidx)) bidx = __int_as_float(0x7fc00000);
  beta_t[c] = beta;
  bidx_t[c] = bidx;
}

cudaError_t launch_rebin_tables(float* d_beta, float* d_bidx, int nch, float c0, float dcol, float sdd,
                                cudaStream_t s) {
  k_rebin_tables<<<(nch + 127) / 128, 128, 0, s>>>(d_beta, d_bidx, nch, c0, dcol, sdd);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// rebin
// ---------------------------------------------------------------------------
//
#include "rebin_sample.cuh"

// A sample's view and channel geometry does not depend on the detector row
// (with a flying focal spot: only through the row's focal state, two tap
// sets): one thread per (view, output channel) computes it once
// (wfbp_rebin_taps / rebin_taps_ffs) and writes the channel's samples of every
// row, consecutive threads on consecutive channels (coalesced loads and
// stores). Same arithmetic per sample as rebin_sample / rebin_sample_ffs.
constexpr int RBR_CH = 128;

template <bool FFS>
__global__ void __launch_bounds__(RBR_CH)
k_rebin_f32_rows(const float* __restrict__ raw, float* __restrict__ out, const float* __restrict__ beta_t,
                 const float* __restrict__ bidx_t, RebinParams p, int vb) {
  const int v = vb + blockIdx.y;
  const int c = blockIdx.x * RBR_CH + threadIdx.x;
  if (c >= p.nch) return;
  float* o = out + (size_t)v * p.nr * p.nch + c;
  if constexpr (FFS) {
    const RebinTapsFfs T = rebin_taps_ffs(p, __ldg(bidx_t + c), __ldg(beta_t + c), v);
#pragma unroll 4
    for (int i = 0; i < p.nr; i++) o[(size_t)i * p.nch] = rebin_taps_ffs_sample(raw, p, T, i);
  } else {
    const RebinTaps t = wfbp_rebin_taps(raw, p, __ldg(bidx_t + c), __ldg(beta_t + c), v);
#pragma unroll 4
    for (int i = 0; i < p.nr; i++) o[(size_t)i * p.nch] = rebin_taps_sample(t, i, p.nch);
  }
}

namespace {
// The view-chunk kernels serve scans without a flying focal spot whose raw
// frames fit 31-bit element offsets; longer ones (over 2^31 samples) take
// the per-view kernels k_rebin_f32_rows / k_rebin_split_rows.
bool use_vchunk_rebin(const RebinParams& p) { return p.G == 1 && (long long)p.V * p.nr * p.nch < (1ll << 31); }
}  // namespace

template <bool SPLIT, bool F64>
__global__ void k_rebin_vchunk(const float* __restrict__ raw, float* __restrict__ out, __half* __restrict__ a_hi,
                               __half* __restrict__ a_lo, unsigned* __restrict__ rowmax,
                               const float* __restrict__ beta_t, const float* __restrict__ bidx_t,
                               const double2* __restrict__ chan64, RebinParams p, int kp, int nrv, int vb, int ve);

cudaError_t launch_rebin_f32(const float* raw, float* out, const float* d_beta, const float* d_bidx,
                             const RebinParams& p, cudaStream_t s, int vb, int ve) {
  if (ve < 0) ve = p.V;
  if (vb < 0 || vb >= ve || ve > p.V) return cudaErrorInvalidValue;
  if (use_vchunk_rebin(p)) {
    const dim3 g((unsigned)((p.nch + RV_CW - 1) / RV_CW), (unsigned)((ve - vb + RV_NY - 1) / RV_NY));
    k_rebin_vchunk<false, false><<<g, RV_CW, 0, s>>>(raw, out, nullptr, nullptr, nullptr, d_beta, d_bidx, nullptr, p,
                                                      0, 0, vb, ve);
    return cudaGetLastError();
  }
  dim3 g((unsigned)((p.nch + RBR_CH - 1) / RBR_CH), (unsigned)(ve - vb));
  if (p.G == 1)
    k_rebin_f32_rows<false><<<g, RBR_CH, 0, s>>>(raw, out, d_beta, d_bidx, p, vb);
  else
    k_rebin_f32_rows<true><<<g, RBR_CH, 0, s>>>(raw, out, d_beta, d_bidx, p, vb);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FP32 Toeplitz filter
// ---------------------------------------------------------------------------
//
// The reference filters each zero-padded row with cuFFT (R2C, multiply by the
// spectrum of the fftshifted taps and 1/N, C2R; ReconstructionMachine.cu:
// 206-290, cuda_kernels.cuh:41-58). Because the zero padding is at least
// nch-1 on each side, the data window of that circular convolution equals the
// linear convolution y[n] = sum_k h[|n-k|] x[k] over the nch channels: a
// [rows x nch] x [nch x nch] product with a symmetric Toeplitz matrix. This
// kernel evaluates it in FP32 on the CUDA cores: 128x128 output tiles, 8 rows
// x 8 consecutive columns per thread. The Toeplitz operand comes from a
// shared-memory tap line htab[d + nch] = h[|d|] (zero past the ends): for
// consecutive k a thread's 8 operand values are a window sliding down the
// line by one, so each k step loads one new tap. Rows are processed in pairs
// with the packed FP32x2 FMA; every output still accumulates its products in
// k order, one rounding per FMA.
constexpr int TF_BM = 128, TF_BN = 128, TF_BK = 16;

// TR = true writes the backprojection layout Y_T[view][channel][row] with
// rows padded to nrp (row m = view * nr + row).
template <bool TR>
__global__ void __launch_bounds__(256)
k_toeplitz_f32(const float* __restrict__ X, float* __restrict__ Y, const float* __restrict__ taps, long M,
               int nch, int nr, int nrp) {
  extern __shared__ float smem[];
  float* As = smem;                          // [TF_BK][TF_BM + 4]
  // tap line htab[d + nch + TF_BK] = h[|d|] for -nch - TF_BK <= d <= nch + TF_BN, 0 where |d| >= nch:
  // the last k block runs up to TF_BK - 1 past nch (zero rows of A) and the
  // last column block up to TF_BN - 1 past nch (columns that are not stored)
  float* htab = smem + TF_BK * (TF_BM + 4);
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const long m0 = (long)blockIdx.x * TF_BM;
  const int n0 = blockIdx.y * TF_BN;
  for (int d = tid; d < 2 * nch + TF_BN + TF_BK + 1; d += 256) {
    int a = d - nch - TF_BK;
    a = a < 0 ? -a : a;
    htab[d] = a < nch ? taps[a] : 0.0f;
  }
  float2 acc[4][8];  // acc[i][j] = (row 2i, row 2i+1) of column j
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = make_float2(0.0f, 0.0f);

  // thread columns n0 + 8 tx + j; operand h[|n - k|] = htab[n - k + nch + TF_BK]
  const int hb = n0 + 8 * tx + nch + TF_BK;
  for (int k0 = 0; k0 < nch; k0 += TF_BK) {
    __syncthreads();
    // A tile: 128 rows x 16 k, stored k-major
    for (int e = tid; e < TF_BM * TF_BK; e += 256) {
      int mm = e / TF_BK, kk = e % TF_BK;
      long m = m0 + mm;
      int k = k0 + kk;
      As[kk * (TF_BM + 4) + mm] = (m < M && k < nch) ? X[m * nch + k] : 0.0f;
    }
    __syncthreads();
    // operand window for k = k0: b[j] = htab[hb - k0 + j]
    float b[TF_BK + 8];
#pragma unroll
    for (int j = 0; j < 8; j++) b[TF_BK + j] = htab[hb - k0 + j];
#pragma unroll
    for (int kk = 0; kk < TF_BK; kk++) {
      // window for k0 + kk is b[TF_BK - kk .. TF_BK - kk + 7]
      if (kk > 0) b[TF_BK - kk] = htab[hb - k0 - kk];
      const float4 a0 = *reinterpret_cast<const float4*>(&As[kk * (TF_BM + 4) + ty * 8]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[kk * (TF_BM + 4) + ty * 8 + 4]);
      const float2 ap[4] = {make_float2(a0.x, a0.y), make_float2(a0.z, a0.w), make_float2(a1.x, a1.y),
                            make_float2(a1.z, a1.w)};
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const float bj = b[TF_BK - kk + j];
        const float2 bb = make_float2(bj, bj);
#pragma unroll
        for (int i = 0; i < 4; i++) acc[i][j] = __ffma2_rn(ap[i], bb, acc[i][j]);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    long m = m0 + ty * 8 + i;
    if (m >= M) continue;
    const long v = m / nr, row = m % nr;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int n = n0 + 8 * tx + j;
      const float val = (i & 1) ? acc[i >> 1][j].y : acc[i >> 1][j].x;
      if (n < nch) {
        if (TR)
          Y[((size_t)v * nch + n) * nrp + row] = val;
        else
          Y[m * nch + n] = val;
      }
    }
  }
}

template <bool TR>
cudaError_t launch_toeplitz_f32(const float* x, float* y, const float* d_taps, long rows, int nch, int nr, int nrp,
                                cudaStream_t s) {
  size_t smem = sizeof(float) * (TF_BK * (TF_BM + 4) + 2 * nch + TF_BN + TF_BK + 1);
  if (smem > 64 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_toeplitz_f32<TR>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((rows + TF_BM - 1) / TF_BM), (unsigned)((nch + TF_BN - 1) / TF_BN));
  k_toeplitz_f32<TR><<<grid, 256, smem, s>>>(x, y, d_taps, rows, nch, nr, nrp);
  return cudaGetLastError();
}

cudaError_t launch_filter_f32(const float* x, float* y, const float* d_taps, long rows, int nch, cudaStream_t s) {
  return launch_toeplitz_f32<false>(x, y, d_taps, rows, nch, 1, 1, s);
}

cudaError_t launch_filter_f32_tr(const float* x, float* yt, const float* d_taps, long rows, int nch, int nr, int nrp,
                                 cudaStream_t s) {
  return launch_toeplitz_f32<true>(x, yt, d_taps, rows, nch, nr, nrp, s);
}

// ---------------------------------------------------------------------------
// thickening
// ---------------------------------------------------------------------------
//
// thicken_slices (cuda_kernels.cuh:289-320): output slice r is the
// triangle-weighted mean of the native slices with nonzero weight
// max(0, 1 - |z_n - z_r| / slice_thickness). The weights and their list per
// output slice are computed on the host in the reference's float arithmetic;
// the per-voxel sums run in the same slice order.
__global__ void k_thicken(const float* __restrict__ vn, float* __restrict__ out, const int* __restrict__ off,
                          const int* __restrict__ idx, const float* __restrict__ w, const float* __restrict__ ws,
                          int nxy, const int* __restrict__ list) {
  const int r = list ? __ldg(list + blockIdx.y) : (int)blockIdx.y;
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  if (px >= nxy) return;
  const int a = off[r], b = off[r + 1];
  float val = 0.0f;
  for (int t = a; t < b; t++) val = fmaf(w[t], __ldg(vn + (size_t)idx[t] * nxy + px), val);
  out[(size_t)r * nxy + px] = val / ws[r];
}

cudaError_t launch_thicken(const float* vn, float* out, const int* off, const int* idx, const float* w,
                           const float* ws, int nxy, int nzr, cudaStream_t s, const int* list) {
  if (nzr < 1) return cudaSuccess;
  dim3 grid((unsigned)((nxy + 255) / 256), (unsigned)nzr);
  k_thicken<<<grid, 256, 0, s>>>(vn, out, off, idx, w, ws, nxy, list);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// rebin for the mixed-precision filter
// ---------------------------------------------------------------------------
//
// Same samples as k_rebin_f32_rows, written as the two FP16 operand planes of
// the tensor-core Toeplitz filter: hi = f16(o x), lo = f16(o x - hi), 22
// bits of x, with a per-view power of two o. One CTA per view writes the
// planes with o = 1 while it finds the row maxima; a view whose largest
// sample exceeds 16384 (far above any line integral, but FP16 ends at 65504)
// is written again with the largest o that brings it to 16384. (FP16 keeps
// 22 bits of the split down to |x| ~ 0.125 and an absolute 3e-8 below, far
// inside the filter's error budget.) The view's rows are padded with zero rows to nrv (a power of two
// that divides the filter's 128-row tile, so no view straddles a tile) and
// every row with zeros to kp (a multiple of 64). The CTA also writes the FP16
// storage scales of the filtered rows: per row, the smallest power of two s
// with max|x| * sum|h| / s <= 16384 (|y| <= sum|h| max|x| bounds every
// filtered value of the row), per view the largest of its rows' scales, and
// the operand scale o.
constexpr int RS_THREADS = 256;

// One thread per channel of the view computes the channel's taps once
// (as k_rebin_f32_rows) and walks every row; the per-row maxima go through a
// warp reduction and one shared-memory atomic per warp and row.
// Scales of one view from its row maxima (shared memory, [nrv]): row and
// view storage scales of the filtered rows and the operand scale (1, or for
// a view whose largest sample exceeds 16384 the power of two that brings it
// to 16384). Returns the operand scale.
__device__ float split_view_scales(const float* s_rowmax, int nrv, int v, float taps_l1, float* __restrict__ row_scale,
                                   float* __restrict__ view_scale, float* __restrict__ op_scale) {
  __shared__ float s_vmax, s_xmax;
  if (threadIdx.x == 0) s_vmax = s_xmax = 0.0f;
  __syncthreads();
  for (int i = threadIdx.x; i < nrv; i += blockDim.x) {
    const float bound = fmaxf(s_rowmax[i] * taps_l1, 1e-30f) * (1.0f / 16384.0f);
    const float sc = exp2f(ceilf(log2f(bound)));
    row_scale[(size_t)v * nrv + i] = sc;
    atomicMax(reinterpret_cast<int*>(&s_vmax), __float_as_int(sc));
    atomicMax(reinterpret_cast<int*>(&s_xmax), __float_as_int(s_rowmax[i]));
  }
  __syncthreads();
  const float xm = s_xmax;
  const float o = xm > 16384.0f ? exp2f(floorf(log2f(16384.0f / xm))) : 1.0f;
  if (threadIdx.x == 0) {
    view_scale[v] = s_vmax;
    op_scale[v] = o;
  }
  return o;
}

// Writes o x as FP16 hi / lo.
__device__ __forceinline__ void split_f16(float x, float o, __half* hi, __half* lo) {
  const float y = x * o;  // o is a power of two: exact
  const __half h = __float2half_rn(y);
  *hi = h;
  *lo = __float2half_rn(y - __half2float(h));
}

template <bool FFS>
__global__ void __launch_bounds__(RS_THREADS)
k_rebin_split_rows(const float* __restrict__ raw, __half* __restrict__ a_hi, __half* __restrict__ a_lo,
                   float* __restrict__ row_scale, float* __restrict__ view_scale, float* __restrict__ op_scale,
                   const float* __restrict__ beta_t, const float* __restrict__ bidx_t,
                   const double2* __restrict__ chan64, RebinParams p, int kp, int nrv, float taps_l1, int vb) {
  extern __shared__ float s_rowmax[];  // [nrv]
  const int v = vb + blockIdx.x;
  const int lane = threadIdx.x % 32;
  for (int i = threadIdx.x; i < nrv; i += blockDim.x) s_rowmax[i] = 0.0f;
  __syncthreads();
  auto taps = [&](int c, RebinTaps& t, RebinTapsFfs& tf) {
    t.ok = false;
    tf.ok = false;
    if (c >= p.nch) return;
    if (chan64) {  // FP64 sample coordinates
      if constexpr (FFS) tf = rebin_taps_ffs64(p, __ldg(chan64 + c), v);
      else t = rebin_taps64(raw, (size_t)p.nr * p.nch, p.V, p.nr, p.nch, __ldg(chan64 + c), v, p.voff);
    } else {
      if constexpr (FFS) tf = rebin_taps_ffs(p, __ldg(bidx_t + c), __ldg(beta_t + c), v);
      else t = wfbp_rebin_taps(raw, p, __ldg(bidx_t + c), __ldg(beta_t + c), v);
    }
  };
  auto sample = [&](const RebinTaps& t, const RebinTapsFfs& tf, int i) -> float {
    return i >= p.nr ? 0.0f  // 0 off the detector and in the padding
                     : FFS ? rebin_taps_ffs_sample(raw, p, tf, i) : rebin_taps_sample(t, i, p.nch);
  };
  // pass 1: the planes with o = 1 and the row maxima; kp is a multiple of 64,
  // so every warp is either wholly inside [0, kp) or wholly outside
  for (int c = threadIdx.x; c < kp; c += blockDim.x) {
    RebinTaps t;
    RebinTapsFfs tf;
    taps(c, t, tf);
    // four rows' samples (16 independent loads) before their stores and reductions
    for (int i0 = 0; i0 < nrv; i0 += 4) {
      float x[4];
#pragma unroll
      for (int u = 0; u < 4; u++) x[u] = sample(t, tf, i0 + u);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int i = i0 + u;
        if (i >= nrv) break;  // warp-uniform
        // fmaxf semantics: a NaN sample does not raise the maximum
        const float ax = isnan(x[u]) ? 0.0f : fabsf(x[u]);
        const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(ax));  // ax >= 0: bits order as values
        if (lane == 0 && m) atomicMax(reinterpret_cast<int*>(&s_rowmax[i]), (int)m);
        const size_t row = (size_t)v * nrv + i;
        split_f16(x[u], 1.0f, a_hi + row * kp + c, a_lo + row * kp + c);
      }
    }
  }
  __syncthreads();
  const float o = split_view_scales(s_rowmax, nrv, v, taps_l1, row_scale, view_scale, op_scale);
  if (o == 1.0f) return;  // block-uniform
  // a view beyond FP16's comfortable range: the planes again with o < 1
  for (int c = threadIdx.x; c < kp; c += blockDim.x) {
    RebinTaps t;
    RebinTapsFfs tf;
    taps(c, t, tf);
    for (int i0 = 0; i0 < nrv; i0 += 4) {
      float x[4];
#pragma unroll
      for (int u = 0; u < 4; u++) x[u] = sample(t, tf, i0 + u);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int i = i0 + u;
        if (i >= nrv) break;
        const size_t row = (size_t)v * nrv + i;
        split_f16(x[u], o, a_hi + row * kp + c, a_lo + row * kp + c);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// view-chunk rebin (no flying focal spot)
// ---------------------------------------------------------------------------
//
// Output sample (v, i, c) blends readings y0(v, c) and y1(v, c) = y0 + 1
// (clamped), and y0(v + 1, c) = y1(v, c) except where the rounding of the
// sample coordinates or the clamp at the scan's ends says otherwise. In the
// per-view kernels above every texel row is fetched twice from L2, once as
// y1 of view v and once as y0 of view v + 1, by CTAs of different views.
// Here a thread owns one channel of RV_NY consecutive views and loads, per
// detector row, the RV_NY + 1 readings y0(v0), y1(v0), ..., y1(v0 + RV_NY - 1)
// once (a separate y0 load only where the chain breaks): (RV_NY + 1) / (2
// RV_NY) of the texel traffic. The lanes of a warp are consecutive channels
// of the same view (full-line stores). Taps and sample arithmetic are the
// per-view kernels' (rebin_taps_x / rebin_taps_y or their FP64 forms,
// rebin_bilinear), so the samples are the same bit for bit.
// SPLIT writes the two FP16 planes with o = 1 and the row maxima (one warp
// reduction per view and row, the CTA's warps merged in shared memory, then
// into the global maxima: bits of |x| in row_scale, zeroed before the
// launch); k_rebin_split_scales turns them into the scales.
template <bool SPLIT, bool F64>
__global__ void __launch_bounds__(RV_CW)
k_rebin_vchunk(const float* __restrict__ raw, float* __restrict__ out, __half* __restrict__ a_hi,
               __half* __restrict__ a_lo, unsigned* __restrict__ rowmax, const float* __restrict__ beta_t,
               const float* __restrict__ bidx_t, const double2* __restrict__ chan64, RebinParams p, int kp, int nrv,
               int vb, int ve) {
  extern __shared__ unsigned s_max[];  // SPLIT: [RV_NY][nrv] largest |sample| (bits; >= 0 orders as values)
  const int lane = threadIdx.x % 32;
  const int c = blockIdx.x * RV_CW + threadIdx.x;
  const int v0 = vb + (int)blockIdx.y * RV_NY;
  const int nv = min(RV_NY, ve - v0);
  const int ncw = SPLIT ? kp : p.nch;  // channels written (the planes' padding channels hold zeros)
  const int cc = min(c, p.nch - 1);
  RebinTapsX tx;
  tx.ok = false;
  tx.c0 = tx.c1 = 0;
  tx.ax = 0.0f;
  if (c < p.nch) tx = F64 ? rebin_taps64_x(p.nch, __ldg(chan64 + c)) : rebin_taps_x(p.nch, __ldg(bidx_t + c), p.q8);
  const float beta = F64 ? 0.0f : __ldg(beta_t + cc);
  const double2 ch = F64 ? __ldg(chan64 + cc) : make_double2(0.0, 0.0);
  // element offsets (reading y, sheet row 0, channel c0) from the last raw row:
  // r[k] = y0 of view k for k = 0, else y1 of view k - 1; b[k] = y0 of view k
  // where it differs from y1 of view k - 1 (brk bit k)
  const int vs = p.nr * p.nch;
  int r[RV_NY + 1], yb[RV_NY];
  float ay[RV_NY];
  unsigned brk = 0u;
#pragma unroll
  for (int k = 0; k < RV_NY; k++) {
    RebinTapsY ty;
    ty.y0 = ty.y1 = 0;
    ty.ay = 0.0f;
    if (k < nv && c < p.nch)
      ty = F64 ? rebin_taps64_y(p.V, ch, v0 + k, p.voff) : rebin_taps_y(p.V, beta, v0 + k, p.dth, p.q8, p.voff);
    const int o0 = ty.y0 * vs + tx.c0, o1 = ty.y1 * vs + tx.c0;
    if (k == 0) r[0] = o0;
    yb[k] = o0;
    if (k > 0 && o0 != r[k]) brk |= 1u << k;
    r[k + 1] = o1;
    ay[k] = ty.ay;
  }
  const int dc = tx.c1 - tx.c0;  // -1, or 0 at the detector's last channel (c0 = 0)
  if constexpr (SPLIT) {
    for (int e = threadIdx.x; e < RV_NY * nrv; e += RV_CW) s_max[e] = 0u;
    __syncthreads();
  }
  const bool wr = c < ncw;
  const float* last = raw + (size_t)(p.nr - 1) * p.nch;
  const int nrows = SPLIT ? nrv : p.nr;
  for (int i = 0; i < nrows; i++) {
    const float* row = last - (size_t)min(i, p.nr - 1) * p.nch;  // rows >= nr: padding, written as zeros
    float ta[RV_NY + 1], tb[RV_NY + 1];
#pragma unroll
    for (int k = 0; k <= RV_NY; k++) {
      ta[k] = tb[k] = 0.0f;
      if (k <= nv) {
        ta[k] = __ldg(row + r[k]);
        tb[k] = __ldg(row + (r[k] + dc));
      }
    }
    float x[RV_NY];
#pragma unroll
    for (int k = 0; k < RV_NY; k++) {
      float t00 = ta[k], t10 = tb[k];
      if ((brk >> k) & 1u) {
        t00 = __ldg(row + yb[k]);
        t10 = __ldg(row + (yb[k] + dc));
      }
      x[k] = tx.ok && i < p.nr ? rebin_bilinear(t00, t10, ta[k + 1], tb[k + 1], tx.ax, ay[k]) : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < RV_NY; k++) {
      if (k < nv && wr) {
        if constexpr (SPLIT) {
          const size_t o = ((size_t)(v0 + k) * nrv + i) * kp + c;
          split_f16(x[k], 1.0f, a_hi + o, a_lo + o);
        } else {
          out[((size_t)(v0 + k) * p.nr + i) * p.nch + c] = x[k];
        }
      }
    }
    if constexpr (SPLIT) {
#pragma unroll
      for (int k = 0; k < RV_NY; k++) {
        // fmaxf semantics: a NaN sample does not raise the maximum
        const float a = wr && k < nv && !isnan(x[k]) ? fabsf(x[k]) : 0.0f;
        const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(a));
        if (lane == 0 && m) atomicMax(&s_max[k * nrv + i], m);
      }
    }
  }
  if constexpr (SPLIT) {
    __syncthreads();
    for (int e = threadIdx.x; e < nv * nrv; e += RV_CW) {
      const unsigned m = s_max[e];
      if (m) atomicMax(rowmax + (size_t)(v0 + e / nrv) * nrv + e % nrv, m);
    }
  }
}

// The scales of the mixed rebin's views from the row maxima that
// k_rebin_vchunk left in row_scale (split_view_scales, one CTA per view); a
// view whose largest sample exceeds 16384 has its planes written again with
// the operand scale o < 1 (the samples recomputed, as the per-view kernels'
// second pass).
template <bool F64>
__global__ void __launch_bounds__(RS_THREADS)
k_rebin_split_scales(const float* __restrict__ raw, __half* __restrict__ a_hi, __half* __restrict__ a_lo,
                     float* __restrict__ row_scale, float* __restrict__ view_scale, float* __restrict__ op_scale,
                     const float* __restrict__ beta_t, const float* __restrict__ bidx_t,
                     const double2* __restrict__ chan64, RebinParams p, int kp, int nrv, float taps_l1, int vb) {
  extern __shared__ float s_rowmax[];  // [nrv]
  const int v = vb + blockIdx.x;
  for (int i = threadIdx.x; i < nrv; i += blockDim.x) s_rowmax[i] = row_scale[(size_t)v * nrv + i];
  __syncthreads();
  const float o = split_view_scales(s_rowmax, nrv, v, taps_l1, row_scale, view_scale, op_scale);
  if (o == 1.0f) return;  // block-uniform
  for (int c = threadIdx.x; c < kp; c += blockDim.x) {
    RebinTaps t;
    t.ok = false;
    t.raw0 = t.raw1 = raw;
    t.c0 = t.c1 = 0;
    t.ax = t.ay = 0.0f;
    if (c < p.nch)
      t = F64 ? rebin_taps64(raw, (size_t)p.nr * p.nch, p.V, p.nr, p.nch, __ldg(chan64 + c), v, p.voff)
              : wfbp_rebin_taps(raw, p, __ldg(bidx_t + c), __ldg(beta_t + c), v);
    for (int i = 0; i < nrv; i++) {
      const float x = i < p.nr ? rebin_taps_sample(t, i, p.nch) : 0.0f;
      const size_t row = (size_t)v * nrv + i;
      split_f16(x, o, a_hi + row * kp + c, a_lo + row * kp + c);
    }
  }
}

cudaError_t launch_rebin_split(const float* raw, void* planes, float* row_scale, float* view_scale,
                               float* op_scale, const float* d_beta, const float* d_bidx, const double2* d_chan64,
                               const RebinParams& p, int kp, int nrv, float taps_l1, cudaStream_t s, int vb, int ve) {
  if (ve < 0) ve = p.V;
  if (vb < 0 || vb >= ve || ve > p.V) return cudaErrorInvalidValue;
  const size_t rows = (size_t)p.V * nrv;
  __half* hi = reinterpret_cast<__half*>(planes);
  __half* lo = hi + rows * kp;
  if (kp % 64 != 0) return cudaErrorInvalidValue;  // whole warps per channel run (the row maxima's reduction)
  if (use_vchunk_rebin(p)) {
    cudaError_t e = cudaMemsetAsync(row_scale + (size_t)vb * nrv, 0, sizeof(float) * (size_t)(ve - vb) * nrv, s);
    if (e != cudaSuccess) return e;
    const dim3 g((unsigned)((kp + RV_CW - 1) / RV_CW), (unsigned)((ve - vb + RV_NY - 1) / RV_NY));
    const size_t sm = sizeof(unsigned) * (size_t)RV_NY * nrv;
    unsigned* rmax = reinterpret_cast<unsigned*>(row_scale);
    if (d_chan64) {
      k_rebin_vchunk<true, true><<<g, RV_CW, sm, s>>>(raw, nullptr, hi, lo, rmax, d_beta, d_bidx, d_chan64, p, kp,
                                                       nrv, vb, ve);
      k_rebin_split_scales<true><<<(unsigned)(ve - vb), RS_THREADS, sizeof(float) * nrv, s>>>(
          raw, hi, lo, row_scale, view_scale, op_scale, d_beta, d_bidx, d_chan64, p, kp, nrv, taps_l1, vb);
    } else {
      k_rebin_vchunk<true, false><<<g, RV_CW, sm, s>>>(raw, nullptr, hi, lo, rmax, d_beta, d_bidx, nullptr, p,
                                                        kp, nrv, vb, ve);
      k_rebin_split_scales<false><<<(unsigned)(ve - vb), RS_THREADS, sizeof(float) * nrv, s>>>(
          raw, hi, lo, row_scale, view_scale, op_scale, d_beta, d_bidx, nullptr, p, kp, nrv, taps_l1, vb);
    }
  } else if (p.G == 1)
    k_rebin_split_rows<false><<<(unsigned)(ve - vb), RS_THREADS, sizeof(float) * nrv, s>>>(
        raw, hi, lo, row_scale, view_scale, op_scale, d_beta, d_bidx, d_chan64, p, kp, nrv, taps_l1, vb);
  else
    k_rebin_split_rows<true><<<(unsigned)(ve - vb), RS_THREADS, sizeof(float) * nrv, s>>>(
        raw, hi, lo, row_scale, view_scale, op_scale, d_beta, d_bidx, d_chan64, p, kp, nrv, taps_l1, vb);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// adaptive filtration of the raw readings
// ---------------------------------------------------------------------------
//
// ReconConfig.adaptive_filtration_s, which fct_wfbp parses
// (parse_config.cpp:57) but never applies, defined here as
// attenuation-adaptive smoothing of the raw line integrals after Kachelriess,
// Watzke and Kalender, Med. Phys. 28 (2001) 475-490: with p_max the largest
// line integral of a reading and p_t = (1 - s) p_max (0 < s <= 1), each sample
// p becomes p + w (pbar - p), pbar = (p[c-1] + 2 p[c] + p[c+1]) / 4 along its
// detector row (edge channels repeated), w = clamp((p - p_t) / (p_max - p_t),
// 0, 1). A reading with p_max <= 0 is copied unchanged. One CTA per reading:
// the maximum by a block reduction, then the smoothing (the reading, a few
// hundred KB, is read twice from L2).
__global__ void __launch_bounds__(256)
k_adaptive_filter(const float* __restrict__ raw, float* __restrict__ out, int nr, int nch, float s, long r0) {
  __shared__ float s_max[8];
  const size_t frame = (size_t)nr * nch;
  const float* x = raw + (size_t)(r0 + blockIdx.x) * frame;
  float* y = out + (size_t)(r0 + blockIdx.x) * frame;
  float m = -INFINITY;
  for (size_t k = threadIdx.x; k < frame; k += blockDim.x) m = fmaxf(m, __ldg(x + k));  // NaN ignored
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (threadIdx.x % 32 == 0) s_max[threadIdx.x / 32] = m;
  __syncthreads();
  float pmax = s_max[0];
  for (int w = 1; w < (int)(blockDim.x / 32); w++) pmax = fmaxf(pmax, s_max[w]);
  if (!(pmax > 0.0f)) {
    for (size_t k = threadIdx.x; k < frame; k += blockDim.x) y[k] = __ldg(x + k);
    return;
  }
  const float pt = (1.0f - s) * pmax;
  const float inv = 1.0f / (pmax - pt);
  for (size_t k = threadIdx.x; k < frame; k += blockDim.x) {
    const int c = (int)(k % (size_t)nch);
    const float p = __ldg(x + k);
    const float a = __ldg(x + k - (c > 0 ? 1 : 0)), b = __ldg(x + k + (c < nch - 1 ? 1 : 0));
    const float pb = 0.25f * (a + 2.0f * p + b);
    const float w = __saturatef((p - pt) * inv);
    y[k] = fmaf(w, pb - p, p);
  }
}

namespace {
__global__ void k_fill(float* __restrict__ dst, float value, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = value;
}
}  // namespace

cudaError_t launch_fill(float* dst, float value, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 1184);
  k_fill<<<blocks, 256, 0, s>>>(dst, value, n);
  return cudaGetLastError();
}

cudaError_t launch_adaptive_filter(const float* raw, float* out, int nr, int nch, float s, long r0, long r1,
                                   cudaStream_t st) {
  if (r1 <= r0) return cudaSuccess;
  if (!(s > 0.0f) || s > 1.0f) return cudaErrorInvalidValue;
  k_adaptive_filter<<<(unsigned)(r1 - r0), 256, 0, st>>>(raw, out, nr, nch, s, r0);
  return cudaGetLastError();
}

