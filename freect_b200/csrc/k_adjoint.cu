// Adjoint kernels of the FP32 path (sm_100a): the exact transposes of the
// forward stages, for gradients with respect to the raw readings and the
// filter taps. No counterpart in the reference, whose fct_wfbp has no
// backward pass; each kernel states the forward loop it transposes.
//
// None of them uses atomics: every output element is owned by one thread,
// which gathers the forward contributions that reach it (so results do not
// depend on scheduling).
#include "wfbp_internal.h"

#include <math.h>

#include "bp_math.cuh"
#include "rebin_sample.cuh"

namespace {

// W(q) exactly as the forward backprojection (k_backproject.cu) evaluates it.
__device__ __forceinline__ float q_weight_fwd(float qh) {
  float t = __saturatef(fmaf(fabsf(qh), 2.5f, -1.5f));
  return fmaf(0.5f, __cosf(3.14159265f * t), 0.5f);
}

// ---------------------------------------------------------------------------
// backprojection adjoint
// ---------------------------------------------------------------------------
//
// Forward (k_bp, the reference-layout FP32 backprojection): for voxel
// (x, y, z) and half-turn angle t, with views j = t + k P/2,
//   vol += dtheta / sum_k W_k * sum_k W_k * bilinear(D_j; p_idx_j, q_idx_j).
// The gradient of one filtered sample D[j][r][c] is therefore
//   sum over voxels of g_vol * dtheta * W_j / sum_k W_k * hat(p_idx_j - c) * hat_row,
// where hat is the bilinear weight. Ownership: a CTA owns view j and a run of
// AD_CH consecutive channels; thread c walks the voxels whose p_idx lies in
// [c, c + 1) (a band one channel wide around a line through the image,
// traversed along its longer axis), so every (voxel, view) pair is visited
// by exactly one thread. For each such voxel it visits the slices inside the
// view's cone, takes g_vol * dtheta / sum_k W_k from the scale table (or
// recomputes sum_k W_k from the same expressions as the forward), and adds
// the row contributions to two accumulators of its own in shared memory: one
// for channel c (weight 1 - frac(p_idx)) and one for channel c + 1 (weight
// frac(p_idx)). At the end channel c = own(c) + next(c - 1), in that order;
// the CTA's first thread only supplies next(c0 - 1) for its neighbour.
constexpr int AD_CH = 128;

__device__ __forceinline__ float xcoord(const BPParams& p, int ix) {
  return ((float)ix - 0.5f * ((float)p.nx - 1.0f)) * p.fov / (float)p.nx + p.x0;
}
__device__ __forceinline__ float ycoord(const BPParams& p, int iy) {
  return ((float)iy - 0.5f * ((float)p.ny - 1.0f)) * p.fov / (float)p.ny + p.y0;
}

struct ViewGeo {
  float zt, A, lt, inv, p_idx;  // lt = l_hat tan(cone), inv = 1 / lt
  bool valid_p;
};

__device__ __forceinline__ ViewGeo view_geo(const BPParams& p, float x, float y, float2 sc, float zt) {
  ViewGeo g;
  g.zt = zt;
  const float p_hat = x * sc.x - y * sc.y;
  // the forward's short forms (bp_math.cuh): hardware square root and
  // reciprocal, arcsine from its series
  const float l_hat = bp_sqrt(p.R2 - p_hat * p_hat) - x * sc.y - y * sc.x;
  g.A = p.zr2pi * bp_asin(p.rR * p_hat);
  g.lt = l_hat * p.tanc;
  g.inv = bp_rcp(g.lt);
  g.p_idx = p.kp - (p_hat * p.ps + p.c0);
  const float pf = floorf(g.p_idx);
  g.valid_p = pf >= 0.0f && ceilf(g.p_idx) <= p.ncm2;
  return g;
}

// Q weight of view geometry g at slice z (0 where the forward skips it).
__device__ __forceinline__ float view_weight(const BPParams& p, const ViewGeo& g, float z, float* q_idx_out) {
  const float dz = z - g.zt;
  const float qh = (dz + g.A) * g.inv;
  const float q_idx = (qh + 1.0f) * p.hn;
  *q_idx_out = q_idx;
  const bool ok = g.valid_p && fabsf(dz) <= p.z_rot && q_idx >= 0.0f && q_idx <= p.nrm2;
  return ok ? q_weight_fwd(qh) : 0.0f;
}

// Weights G[t][y][x][s] = dtheta / sum_k W_k for each half-turn angle t
// (0 where no half turn contributes, as the forward's NaN voxel has no
// gradient), slices innermost with a stride of nzp = nz rounded up to 4: one
// thread per (x, y) column and ZS slices, the weights summed in the
// forward's order. They depend on the geometry alone (views, slices, grid),
// so the context computes them once and every later gradient reuses them;
// with the table the gather below needs one load instead of the other half
// turns' geometry, and a voxel's slice run is one contiguous span.
constexpr int AN_ZS = 8, AN_TX = 16, AN_TY = 8;

__global__ void __launch_bounds__(AN_TX * AN_TY)
k_bp_adjoint_scale(float* __restrict__ G, const float2* __restrict__ view_sc,
                   const float* __restrict__ view_z, const float* __restrict__ zslices, BPParams p, int nzp) {
  const int ix = blockIdx.x * AN_TX + (threadIdx.x % AN_TX);
  const int iy = blockIdx.y * AN_TY + (threadIdx.x / AN_TX);
  const int s0 = blockIdx.z * AN_ZS;
  if (ix >= p.nx || iy >= p.ny) return;
  const float x = xcoord(p, ix), y = ycoord(p, iy);
  const size_t plane = (size_t)p.nx * p.ny, vox = (size_t)iy * p.nx + ix;
  const bool active = !(x * x + y * y > p.fov_half2);
  float z[AN_ZS];
#pragma unroll
  for (int i = 0; i < AN_ZS; i++) z[i] = s0 + i < p.nz ? __ldg(zslices + s0 + i) : 0.0f;
  for (int t = 0; t < p.P2; t++) {
    float aw[AN_ZS];
#pragma unroll
    for (int i = 0; i < AN_ZS; i++) aw[i] = 0.0f;
    if (active) {
      for (int k = 0; k < p.K; k++) {
        const int j = t + k * p.P2;
        const float zt = __ldg(view_z + j);
        const ViewGeo g = view_geo(p, x, y, __ldg(view_sc + j), zt);
        if (!g.valid_p) continue;
#pragma unroll
        for (int i = 0; i < AN_ZS; i++) {
          float qi;
          aw[i] += view_weight(p, g, z[i], &qi);
        }
      }
    }
    float* out = G + ((size_t)t * plane + vox) * nzp + s0;
#pragma unroll
    for (int i = 0; i < AN_ZS; i++)
      if (s0 + i < nzp) out[i] = s0 + i < p.nz && aw[i] > 0.0f ? p.dtheta * (1.0f / aw[i]) : 0.0f;
  }
}

template <bool TABLE>
__global__ void __launch_bounds__(AD_CH, 8)
k_bp_adjoint(const float* __restrict__ gvol, const float* __restrict__ G, float* __restrict__ gD,
             const float2* __restrict__ view_sc, const float* __restrict__ view_z, const float* __restrict__ zslices,
             BPParams p, float z0, float dzs, int nzp) {
  extern __shared__ float2 acc2[];  // [nr][AD_CH]: (own channel, next channel) of thread cl
  // views of one half-turn angle run in consecutive blocks, so that they
  // share its slice of the scale table in L2: block row b < K P/2 is view
  // t + k P/2 with t = b / K, k = b % K; the views the forward never reads
  // (j >= K P/2) follow in order
  const int b = blockIdx.y, used = p.K * p.P2;
  const int j = b < used ? (b / p.K) + (b % p.K) * p.P2 : b;
  const int cl = threadIdx.x;
  const int c = blockIdx.x * (AD_CH - 1) - 1 + cl;  // channels c0 - 1 .. c0 + AD_CH - 2
  for (int r = 0; r < p.nr; r++) acc2[r * AD_CH + cl] = make_float2(0.0f, 0.0f);

  const int t = j % p.P2, kj = j / p.P2;
  if (kj < p.K && c >= 0 && c < p.nch) {
    const float2 sc = __ldg(view_sc + j);
    const float zt = __ldg(view_z + j);
    // p_idx in [c, c + 1) <=> p_hat in this interval (widened by a rounding
    // margin; the exact forward test below decides)
    const float ph_a = (p.kp - p.c0 - ((float)c + 1.0f)) / p.ps, ph_b = (p.kp - p.c0 - (float)c) / p.ps;
    const float marg = 0.02f / p.ps + 1e-3f * p.fov / (float)p.nx;
    const float plo = fminf(ph_a, ph_b) - marg, phi = fmaxf(ph_a, ph_b) + marg;
    const float sx = p.fov / (float)p.nx, sy = p.fov / (float)p.ny;
    const float nxm = 0.5f * ((float)p.nx - 1.0f), nym = 0.5f * ((float)p.ny - 1.0f);
    const bool along_y = fabsf(sc.x) >= fabsf(sc.y);  // p_hat = x sin - y cos: solve for x per row y
    const int n_outer = along_y ? p.ny : p.nx;
    // the candidate range of each row through reciprocals computed once: their
    // rounding (a few 1e-5 mm) stays far inside the margin, and the exact
    // channel test below decides which voxels the thread owns
    const float r_sc = 1.0f / (along_y ? sc.x : sc.y), r_sx = 1.0f / sx, r_sy = 1.0f / sy;
    for (int o = 0; o < n_outer; o++) {
      int i_lo, i_hi;
      if (along_y) {
        const float y = ycoord(p, o);
        float xa = (plo + y * sc.y) * r_sc, xb = (phi + y * sc.y) * r_sc;
        if (xa > xb) { const float tt = xa; xa = xb; xb = tt; }
        i_lo = max(0, (int)floorf((xa - p.x0) * r_sx + nxm));
        i_hi = min(p.nx - 1, (int)ceilf((xb - p.x0) * r_sx + nxm));
      } else {
        const float x = xcoord(p, o);
        float ya = (x * sc.x - phi) * r_sc, yb = (x * sc.x - plo) * r_sc;
        if (ya > yb) { const float tt = ya; ya = yb; yb = tt; }
        i_lo = max(0, (int)floorf((ya - p.y0) * r_sy + nym));
        i_hi = min(p.ny - 1, (int)ceilf((yb - p.y0) * r_sy + nym));
      }
      for (int in = i_lo; in <= i_hi; in++) {
        const int ix = along_y ? in : o, iy = along_y ? o : in;
        const float x = xcoord(p, ix), y = ycoord(p, iy);
        if (x * x + y * y > p.fov_half2) continue;  // cuda_kernels.cuh:220
        {
          // the channel test first (three FMAs), the square root, arcsine
          // and division of the geometry only for the voxel that passes it
          const float ph = x * sc.x - y * sc.y;
          if ((int)floorf(p.kp - (ph * p.ps + p.c0)) != c) continue;
        }
        const ViewGeo g = view_geo(p, x, y, sc, zt);
        if (!g.valid_p) continue;
        const float pf = floorf(g.p_idx), wp = g.p_idx - pf;
        if ((int)pf != c) continue;
        const float h0 = 1.0f - wp;  // channel c; channel c + 1 gets wp
        // slices that can pass this view's tests: |z - zt| <= z_rot and
        // q_idx in [0, nr-2], a z interval around zt - A
        const float za = zt - g.A - g.lt, zb = zt - g.A + (p.nrm2 / p.hn - 1.0f) * g.lt;
        const float zlo = fmaxf(fminf(za, zb), zt - p.z_rot), zhi = fminf(fmaxf(za, zb), zt + p.z_rot);
        if (zlo > zhi) continue;
        int s_lo, s_hi;
        if (p.nz == 1 || dzs == 0.0f) {
          s_lo = 0;
          s_hi = p.nz - 1;
        } else {
          float fa = (zlo - z0) / dzs, fb = (zhi - z0) / dzs;
          if (fa > fb) { const float tt = fa; fa = fb; fb = tt; }
          s_lo = max(0, (int)floorf(fa) - 1);
          s_hi = min(p.nz - 1, (int)ceilf(fb) + 1);
        }
        if constexpr (TABLE) {
          // the voxel's weights and gradients are contiguous runs over the
          // slices (both [.][y][x][nzp]): aligned float4 blocks, the next
          // block's loads issued before this block's arithmetic
          const float4* wrow = reinterpret_cast<const float4*>(G + (((size_t)t * p.ny + iy) * p.nx + ix) * nzp);
          const float4* grow = reinterpret_cast<const float4*>(gvol + ((size_t)iy * p.nx + ix) * nzp);
          const int e4 = s_hi >> 2;
          int b4 = s_lo >> 2;
          float4 wn = __ldg(wrow + b4), gn = __ldg(grow + b4);
          for (; b4 <= e4; b4++) {
            const float wa[4] = {wn.x, wn.y, wn.z, wn.w}, ga[4] = {gn.x, gn.y, gn.z, gn.w};
            if (b4 < e4) {
              wn = __ldg(wrow + b4 + 1);
              gn = __ldg(grow + b4 + 1);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
              const int s = 4 * b4 + u;
              if (s < s_lo || s > s_hi || wa[u] == 0.0f) continue;
              float q_idx;
              const float Wj = view_weight(p, g, __ldg(zslices + s), &q_idx);
              if (Wj == 0.0f) continue;
              const float scaled = ga[u] * wa[u];  // g_vol * dtheta / sum_k W_k (cuda_kernels.cuh:283)
            const float sw = scaled * Wj;
            const float c0v = sw * h0, c1v = sw * wp;
            const float qf = floorf(q_idx), wq = q_idx - qf;
            const int r = min(max((int)qf, 0), p.nr - 2);
            float2* a0 = acc2 + r * AD_CH + cl;
            float2 v0 = a0[0], v1 = a0[AD_CH];
            v0.x += c0v * (1.0f - wq);
            v0.y += c1v * (1.0f - wq);
            v1.x += c0v * wq;
            v1.y += c1v * wq;
            a0[0] = v0;
            a0[AD_CH] = v1;
            }
          }
        } else {
          for (int s = s_lo; s <= s_hi; s++) {
            const float z = __ldg(zslices + s);
            float q_idx;
            const float Wj = view_weight(p, g, z, &q_idx);
            if (Wj == 0.0f) continue;
            const float gv = __ldg(gvol + ((size_t)s * p.ny + iy) * p.nx + ix);
            if (gv == 0.0f) continue;
            // sum of the weights of all half turns, in the forward's order
            float aw = 0.0f;
            for (int k = 0; k < p.K; k++) {
              const int jj = t + k * p.P2;
              if (jj == j) {
                aw += Wj;
                continue;
              }
              const float ztk = __ldg(view_z + jj);
              if (!(fabsf(z - ztk) <= p.z_rot)) continue;
              const ViewGeo gk = view_geo(p, x, y, __ldg(view_sc + jj), ztk);
              float qk;
              aw += view_weight(p, gk, z, &qk);
            }
            const float scaled = gv * (p.dtheta * (1.0f / aw));  // cuda_kernels.cuh:283
            const float sw = scaled * Wj;
            const float c0v = sw * h0, c1v = sw * wp;
            const float qf = floorf(q_idx), wq = q_idx - qf;
            const int r = min(max((int)qf, 0), p.nr - 2);
            float2* a0 = acc2 + r * AD_CH + cl;
            float2 v0 = a0[0], v1 = a0[AD_CH];
            v0.x += c0v * (1.0f - wq);
            v0.y += c1v * (1.0f - wq);
            v1.x += c0v * wq;
            v1.y += c1v * wq;
            a0[0] = v0;
            a0[AD_CH] = v1;
          }
        }
      }
    }
  }
  __syncthreads();
  if (cl >= 1 && c < p.nch) {
    float* out = gD + (size_t)j * p.nr * p.nch + c;
    for (int r = 0; r < p.nr; r++) out[(size_t)r * p.nch] = acc2[r * AD_CH + cl].x + acc2[r * AD_CH + cl - 1].y;
  }
}

// gvt[vox][s] = gvol[s][vox] (s < nz), 0 for the padding up to nzp.
__global__ void k_adj_gvol_t(const float* __restrict__ gvol, float* __restrict__ gvt, int nxy, int nz, int nzp) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)nxy * nzp) return;
  const long vox = i / nzp;
  const int sl = (int)(i % nzp);
  gvt[i] = sl < nz ? __ldg(gvol + (size_t)sl * nxy + vox) : 0.0f;
}

// ---------------------------------------------------------------------------
// thickening adjoint
// ---------------------------------------------------------------------------
// Forward: vol[r] = sum_n w_rn vol_n / ws_r over the CSR of requested slice r.
// Transposed CSR (built on the host): native slice n lists (r, w_rn / ws_r).
__global__ void k_thicken_adjoint(const float* __restrict__ gvol, float* __restrict__ gvn, const int* __restrict__ off,
                                  const int* __restrict__ ridx, const float* __restrict__ w, int nxy, int nz) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)nxy * nz) return;
  const int n = (int)(i / nxy);
  const long px = i % nxy;
  float acc = 0.0f;
  for (int e = off[n]; e < off[n + 1]; e++) acc = fmaf(w[e], gvol[(size_t)ridx[e] * nxy + px], acc);
  gvn[i] = acc;
}

// ---------------------------------------------------------------------------
// rebin adjoint
// ---------------------------------------------------------------------------
// Forward (rebin_sample, k_stages.cu): output sample (v, i, c) is the
// bilinear texel sample of raw row nr-1-i at sheet column bidx[c] and sheet
// view aidx(v, c), clamp addressing, sheet column x <- raw channel nch-1-x.
// Column lists: sheet column x receives weight wx from channel c when one of
// c's two clamped column taps is x (both taps, when they clamp to the same
// column). Built once per context by k_rebin_adj_cols.
__global__ void k_rebin_adj_cols(const float* __restrict__ bidx_t, int nch, int q8, int* __restrict__ cnt,
                                 int* __restrict__ cidx, float* __restrict__ cw, int maxl, int* __restrict__ err) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= nch) return;
  int n = 0;
  // bidx is monotone in c with slope >= 1, so the channels reaching x lie near x
  for (int c = 0; c < nch; c++) {
    const float b = bidx_t[c];
    if (isnan(b)) continue;
    const float xb = (b + 0.5f) - 0.5f;
    const float fx = floorf(xb);
    float ax = xb - fx;
    if (q8) ax = rintf(ax * 256.0f) * (1.0f / 256.0f);
    const int x0 = min(max((int)fx, 0), nch - 1), x1 = min(max((int)fx + 1, 0), nch - 1);
    float wgt = 0.0f;
    if (x0 == x) wgt += 1.0f - ax;
    if (x1 == x) wgt += ax;
    if (x0 != x && x1 != x) continue;
    if (n == maxl) {
      atomicOr(err, WFBP_ERRBIT_ADJ_LIST);
      break;
    }
    cidx[x * maxl + n] = c;
    cw[x * maxl + n] = wgt;
    n++;
  }
  cnt[x] = n;
}

// Weight with which sheet view y enters output view v's sample of channel
// (fan angle beta): the transposed row taps of rebin_sample.
__device__ __forceinline__ float rebin_view_weight(int v, int y, float beta, float dth, int V, int q8, int voff) {
  const float theta = (float)(v + voff) * dth;
  const float alpha = theta - beta;
  const float aidx = alpha / dth;
  const float yb = (aidx + 0.5f) - 0.5f;
  const float fy = floorf(yb);
  float ay = yb - fy;
  if (q8) ay = rintf(ay * 256.0f) * (1.0f / 256.0f);
  const int y0 = min(max((int)fy - voff, 0), V - 1), y1 = min(max((int)fy + 1 - voff, 0), V - 1);
  float w = 0.0f;
  if (y0 == y) w += 1.0f - ay;
  if (y1 == y) w += ay;
  return w;
}

// One thread per raw sample (reading y, raw row, raw channel).
__global__ void k_rebin_adjoint(const float* __restrict__ gR, float* __restrict__ graw, const float* __restrict__ beta_t,
                                const int* __restrict__ cnt, const int* __restrict__ cidx, const float* __restrict__ cw,
                                int maxl, RebinParams p) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)p.V * p.nr * p.nch;
  if (i >= total) return;
  const int xr = (int)(i % p.nch);
  const int rr = (int)((i / p.nch) % p.nr);
  const int y = (int)(i / ((long)p.nch * p.nr));
  const int x = p.nch - 1 - xr;   // sheet column
  const int row = p.nr - 1 - rr;  // sheet row index i of the output
  float acc = 0.0f;
  const int n = cnt[x];
  for (int e = 0; e < n; e++) {
    const int c = cidx[x * maxl + e];
    const float wx = cw[x * maxl + e];
    const float beta = __ldg(beta_t + c);
    const float sh = beta / p.dth;  // aidx ~ v - sh
    int v_lo = (int)floorf((float)y + sh) - 2, v_hi = (int)ceilf((float)y + sh) + 2;
    if (y == 0) v_lo = 0;            // every view whose taps clamp to the first reading
    if (y == p.V - 1) v_hi = p.V - 1;  // ... or to the last
    if (y == 0) v_hi = max(v_hi, (int)ceilf(sh) + 2);
    if (y == p.V - 1) v_lo = min(v_lo, (int)floorf((float)(p.V - 1) + sh) - 2);
    v_lo = max(v_lo, 0);
    v_hi = min(v_hi, p.V - 1);
    float sum = 0.0f;
    for (int v = v_lo; v <= v_hi; v++) {
      const float wy = rebin_view_weight(v, y, beta, p.dth, p.V, p.q8, p.voff);
      if (wy != 0.0f) sum = fmaf(wy, __ldg(gR + ((size_t)v * p.nr + row) * p.nch + c), sum);
    }
    acc = fmaf(wx, sum, acc);
  }
  graw[i] = acc;
}

// ---------------------------------------------------------------------------
// filter-tap gradient, with the rebinned rows recomputed on the fly
// ---------------------------------------------------------------------------
// Forward: y[n] = sum_m h[|n - m|] x[m] over the nch channels of each row.
// dL/dh[0] = sum_rows sum_n g[n] x[n]; dL/dh[d] = sum_rows sum_n g[n] (x[n-d] + x[n+d]).
// A CTA takes TG_ROWS rows and recomputes their rebinned samples x from the
// raw readings into shared memory (nothing of the rebinned array is stored).
// Thread (tap group, row) correlates its row for TG_TAPS consecutive taps d0..
// d0+3: one gradient load and two sliding-window loads of x feed 8 FMAs per
// channel. The rows of a CTA (8 consecutive lanes) are summed with shuffles
// in a fixed order, and the per-CTA partial sums by k_taps_reduce, so the
// result does not depend on scheduling.
constexpr int TG_ROWS = 8;
constexpr int TG_TAPS = 4;
constexpr int TG_THREADS = 128;  // 16 tap groups x 8 rows

__global__ void __launch_bounds__(TG_THREADS)
k_taps_grad(const float* __restrict__ raw, const float* __restrict__ gY, const float* __restrict__ beta_t,
            const float* __restrict__ bidx_t, RebinParams p, int ntaps, float* __restrict__ partial) {
  extern __shared__ float sm[];
  const int ns = p.nch | 1;               // odd row stride: the 8 rows of a warp fall in different banks
  float* xs = sm;                         // [TG_ROWS][ns]
  float* gs = sm + TG_ROWS * ns;          // [TG_ROWS][ns]
  const long m0 = (long)blockIdx.x * TG_ROWS;
  const long M = (long)p.V * p.nr;
  const int rows = (int)min((long)TG_ROWS, M - m0);
  for (int e = threadIdx.x; e < TG_ROWS * p.nch; e += TG_THREADS) {
    const int rr = e / p.nch, c = e % p.nch;
    const long m = m0 + rr;
    float xv = 0.0f, gv = 0.0f;  // rows past the end contribute nothing
    if (rr < rows) {
      const int v = (int)(m / p.nr), i = (int)(m % p.nr);
      xv = wfbp_rebin_sample(raw, p, __ldg(bidx_t + c), __ldg(beta_t + c), v, i);
      gv = __ldg(gY + m * p.nch + c);
    }
    xs[rr * ns + c] = xv;
    gs[rr * ns + c] = gv;
  }
  __syncthreads();
  const int rr = threadIdx.x % TG_ROWS;
  const float* xr = xs + rr * ns;
  const float* gr = gs + rr * ns;
  const int ngroups = (ntaps + TG_TAPS - 1) / TG_TAPS;
  // every lane of a warp runs the same number of group iterations (the shuffles below)
  for (int g0 = 0; g0 < ngroups; g0 += TG_THREADS / TG_ROWS) {
    const int gi = g0 + threadIdx.x / TG_ROWS;
    const int d0 = gi * TG_TAPS;
    float af[TG_TAPS], ab[TG_TAPS], wf[TG_TAPS], wb[TG_TAPS];
#pragma unroll
    for (int k = 0; k < TG_TAPS; k++) {
      af[k] = ab[k] = 0.0f;
      wf[k] = 0.0f;  // wf[k] = x[n - d0 - k]
      const int jb = d0 + k;
      wb[k] = jb < p.nch ? xr[jb] : 0.0f;  // wb[k] = x[n + d0 + k]
    }
    if (gi < ngroups) {
      for (int n = 0; n < p.nch; n++) {
        const float g = gr[n];
        // slide the forward window: wf[k] = x[n - d0 - k]
#pragma unroll
        for (int k = TG_TAPS - 1; k > 0; k--) wf[k] = wf[k - 1];
        wf[0] = n - d0 >= 0 ? xr[n - d0] : 0.0f;
#pragma unroll
        for (int k = 0; k < TG_TAPS; k++) {
          af[k] = fmaf(g, wf[k], af[k]);
          ab[k] = fmaf(g, wb[k], ab[k]);
        }
        // slide the backward window to n + 1: wb[k] = x[n + 1 + d0 + k]
#pragma unroll
        for (int k = 0; k < TG_TAPS - 1; k++) wb[k] = wb[k + 1];
        const int jb = n + 1 + d0 + TG_TAPS - 1;
        wb[TG_TAPS - 1] = jb < p.nch ? xr[jb] : 0.0f;
      }
    }
#pragma unroll
    for (int k = 0; k < TG_TAPS; k++) {
      // dL/dh[0] counts the product once, dL/dh[d > 0] both neighbours
      float v = d0 + k == 0 ? af[k] : af[k] + ab[k];
#pragma unroll
      for (int o = TG_ROWS / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (rr == 0 && gi < ngroups && d0 + k < ntaps) partial[(size_t)blockIdx.x * ntaps + d0 + k] = v;
    }
  }
}

// One CTA per tap: thread i sums partials i, i + TR_THREADS, ... in double,
// then a tree over the threads in a fixed order (deterministic).
constexpr int TR_THREADS = 256;

__global__ void __launch_bounds__(TR_THREADS)
k_taps_reduce(const float* __restrict__ partial, int nblk, int ntaps, float* __restrict__ out) {
  __shared__ double red[TR_THREADS];
  const int d = blockIdx.x;
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblk; b += TR_THREADS) acc += (double)partial[(size_t)b * ntaps + d];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = TR_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[d] = (float)red[0];
}

}  // namespace

cudaError_t launch_bp_adjoint(const float* gvol, float* gD, const float2* sc, const float* vz, const float* zs,
                              const BPParams& p, float z0, float dzs, float* scale_table, bool fill_table,
                              float* gvol_t, cudaStream_t s) {
  if (scale_table && fill_table) {
    dim3 g((unsigned)((p.nx + AN_TX - 1) / AN_TX), (unsigned)((p.ny + AN_TY - 1) / AN_TY),
           (unsigned)((p.nz + AN_ZS - 1) / AN_ZS));
    k_bp_adjoint_scale<<<g, AN_TX * AN_TY, 0, s>>>(scale_table, sc, vz, zs, p, bp_adjoint_nzp(p.nz));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  dim3 grid((unsigned)((p.nch + AD_CH - 2) / (AD_CH - 1)), (unsigned)p.V);
  const size_t smem = (size_t)p.nr * AD_CH * sizeof(float2);
  auto kern = scale_table ? k_bp_adjoint<true> : k_bp_adjoint<false>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  if (scale_table) {
    // the gradient volume with the table's layout [y][x][nzp]
    const int nzp = bp_adjoint_nzp(p.nz);
    const long n = (long)p.nx * p.ny * nzp;
    k_adj_gvol_t<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(gvol, gvol_t, p.nx * p.ny, p.nz, nzp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    gvol = gvol_t;
  }
  kern<<<grid, AD_CH, smem, s>>>(gvol, scale_table, gD, sc, vz, zs, p, z0, dzs, bp_adjoint_nzp(p.nz));
  return cudaGetLastError();
}

cudaError_t launch_thicken_adjoint(const float* gvol, float* gvn, const int* off, const int* ridx, const float* w,
                                   int nxy, int nz, cudaStream_t s) {
  const long n = (long)nxy * nz;
  k_thicken_adjoint<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(gvol, gvn, off, ridx, w, nxy, nz);
  return cudaGetLastError();
}

cudaError_t launch_rebin_adj_cols(const float* bidx, int nch, int q8, int* cnt, int* cidx, float* cw, int maxl,
                                  int* err, cudaStream_t s) {
  k_rebin_adj_cols<<<(nch + 127) / 128, 128, 0, s>>>(bidx, nch, q8, cnt, cidx, cw, maxl, err);
  return cudaGetLastError();
}

cudaError_t launch_rebin_adjoint(const float* gR, float* graw, const float* beta, const int* cnt, const int* cidx,
                                 const float* cw, int maxl, const RebinParams& p, cudaStream_t s) {
  const long n = (long)p.V * p.nr * p.nch;
  k_rebin_adjoint<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(gR, graw, beta, cnt, cidx, cw, maxl, p);
  return cudaGetLastError();
}

int taps_grad_blocks(const RebinParams& p) { return (int)(((long)p.V * p.nr + TG_ROWS - 1) / TG_ROWS); }

cudaError_t launch_taps_gradient(const float* raw, const float* gY, const float* beta, const float* bidx,
                                 const RebinParams& p, int ntaps, float* partial, float* out, cudaStream_t s) {
  const int nblk = taps_grad_blocks(p);
  const size_t smem = (size_t)2 * TG_ROWS * (p.nch | 1) * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_taps_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_taps_grad<<<nblk, TG_THREADS, smem, s>>>(raw, gY, beta, bidx, p, ntaps, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_taps_reduce<<<ntaps, TR_THREADS, 0, s>>>(partial, nblk, ntaps, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// self-test of the bounded waits
// ---------------------------------------------------------------------------
#include "wait.cuh"

namespace {
// Waits on an mbarrier that nothing ever arrives at, with a limit of
// limit_ns; when the wait gives up (as it must) the error word is set to
// WFBP_ERR_TIMEOUT, exactly as a stalled pipeline in the production kernels
// reports itself.
__global__ void k_selftest_wait(int* err, unsigned long long limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(&bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !wfbp_mbar_wait(&bar, 0, limit_ns)) atomicExch(err, WFBP_ERR_TIMEOUT);
}
}  // namespace

cudaError_t launch_selftest_wait(int* err, unsigned long long limit_ns, cudaStream_t s) {
  k_selftest_wait<<<1, 32, 0, s>>>(err, limit_ns);
  return cudaGetLastError();
}
