// Helical Q-weighted backprojection, TMA-staged (sm_100a).
//
// Same algorithm as backproject_kernel (cuda_kernels.cuh:198-287) and
// k_bp (k_backproject.cu); this kernel is organised for throughput:
//
//  * Lanes are slices. A warp owns CPW (x, y) columns and the SL consecutive
//    native slices of a slab (SL = 32, or 16 with the warp's lanes 0-15 and
//    16-31 on two groups of CPW / 2 columns); lane l holds slice s0 + l % SL
//    of its group's columns. The geometry of a (column, view) pair -- p_hat,
//    l_hat, the asin term, the channel index and weight, and the row
//    coordinate as a linear function of z -- is computed once, by one lane,
//    and broadcast to the group's lanes through shared memory.
//  * Filtered rows are read in the backprojection layout [view][channel][row]
//    (rows contiguous), so the lanes of a column group, which sit at
//    consecutive rows of the same two channels, read consecutive shared-memory
//    words.
//  * A producer warp walks the half-turn angles theta~ and, for each, selects
//    the views j = theta~ + k P/2 whose table position can reach the CTA's
//    slab (the reference's z cull, cuda_kernels.cuh:232, and the detector's
//    cone), and TMA-loads the channel window each view needs for the CTA's
//    column tile (all rows) into a 2-stage mbarrier ring.
//  * For every column the NW consumer warps accumulate sum(W g) and sum(W)
//    over the staged views of theta~ and add (2 pi/P) sum(W g)/sum(W) to the
//    column's slice in registers (NaN when no view contributes, like the
//    reference). In wfbp_run the write-back also forms the requested slices
//    that lie inside the slab (fused thickening, bp_fused_thicken).
//
// Element types: float (FP32 rows) or uint32_t holding half2 pairs
// (row r, row r+1) of FP16 rows divided by one power of two for the whole
// scan, which the host folds into the write-back's 2 pi / P.
//
// Every mbarrier wait is bounded; on timeout the CTA records WFBP_ERR_TIMEOUT
// in the error word and stops. Window or slot overflows (which the host's
// sizing rules out) are recorded as well and the affected samples skipped.
#include "wfbp_internal.h"
#include "bp_math.cuh"
#include "wait.cuh"

#include <cuda.h>

#include <algorithm>
#include <cstring>

#include <type_traits>

namespace {


__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait on phase parity (wait.cuh); false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) { return wfbp_mbar_wait(bar, parity); }

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Geometry of a pair of columns for one view, stored so that 16-byte
// shared-memory loads give both columns' fields as float2 operands of the
// packed FP32x2 instructions (FFMA2 / FADD2 / FMUL2). GeoP carries the row
// range the table-position cull leaves (cuda_kernels.cuh:232); when the
// host has shown that the cull never removes a sample whose row lies in
// [0, nr - 2] (the detector's cone is shorter than z_rot), that range is
// [0, nr - 2] for every record, GeoQ drops it and the test uses its centre
// and half width (nr - 2) / 2 as constants: the same compare on the same
// values, so both records give the same samples.
struct __align__(16) GeoP {
  float2 bq, cq;    // q(z) = bq z + cq
  float2 qmid, qhw;  // valid for |q - qmid| <= qhw (the row range [qlo, qhi] as centre and half width)
  int2 addr;        // shared-memory byte offset of (channel pf, row 0) of the view's slot
  float2 wp;        // FP32 rows: channel weight; half2 pairs: bits of the half2 (wp, wp)
};
struct __align__(16) GeoQ {
  float2 bq, cq;    // q(z) = bq z + cq (an invalid record: bq = 0, cq = -1e30)
  int2 addr;
  float2 wp;
};
static_assert(sizeof(GeoP) == BP_GEO_BYTES_ZCULL && sizeof(GeoQ) == BP_GEO_BYTES, "record sizes of bp_smem_layout");

__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// Shared memory of a CTA: the mbarriers and small words at fixed offsets
// (they persist across the tiles of a persistent launch), then the regions
// of bp_smem_layout for the tile's scan.
// int [16]: [0..1] views per stage, [8] failure flag, [9] next item, [10] fused-thickening words
constexpr int BT_OFF_NVS = 64;

__device__ __forceinline__ void bp_init_barriers(uint8_t* smem, int nw) {
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  if (threadIdx.x == 0) {
    reinterpret_cast<int*>(smem + BT_OFF_NVS)[8] = 0;
    reinterpret_cast<int*>(smem + BT_OFF_NVS)[10] = 0;
    for (int s = 0; s < BT_STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&full[BT_STAGES + s], nw);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
}

// Fused thickening of one slab (ThickFuse). The producer warp has copied the
// slab's records into shared memory (fz, nfz words) while the ring filled.
// For every interior requested slice r each group of SL lanes (lane = slice
// s0 + lane % SL) gathers its native values with shuffles, in the CSR order
// and with the same FMA chain and division as k_thicken, so the result is
// bit-identical to thickening the written native volume. Lane c of a group
// writes column c of the group. All 32 lanes of the warp take part.
template <int CPW, int SL, int CPG>
__device__ __forceinline__ void bp_fused_thicken(const ThickFuse& tf, const float (&vals)[CPG], const int* fz,
                                                 int nfz, int warp, int lane, int ix0, int iy0, const BPTile& bt,
                                                 const BPParams& p) {
  const int grp = lane / SL, ll = lane % SL;
  const int tt = warp * CPW + grp * CPG + min(ll, CPG - 1);
  const int ix = ix0 + tt % bt.tx, iy = iy0 + tt / bt.tx;
  const bool wr = ll < CPG && ix < p.nx && iy < p.ny;
  const size_t plane = (size_t)p.nx * p.ny, vox = (size_t)iy * p.nx + ix;
  nfz = min(nfz, BT_FUSE_WORDS);
  for (int pos = 0; pos + 3 <= nfz;) {
    const int r = fz[pos], n = fz[pos + 1];
    const float ws = __int_as_float(fz[pos + 2]);
    if (n < 0 || pos + 3 + 2 * n > nfz) break;  // malformed records (host sizing guarantees otherwise)
    float acc[CPG];
#pragma unroll
    for (int c = 0; c < CPG; c++) acc[c] = 0.0f;
    for (int e = 0; e < n; e++) {
      const int src = grp * SL + (fz[pos + 3 + 2 * e] & (SL - 1));
      const float wt = __int_as_float(fz[pos + 4 + 2 * e]);
#pragma unroll
      for (int c = 0; c < CPG; c++) acc[c] = fmaf(wt, __shfl_sync(0xffffffffu, vals[c], src), acc[c]);
    }
    float v = 0.0f;
#pragma unroll
    for (int c = 0; c < CPG; c++)
      if (c == ll) v = acc[c];
    if (wr && r >= 0 && r < tf.nzr) tf.out[(size_t)r * plane + vox] = v / ws;
    pos += 3 + 2 * n;
  }
}

// The same for a tile outside the FOV, whose native values are all +0:
// k_thicken gives +0 / sum of weights = +0 for every interior slice.
template <int CPW, int SL, int CPG>
__device__ __forceinline__ void bp_fused_zero(const ThickFuse& tf, int bz, int warp, int lane, int ix0, int iy0,
                                              const BPTile& bt, const BPParams& p) {
  const int2 rr = tf.slab_req[bz];
  const int grp = lane / SL, ll = lane % SL;
  const int tt = warp * CPW + grp * CPG + min(ll, CPG - 1);
  const int ix = ix0 + tt % bt.tx, iy = iy0 + tt / bt.tx;
  const bool wr = ll < CPG && ix < p.nx && iy < p.ny;
  const size_t plane = (size_t)p.nx * p.ny, vox = (size_t)iy * p.nx + ix;
  for (int k0 = rr.x; k0 < rr.y; k0 += 32) {
    const int mine = k0 + lane < rr.y ? __ldg(tf.req + k0 + lane) : -1;  // one load per lane
    const int cnt = min(32, rr.y - k0);
    for (int k = 0; k < cnt; k++) {
      const int r = __shfl_sync(0xffffffffu, mine, k);
      if (wr && r >= 0 && r < tf.nzr) tf.out[(size_t)r * plane + vox] = 0.0f;
    }
  }
}

// One column tile (bt.tx x bt.ty columns, SL slices from slab bz) of one scan.
// `ring` counts the theta~ steps this CTA has run through its two-stage
// ring before this tile (stage = ring & 1, phase = (ring >> 1) & 1), so a
// persistent CTA continues the barriers' phases from tile to tile. Returns
// the number of ring steps the tile used: p.P2, or 0 for a tile entirely
// outside the reconstruction FOV (whose voxels are written as 0, the value
// the reference leaves there). A bounded wait that gave up sets the failure
// word (the CTA must stop).
template <typename T, int CPW, int CU, int NW, int SL, bool ZC, bool COUNT, bool FUSE>
__device__ __forceinline__ int bp_tile(const CUtensorMap* map, float* __restrict__ vol,
                                        const float2* __restrict__ view_sc, const float* __restrict__ view_z,
                                        const float* __restrict__ zslices,
                                        const BPParams& p, const BPTile& bt, int bx, int by, int bz,
                                        unsigned long long* __restrict__ count, int* __restrict__ err, uint8_t* smem,
                                        uint32_t ring, const ThickFuse& tf) {
  constexpr bool HALF = !std::is_same<T, float>::value;
  using Geo = typename std::conditional<ZC, GeoP, GeoQ>::type;
  constexpr int NPW = CPW / 2;  // column pairs per warp
  // SL = 32: the warp's 32 lanes are 32 slices of each of its CPW columns.
  // SL = 16: lanes 0-15 and 16-31 are 16 slices of two column groups of
  // CPW / 2 columns each (a 16-slice slab: fewer lanes outside a view's cone).
  constexpr int NG = 32 / SL, CPG = CPW / NG;  // column groups per warp, columns per group
  static_assert(SL == 32 || SL == 16, "slab of 32 or 16 slices");
  static_assert(CU % 2 == 0 && CPG % CU == 0, "columns per step must be even and divide the columns per group");
  const BpSmem L = bp_smem_layout(bt, CPW);  // bt.zc == ZC (the launch picks the instantiation)
  uint8_t* slots = smem + L.slots;                            // [STAGES][nv_max][slot_bytes]
  int2* vinfo = reinterpret_cast<int2*>(smem + L.vinfo);      // [STAGES][nv_max] (view, first channel)
  BpViewGeo* vgeo = reinterpret_cast<BpViewGeo*>(smem + L.vgeo);  // [STAGES][nv_max] the views' angle and z
  int* nvs = reinterpret_cast<int*>(smem + BT_OFF_NVS);       // [STAGES] views, [8] failure flag
  Geo* geo = reinterpret_cast<Geo*>(smem + L.geo);            // [warps][nv_max][NPW]
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + BT_STAGES;
  volatile int* s_fail = nvs + 8;

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int ix0 = bx * bt.tx, iy0 = by * bt.ty;
  const int s0 = bz * SL;
  const int grp = lane / SL;  // column group of this lane

  // slab z range (all warps and groups compute the same values)
  const int my_s = s0 + lane % SL;
  const float zl = my_s < p.nz ? zslices[my_s] : __int_as_float(0x7fc00000);
  float zmn = my_s < p.nz ? zl : 3.0e38f, zmx = my_s < p.nz ? zl : -3.0e38f;
#pragma unroll
  for (int o = SL / 2; o > 0; o >>= 1) {
    zmn = fminf(zmn, __shfl_xor_sync(0xffffffffu, zmn, o));
    zmx = fmaxf(zmx, __shfl_xor_sync(0xffffffffu, zmx, o));
  }

  const float nxm = 0.5f * ((float)p.nx - 1.0f), nym = 0.5f * ((float)p.ny - 1.0f);
  auto xcoord = [&](int ix) { return ((float)ix - nxm) * p.fov / (float)p.nx + p.x0; };
  auto ycoord = [&](int iy) { return ((float)iy - nym) * p.fov / (float)p.ny + p.y0; };

  {
    // the voxel centre of the tile nearest the isocentre; with a margin for
    // rounding, a tile beyond the FOV circle holds no voxel the reference
    // backprojects (cuda_kernels.cuh:220)
    const float xa = xcoord(ix0), xb = xcoord(min(ix0 + bt.tx - 1, p.nx - 1));
    const float ya = ycoord(iy0), yb = ycoord(min(iy0 + bt.ty - 1, p.ny - 1));
    const float xn = fminf(fmaxf(0.0f, xa), xb), yn = fminf(fmaxf(0.0f, ya), yb);
    if (xn * xn + yn * yn > p.fov_half2 * 1.0001f + 1e-3f) {
      if (warp < NW && my_s < p.nz) {
        const size_t plane = (size_t)p.nx * p.ny;
        for (int c = 0; c < CPG; c++) {
          const int tt = warp * CPW + grp * CPG + c;
          const int ix = ix0 + tt % bt.tx, iy = iy0 + tt / bt.tx;
          if (ix < p.nx && iy < p.ny) vol[(size_t)my_s * plane + (size_t)iy * p.nx + ix] = 0.0f;
        }
      }
      if (FUSE && tf.out && warp < NW) bp_fused_zero<CPW, SL, CPG>(tf, bz, warp, lane, ix0, iy0, bt, p);
      return 0;
    }
  }

  if (warp == NW) {
    // ---------------- producer ----------------
    // The 32 lanes test the half turns k of theta~ in parallel (lane = k
    // mod 32), the selected views are compacted in k order with a ballot, and
    // their copies are issued by as many lanes.
    const float zlo = zmn - bt.reach, zhi = zmx + bt.reach;
    const float xa = xcoord(ix0), xb = xcoord(min(ix0 + bt.tx - 1, p.nx - 1));
    const float ya = ycoord(iy0), yb = ycoord(min(iy0 + bt.ty - 1, p.ny - 1));
    const uint32_t view_bytes = (uint32_t)(bt.W * bt.nrp * sizeof(T));
    const unsigned below = (1u << lane) - 1u;
    int issued_upto = 0;
    bool failed = false;
    for (int t = 0; t < p.P2; t++) {
      const uint32_t g = ring + (uint32_t)t;
      const int s = (int)(g & 1u);
      const uint32_t u = g >> 1;
      int ok = 1;
      if (lane == 0) ok = (u < 1 || mbar_wait(&empty[s], (u - 1) & 1)) && !*s_fail;
      if (!__shfl_sync(0xffffffffu, ok, 0)) {
        failed = true;
        break;
      }
      if (FUSE && tf.out && t == min(1, p.P2 - 1)) {
        // the slab's fused-thickening records, copied while the consumers work
        // on the first stage and published by this stage's full-barrier arrive
        const int2 fr = tf.slab_tab[bz];
        const int nw = max(0, min(fr.y - fr.x, BT_FUSE_WORDS));
        int* fz = reinterpret_cast<int*>(smem + L.fuse);
        for (int j = lane; j < nw; j += 32) fz[j] = __ldg(tf.tab + fr.x + j);
        if (lane == 0) nvs[10] = nw;
        __syncwarp();
      }
      int nv = 0;
      for (int kb = 0; kb < p.K; kb += 32) {
        const int k = kb + lane;
        const int j = t + k * p.P2;
        bool sel = false;
        int c_lo = 0;
        float4 vf = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // FP32 form: the view's sin, cos, z for the records
        if (k < p.K) {
          const float zt = __ldg(view_z + j);
          const float2 sc = __ldg(view_sc + j);
          vf = make_float4(sc.x, sc.y, zt, 0.0f);
          if (!(zt < zlo || zt > zhi)) {
            const float p1 = xa * sc.x - ya * sc.y, p2 = xa * sc.x - yb * sc.y;
            const float p3 = xb * sc.x - ya * sc.y, p4 = xb * sc.x - yb * sc.y;
            const float pmax = fmaxf(fmaxf(p1, p2), fmaxf(p3, p4));
            const float pmin = fminf(fminf(p1, p2), fminf(p3, p4));
            // rows this tile can use: q in [0, nr-2] needs |z - zt + A| <= l_hat tan,
            // with l_hat <= R - min(t) over the tile and A monotonic in p_hat
            const float t1 = xa * sc.y + ya * sc.x, t2 = xa * sc.y + yb * sc.x;
            const float t3 = xb * sc.y + ya * sc.x, t4 = xb * sc.y + yb * sc.x;
            const float lhi = sqrtf(p.R2) - fminf(fminf(t1, t2), fminf(t3, t4));
            const float amin = p.zr2pi * asinf(p.rR * pmin), amax = p.zr2pi * asinf(p.rR * pmax);
            const float eps = 1e-3f * (1.0f + fabsf(zt));
            const float wlo = zt - amax - lhi * p.tanc - eps, whi = zt - amin + lhi * p.tanc + eps;
            sel = !(whi < zmn || wlo > zmx);
            const float idx_min = p.kp - (pmax * p.ps + p.c0);  // p_idx decreases with p_hat
            c_lo = max(0, min((int)floorf(idx_min) - 1, p.nch - bt.W));
          }
        }
        const unsigned m = __ballot_sync(0xffffffffu, sel);
        const int pos = nv + __popc(m & below);
        if (sel) {
          if (pos < bt.nv_max) {
            vinfo[s * bt.nv_max + pos] = make_int2(j, c_lo);
            // the view's angle and z for the consumers' record pass (the
            // mixed form's FP64 tables; the FP32 form's values of the test)
            BpViewGeo* g = vgeo + s * bt.nv_max + pos;
            if constexpr (HALF) {
              const double2 sc64 = __ldg(p.sc64 + j);
              const double z64 = __ldg(p.z64 + j);
              g->s = sc64.x;
              g->c = sc64.y;
              g->z = z64;
            } else {
              *reinterpret_cast<float4*>(g) = vf;
            }
          } else {
            atomicOr(err, WFBP_ERRBIT_BP_SLOTS);  // more views than slots: host sizing violated
          }
        }
        nv = min(nv + __popc(m), bt.nv_max);
      }
      __syncwarp();
      if (lane == 0) {
        nvs[s] = nv;
        mbar_arrive_tx(&full[s], (uint32_t)nv * view_bytes);
      }
      __syncwarp();
      for (int v = lane; v < nv; v += 32) {
        const int2 vi = vinfo[s * bt.nv_max + v];
        tma_load_3d(slots + ((size_t)s * bt.nv_max + v) * bt.slot_bytes, map, &full[s], 0, vi.y, vi.x);
      }
      issued_upto = t + 1;
    }
    if (failed && lane == 0) {
      *s_fail = 1;
      atomicExch(err, WFBP_ERR_TIMEOUT);
      // let copies already issued land before the CTA's shared memory goes away
      for (int t = max(0, issued_upto - BT_STAGES); t < issued_upto; t++) {
        const uint32_t g = ring + (uint32_t)t;
        mbar_wait(&full[g & 1u], (g >> 1) & 1u);
      }
    }
    return p.P2;
  }

  // ---------------- consumers ----------------
  float2 vacc[CPG / 2];  // columns (2i, 2i + 1) of this lane's group
#pragma unroll
  for (int c = 0; c < CPG / 2; c++) vacc[c] = make_float2(0.0f, 0.0f);
  unsigned long long cnt = 0;
  const float k1 = 2.5f / p.hn;
  Geo* wgeo = geo + (size_t)warp * bt.nv_max * NPW;
  constexpr int VPP = 32 / CPW;  // views per geometry pass
  const int gc = lane % CPW, gv = lane / CPW;
  const int gt = warp * CPW + gc;  // tile column handled by this lane in geometry passes
  const int gix = ix0 + gt % bt.tx, giy = iy0 + gt / bt.tx;
  const float gx = xcoord(gix), gy = ycoord(giy);
  const bool gactive = gix < p.nx && giy < p.ny && !(gx * gx + gy * gy > p.fov_half2);
  unsigned active_mask = 0;  // bit c: column c of this warp is inside the grid and the FOV
#pragma unroll
  for (int c = 0; c < CPW; c++) active_mask |= (__shfl_sync(0xffffffffu, gactive ? 1u : 0u, c) & 1u) << c;
  const int nrpb = bt.nrp * 4;  // bytes between channels of a slot
  const float2 zl2 = make_float2(zl, zl);
  const float2 mhn2 = make_float2(-p.hn, -p.hn);
  const float2 pi2 = make_float2(3.14159265f, 3.14159265f);
  const float2 half2c = make_float2(0.5f, 0.5f);
  const unsigned nrm2u = (unsigned)(p.nr - 2);
  const float hrow = 0.5f * p.nrm2;  // rows [0, nr - 2] as centre and half width (records without the cull)
  const float2 mhrow2 = make_float2(-hrow, -hrow);

  for (int t = 0; t < p.P2; t++) {
    const uint32_t g = ring + (uint32_t)t;
    const int s = (int)(g & 1u);
    const uint32_t u = g >> 1;
    if (!mbar_wait(&full[s], u & 1u)) {
      *s_fail = 1;
      atomicExch(err, WFBP_ERR_TIMEOUT);
      break;
    }
    const int nv = nvs[s];
    // geometry of (column gc, view v) for v = gv, gv + VPP, ...
    for (int v = gv; v < nv; v += VPP) {
      const int2 vi = vinfo[s * bt.nv_max + v];
      const BpViewGeo& vg = vgeo[s * bt.nv_max + v];  // the view's angle and z, staged by the producer
      float p_hat, t_hat, zt;
      if constexpr (HALF) {
        // the mixed form's per-view geometry is FP64 (sin, cos and table
        // position of the view, from the FP64 tables of wfbp_set_views)
        const double2 sc = make_double2(vg.s, vg.c);
        const double gxd = (double)gx, gyd = (double)gy;
        p_hat = (float)fma(gxd, sc.x, -gyd * sc.y);
        t_hat = (float)fma(gxd, sc.y, gyd * sc.x);
        zt = (float)vg.z;
      } else {
        const float4 vf = *reinterpret_cast<const float4*>(&vg);
        // x sin - y cos and x cos + y sin (cuda_kernels.cuh:235-238) with one
        // rounding of the second product each, as the FP64 form's
        p_hat = fmaf(gx, vf.x, -(gy * vf.y));
        t_hat = fmaf(gx, vf.y, gy * vf.x);
        zt = vf.z;
      }
      const float l_hat = bp_sqrt(p.R2 - p_hat * p_hat) - t_hat;
      const float A = p.zr2pi * bp_asin(p.rR * p_hat);
      const float inv = bp_rcp(l_hat * p.tanc);
      const float p_idx = p.kp - (p_hat * p.ps + p.c0);
      const float pf = floorf(p_idx);
      // floor(p_idx) >= 0 and ceil(p_idx) <= nch - 2 (cuda_kernels.cuh:259-263)
      bool valid = gactive && p_idx >= 0.0f && p_idx <= p.ncm2;
      const int cofs = (int)pf - vi.y;
      if (valid && (cofs < 0 || cofs > bt.W - 2)) {
        atomicOr(err, WFBP_ERRBIT_BP_WINDOW);  // channel window too narrow: host sizing violated
        valid = false;
      }
      const float bq = inv * p.hn;
      const float cq = p.hn * fmaf(A - zt, inv, 1.0f);
      const float wp = p_idx - pf;
      float* gf = reinterpret_cast<float*>(wgeo + v * NPW + (gc >> 1)) + (gc & 1);
      constexpr int O = ZC ? 4 : 0;  // float offset of addr / wp behind the row range
      if constexpr (ZC) {
        gf[0] = bq;
        gf[2] = cq;
        // rows q in [0, nr - 2] (cuda_kernels.cuh:259-263) of views within z_rot (:232)
        const float qlo = fmaxf(0.0f, fmaf(zt - p.z_rot, bq, cq)), qhi = fminf(p.nrm2, fmaf(zt + p.z_rot, bq, cq));
        gf[4] = valid ? 0.5f * (qlo + qhi) : 0.0f;
        gf[6] = valid ? 0.5f * (qhi - qlo) : -1.0f;
      } else {
        // rows q in [0, nr - 2] (cuda_kernels.cuh:259-263); an invalid record
        // gives every lane q = -1e30, outside the rows, and finite row weights
        // (a NaN q would make 0 x NaN in the column's sums)
        gf[0] = valid ? bq : 0.0f;
        gf[2] = valid ? cq : -1.0e30f;
      }
      reinterpret_cast<int*>(gf)[4 + O] =
          (int)(L.slots + (size_t)(s * bt.nv_max + v) * bt.slot_bytes) + (valid ? cofs : 0) * nrpb;
      if constexpr (HALF) {
        const __half2 w2 = __float2half2_rn(wp);
        gf[6 + O] = __uint_as_float(*reinterpret_cast<const uint32_t*>(&w2));
      } else {
        gf[6 + O] = wp;
      }
    }
    __syncwarp();
#pragma unroll
    for (int c0 = 0; c0 < CPG; c0 += CU) {
      unsigned any = 0u;  // warp-uniform: some group has an active column in this step
#pragma unroll
      for (int g2 = 0; g2 < NG; g2++) any |= (active_mask >> (g2 * CPG + c0)) & ((1u << CU) - 1u);
      if (!any) continue;
      float2 ag[CU / 2], aw[CU / 2];
#pragma unroll
      for (int u2 = 0; u2 < CU / 2; u2++) {
        ag[u2] = make_float2(0.0f, 0.0f);
        aw[u2] = make_float2(0.0f, 0.0f);
      }
      for (int v = 0; v < nv; v++) {
        const Geo* gpv = wgeo + v * NPW + (grp * CPG + c0) / 2;
#pragma unroll
        for (int u2 = 0; u2 < CU / 2; u2++) {
          const Geo g = gpv[u2];
          const float2 q = __ffma2_rn(zl2, g.bq, g.cq);
          bool okx, oky;
          if constexpr (ZC) {
            const float2 dq = __fadd2_rn(q, neg2(g.qmid));
            okx = fabsf(dq.x) <= g.qhw.x;
            oky = fabsf(dq.y) <= g.qhw.y;
          } else {
            const float2 dq = __fadd2_rn(q, mhrow2);
            okx = fabsf(dq.x) <= hrow;
            oky = fabsf(dq.y) <= hrow;
          }
          // Row index and fraction through the FP32 pipe: for 0 <= q < 2^23,
          // q + 2^23 rounded down is 2^23 + floor(q), an integer held in the
          // low mantissa bits, and subtracting 2^23 again is exact. Invalid
          // lanes (weight 0; negative, huge or NaN q) read any in-range row:
          // the unsigned difference of the bit patterns is clamped to nr - 2.
          const float2 tq = __fadd2_rd(q, make_float2(8388608.0f, 8388608.0f));
          const float2 fq = __fadd2_rn(tq, make_float2(-8388608.0f, -8388608.0f));
          const unsigned rx = min(__float_as_uint(tq.x) - 0x4B000000u, nrm2u);
          const unsigned ry = min(__float_as_uint(tq.y) - 0x4B000000u, nrm2u);
          const float2 wq = __fadd2_rn(q, neg2(fq));
          const uint8_t* ex = smem + g.addr.x + (rx << 2);
          const uint8_t* ey = smem + g.addr.y + (ry << 2);
          float2 top, bot;
          if constexpr (!HALF) {
            const float2 d00 = make_float2(*reinterpret_cast<const float*>(ex), *reinterpret_cast<const float*>(ey));
            const float2 d01 =
                make_float2(*reinterpret_cast<const float*>(ex + 4), *reinterpret_cast<const float*>(ey + 4));
            const float2 d10 = make_float2(*reinterpret_cast<const float*>(ex + nrpb),
                                           *reinterpret_cast<const float*>(ey + nrpb));
            const float2 d11 = make_float2(*reinterpret_cast<const float*>(ex + nrpb + 4),
                                           *reinterpret_cast<const float*>(ey + nrpb + 4));
            top = __ffma2_rn(g.wp, __fadd2_rn(d10, neg2(d00)), d00);
            bot = __ffma2_rn(g.wp, __fadd2_rn(d11, neg2(d01)), d01);
          } else {
            // (row r, row r+1) pairs of channels pf and pf+1, interpolated
            // across channels in half2 arithmetic
            const __half2 h0x = *reinterpret_cast<const __half2*>(ex);
            const __half2 h1x = *reinterpret_cast<const __half2*>(ex + nrpb);
            const __half2 h0y = *reinterpret_cast<const __half2*>(ey);
            const __half2 h1y = *reinterpret_cast<const __half2*>(ey + nrpb);
            const uint32_t wbx = __float_as_uint(g.wp.x), wby = __float_as_uint(g.wp.y);
            const __half2 wpx = *reinterpret_cast<const __half2*>(&wbx);
            const __half2 wpy = *reinterpret_cast<const __half2*>(&wby);
            const float2 fx = __half22float2(__hfma2(wpx, __hsub2(h1x, h0x), h0x));
            const float2 fy = __half22float2(__hfma2(wpy, __hsub2(h1y, h0y), h0y));
            top = make_float2(fx.x, fy.x);
            bot = make_float2(fx.y, fy.y);
          }
          const float2 gval = __ffma2_rn(wq, __fadd2_rn(bot, neg2(top)), top);
          // W(q) of cuda_kernels.cuh:79-93 with |q_hat| = |q - hn| / hn
          const float2 a = __fadd2_rn(q, mhn2);
          const float2 tt = __fmul2_rn(make_float2(__saturatef(fmaf(fabsf(a.x), k1, -1.5f)),
                                                   __saturatef(fmaf(fabsf(a.y), k1, -1.5f))),
                                       pi2);
          float2 W = __ffma2_rn(half2c, make_float2(__cosf(tt.x), __cosf(tt.y)), half2c);
          W.x = okx ? W.x : 0.0f;
          W.y = oky ? W.y : 0.0f;
          ag[u2] = __ffma2_rn(W, gval, ag[u2]);
          aw[u2] = __fadd2_rn(aw[u2], W);
          if (COUNT) cnt += (okx ? 1 : 0) + (oky ? 1 : 0);
        }
      }
      // cuda_kernels.cuh:283, vol += (2 pi / P) (sum W g) / (sum W): the
      // quotient through the hardware reciprocal (0 / 0 stays NaN), 2 pi / P
      // (times the FP16 rows' scale) applied once at the write-back
#pragma unroll
      for (int u2 = 0; u2 < CU / 2; u2++)
        vacc[c0 / 2 + u2] = __ffma2_rn(ag[u2], make_float2(bp_rcp(aw[u2].x), bp_rcp(aw[u2].y)), vacc[c0 / 2 + u2]);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }

  // write the slab: columns outside the grid or the FOV keep the 0 the
  // reference leaves there
  const unsigned my_cols = (active_mask >> (grp * CPG)) & ((1u << CPG) - 1u);
  float vals[CPG];
#pragma unroll
  for (int c = 0; c < CPG; c++)
    vals[c] = ((my_cols >> c) & 1u) ? p.dtheta * ((c & 1) ? vacc[c / 2].y : vacc[c / 2].x) : 0.0f;
  if (my_s < p.nz) {
    const size_t plane = (size_t)p.nx * p.ny;
#pragma unroll
    for (int c = 0; c < CPG; c++) {
      const int tt = warp * CPW + grp * CPG + c;
      const int ix = ix0 + tt % bt.tx, iy = iy0 + tt / bt.tx;
      if (ix < p.nx && iy < p.ny) vol[(size_t)my_s * plane + (size_t)iy * p.nx + ix] = vals[c];
    }
  }
  if (FUSE && tf.out)
    bp_fused_thicken<CPW, SL, CPG>(tf, vals, reinterpret_cast<const int*>(smem + L.fuse),
                                   reinterpret_cast<volatile int*>(nvs)[10], warp, lane, ix0, iy0, bt, p);
  if (COUNT) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(count, cnt);
  }
  return p.P2;
}

// CTAs per SM the launch bounds of the one-tile kernel ask for: three 9-warp
// CTAs (their registers, at most 75 per thread, and shared memory fit) for
// four columns per pass or 16-slice slabs, in both forms; eight columns per
// pass over 32-slice slabs would spill at that budget and keep two; the wider
// shapes one. (The persistent batch kernel holds more state per thread:
// three only for four columns per pass over 16-slice slabs.)
template <int NW, int CU, int SL, bool BATCH = false>
constexpr int bp_min_ctas() {
  return NW > 8 ? 1 : (BATCH ? (CU == 4 && SL == 16) : (CU == 4 || SL == 16)) ? 3 : 2;
}

// One tile per CTA: grid (tiles x, tiles y, SL-slice slabs).
template <typename T, int CPW, int CU, int NW, int SL, bool ZC, bool COUNT>
__global__ void __launch_bounds__((NW + 1) * 32, bp_min_ctas<NW, CU, SL>())
k_bp_tma(const __grid_constant__ CUtensorMap map, float* __restrict__ vol, const float2* __restrict__ view_sc,
         const float* __restrict__ view_z, const float* __restrict__ zslices, BPParams p, BPTile bt,
         unsigned long long* __restrict__ count, int* __restrict__ err, ThickFuse tf) {
  // the dynamic shared memory is the only shared memory of this kernel, so
  // it starts at the (128-byte aligned) base of the CTA's window
  extern __shared__ __align__(128) uint8_t smem[];
  bp_init_barriers(smem, NW);
  bp_tile<T, CPW, CU, NW, SL, ZC, COUNT, true>(&map, vol, view_sc, view_z, zslices, p, bt, blockIdx.x, blockIdx.y,
                                 bt.zb0 + blockIdx.z, count, err, smem, 0u, tf);
}

// Persistent launch over the column tiles of several scans: each CTA takes
// the next work item (scan, tile x, tile y, slab) from a global counter until
// the list is exhausted. Items are listed by decreasing estimated cost.
template <typename T, int CPW, int CU, int NW, int SL, bool ZC>
__global__ void __launch_bounds__((NW + 1) * 32, bp_min_ctas<NW, CU, SL, true>())
k_bp_tma_batch(const BpScan* __restrict__ scans, const int4* __restrict__ items, int n_items,
               unsigned* __restrict__ next, int* __restrict__ err) {
  extern __shared__ __align__(128) uint8_t smem[];
  bp_init_barriers(smem, NW);
  volatile int* words = reinterpret_cast<volatile int*>(smem + BT_OFF_NVS);
  uint32_t ring = 0;
  for (;;) {
    if (threadIdx.x == 0) words[9] = (int)atomicAdd(next, 1u);
    __syncthreads();
    const int it = words[9];
    if (it >= n_items || words[8] != 0) break;
    const int4 w = items[it];
    const BpScan* sd = scans + w.x;
    const BPParams p = sd->p;
    const BPTile bt = sd->bt;
    ring += (uint32_t)bp_tile<T, CPW, CU, NW, SL, ZC, false, false>(&sd->map, sd->vol, sd->view_sc, sd->view_z,
                                                 sd->zslices, p, bt, w.y, w.z, w.w, nullptr, err, smem, ring,
                                                 sd->tf);
    __syncthreads();  // the tile's shared memory and words[9] are free again
  }
}

// Dynamic shared memory of `smem` bytes. Shapes meant to run two CTAs per SM
// (8 consumer warps) also ask for the whole unified L1 / shared memory as
// shared memory; the others leave the split to the driver, which keeps more
// L1 for the geometry and view-table loads.
template <int NW, typename K>
cudaError_t prepare_kernel(K* kern, int smem) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess && NW <= 8)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  return e;
}

template <typename T, int CPW, int CU, int NW, int SL, bool ZC>
cudaError_t launch_one(const CUtensorMap& map, float* vol, const float2* sc,
                       const float* vz, const float* zs, const BPParams& p, const BPTile& bt,
                       unsigned long long* count, int* err, cudaStream_t s, const ThickFuse& tf) {
  const int nslab = (p.nz + SL - 1) / SL;
  if (bt.zb0 < 0 || bt.zb0 >= nslab || bt.nzb < 0 || bt.zb0 + bt.nzb > nslab) return cudaErrorInvalidValue;
  dim3 grid((unsigned)((p.nx + bt.tx - 1) / bt.tx), (unsigned)((p.ny + bt.ty - 1) / bt.ty),
            (unsigned)(bt.nzb ? bt.nzb : nslab - bt.zb0));
  constexpr int threads = (NW + 1) * 32;
  cudaError_t e;
  if (count) {
    e = prepare_kernel<NW>(k_bp_tma<T, CPW, CU, NW, SL, ZC, true>, bt.smem_bytes);
    if (e != cudaSuccess) return e;
    k_bp_tma<T, CPW, CU, NW, SL, ZC, true><<<grid, threads, bt.smem_bytes, s>>>(map, vol, sc, vz, zs, p, bt, count,
                                                                             err, tf);
  } else {
    e = prepare_kernel<NW>(k_bp_tma<T, CPW, CU, NW, SL, ZC, false>, bt.smem_bytes);
    if (e != cudaSuccess) return e;
    k_bp_tma<T, CPW, CU, NW, SL, ZC, false><<<grid, threads, bt.smem_bytes, s>>>(map, vol, sc, vz, zs, p, bt, count,
                                                                              err, tf);
  }
  return cudaGetLastError();
}

template <typename T, int CPW, int CU, int NW, int SL>
cudaError_t launch_batch_one(int zc, const BpScan* scans, const int4* items, int n_items, unsigned* next, int* err,
                             int smem_bytes, int grid, cudaStream_t s) {
  auto kern = zc ? k_bp_tma_batch<T, CPW, CU, NW, SL, true> : k_bp_tma_batch<T, CPW, CU, NW, SL, false>;
  cudaError_t e = prepare_kernel<NW>(kern, smem_bytes);
  if (e != cudaSuccess) return e;
  // grid = SMs; persistent CTAs: as many per SM as fit
  int per_sm = 1;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (NW + 1) * 32, smem_bytes);
  if (e != cudaSuccess) return e;
  grid = std::max(1, std::min(grid * std::max(per_sm, 1), n_items));
  kern<<<grid, (NW + 1) * 32, smem_bytes, s>>>(scans, items, n_items, next, err);
  return cudaGetLastError();
}

// The instantiated launch shapes: (columns per warp, columns per pass, consumer warps, slab slices).
// With 8 consumer warps two CTAs share an SM (registers and shared memory
// permitting), so one CTA's ring refills and tile tails overlap the other's
// updates.
#define WFBP_BP_SHAPES(X)                                                                                        \
  X(16, 4, 16, 32) X(16, 8, 16, 32) X(8, 4, 16, 32) X(8, 8, 16, 32) X(4, 4, 16, 32) X(8, 4, 20, 32) X(8, 8, 20, 32) \
  X(4, 4, 24, 32) X(16, 4, 16, 16) X(16, 8, 16, 16) X(8, 4, 20, 16) X(16, 4, 20, 16) X(16, 8, 20, 16)           \
  X(16, 4, 8, 32) X(16, 8, 8, 32) X(16, 4, 8, 16) X(16, 8, 8, 16)

template <typename T>
cudaError_t launch_elem(const CUtensorMap& map, float* vol, const float2* sc,
                        const float* vz, const float* zs, const BPParams& p, const BPTile& bt,
                        unsigned long long* count, int* err, cudaStream_t s, const ThickFuse& tf) {
  const int cpw = bt.tx * bt.ty / bt.nw;
#define WFBP_ONE(C, U, N, S) \
  if (cpw == C && bt.cu == U && bt.nw == N && bt.slab == S)                                                      \
    return bt.zc ? launch_one<T, C, U, N, S, true>(map, vol, sc, vz, zs, p, bt, count, err, s, tf)               \
                 : launch_one<T, C, U, N, S, false>(map, vol, sc, vz, zs, p, bt, count, err, s, tf);
  WFBP_BP_SHAPES(WFBP_ONE)
#undef WFBP_ONE
  return cudaErrorInvalidValue;
}

}  // namespace

// Shared-memory bytes of one launch configuration.
size_t bp_tma_smem_bytes(const BPTile& bt, int elem_bytes) {
  (void)elem_bytes;
  return bp_smem_layout(bt, bt.tx * bt.ty / bt.nw).total;
}

bool bp_tma_supported(const BPTile& bt) {
  if (bt.nw < 1) return false;
  const int cpw = bt.tx * bt.ty / bt.nw;
  if (bt.tx * bt.ty != cpw * bt.nw) return false;
#define WFBP_SUP(C, U, N, S) \
  if (cpw == C && bt.cu == U && bt.nw == N && bt.slab == S) return true;
  WFBP_BP_SHAPES(WFBP_SUP)
#undef WFBP_SUP
  return false;
}

cudaError_t bp_tma_encode_map(const void* D, int elem_half2, const BPParams& p, const BPTile& bt, CUtensorMap* map) {
  // 3-D map over [V][nch][nrp] 4-byte elements, box {nrp, W, 1}
  EncodeTiledFn fn = wfbp_encode_tiled_fn();
  if (!fn) return cudaErrorNotSupported;
  cuuint64_t dims[3] = {(cuuint64_t)bt.nrp, (cuuint64_t)p.nch, (cuuint64_t)p.V};
  cuuint64_t strides[2] = {(cuuint64_t)bt.nrp * 4, (cuuint64_t)bt.nrp * 4 * p.nch};
  cuuint32_t box[3] = {(cuuint32_t)bt.nrp, (cuuint32_t)bt.W, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, elem_half2 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                  const_cast<void*>(D), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_backproject_tma(const void* D, int elem_half2, float row_scale, float* vol,
                                   const float2* sc, const float* vz, const float* zs, const BPParams& p0,
                                   const BPTile& bt, unsigned long long* count, int* err, cudaStream_t s,
                                   const ThickFuse* tf) {
  // half2 pairs hold the rows divided by row_scale (a power of two): the
  // write-back's 2 pi / P takes it back, exactly
  BPParams p = p0;
  if (elem_half2) p.dtheta *= row_scale;
  if (!bp_tma_supported(bt)) return cudaErrorInvalidValue;
  CUtensorMap map;
  cudaError_t e = bp_tma_encode_map(D, elem_half2, p, bt, &map);
  if (e != cudaSuccess) return e;
  ThickFuse none;
  memset(&none, 0, sizeof(none));
  const ThickFuse& f = tf ? *tf : none;
  if (elem_half2) return launch_elem<uint32_t>(map, vol, sc, vz, zs, p, bt, count, err, s, f);
  return launch_elem<float>(map, vol, sc, vz, zs, p, bt, count, err, s, f);
}

cudaError_t launch_backproject_tma_batch(int elem_half2, int cpw, int cu, int nw, int slab, int zc, const BpScan* scans,
                                         const int4* items, int n_items, unsigned* next, int* err, int smem_bytes,
                                         int grid, cudaStream_t s) {
#define WFBP_B32(C, U, N, S) \
  if (cpw == C && cu == U && nw == N && slab == S) return launch_batch_one<uint32_t, C, U, N, S>(zc, scans, items, n_items, next, err, smem_bytes, grid, s);
#define WFBP_BF(C, U, N, S) \
  if (cpw == C && cu == U && nw == N && slab == S) return launch_batch_one<float, C, U, N, S>(zc, scans, items, n_items, next, err, smem_bytes, grid, s);
  if (elem_half2) {
    WFBP_BP_SHAPES(WFBP_B32)
  } else {
    WFBP_BP_SHAPES(WFBP_BF)
  }
#undef WFBP_B32
#undef WFBP_BF
  return cudaErrorInvalidValue;
}
