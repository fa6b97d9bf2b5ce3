// Helical Q-weighted backprojection, TMA-staged (sm_100a).
//
// Same algorithm as backproject_kernel (cuda_kernels.cuh:198-287) and
// k_bp (k_backproject.cu); this kernel is organised for throughput:
//
//  * Lanes are slices. A warp owns CPW (x, y) columns and the 32 consecutive
//    native slices of a slab; lane l holds slice s0 + l of every column. The
//    geometry of a (column, view) pair -- p_hat, l_hat, the asin term, the
//    channel index and weight, and the row coordinate as a linear function of
//    z -- is computed once, by one lane, and broadcast to the 32 lanes through
//    shared memory.
//  * Filtered rows are read in the backprojection layout [view][channel][row]
//    (rows contiguous), so the 32 lanes of a warp, which sit at consecutive
//    rows of the same two channels, read consecutive shared-memory words.
//  * A producer warp walks the half-turn angles theta~ and, for each, selects
//    the views j = theta~ + k P/2 whose table position can reach the CTA's
//    slab (the reference's z cull, cuda_kernels.cuh:232, and the detector's
//    cone), and TMA-loads the channel window each view needs for the CTA's
//    column tile (all rows) into a 2-stage mbarrier ring.
//  * For every column the 16 consumer warps accumulate sum(W g) and sum(W)
//    over the staged views of theta~ and add (2 pi/P) sum(W g)/sum(W) to the
//    column's slice in registers (NaN when no view contributes, like the
//    reference).
//
// Element types: float (FP32 rows) or uint32_t holding half2 pairs
// (row r, row r+1) of FP16 rows scaled by a per-view power of two.
//
// Every mbarrier wait is bounded; on timeout the CTA records WFBP_ERR_TIMEOUT
// in the error word and stops. Window or slot overflows (which the host's
// sizing rules out) are recorded as well and the affected samples skipped.
#include "wfbp_internal.h"

#include <cuda.h>

#include <type_traits>

namespace {

constexpr int BT_CWARPS = 16;                    // consumer warps
constexpr int BT_THREADS = (BT_CWARPS + 1) * 32;  // + producer warp
constexpr int BT_STAGES = 2;
constexpr long long BT_SPIN = 1ll << 26;

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

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < BT_SPIN; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// W(q) of cuda_kernels.cuh:79-93 as a function of the row coordinate
// q = (q_hat + 1) hn: |q_hat| = |q - hn| / hn.
__device__ __forceinline__ float q_weight_row(float q, float hn, float k1) {
  float t = __saturatef(fmaf(fabsf(q - hn), k1, -1.5f));
  return fmaf(0.5f, __cosf(3.14159265f * t), 0.5f);
}

struct __align__(16) Geo {
  float bq, cq, qlo, qhi;  // q(z) = bq z + cq; valid for qlo <= q <= qhi
  int base;                // element offset of (channel pf, row 0) in the stage buffer
  float wp;                // channel weight
  float sv;                // per-view scale (FP16 rows) or 1
  float pad;
};

template <typename T, int CPW, bool COUNT>
__global__ void __launch_bounds__(BT_THREADS, 1)
k_bp_tma(const __grid_constant__ CUtensorMap map, const float* __restrict__ view_scale, float* __restrict__ vol,
         const float2* __restrict__ view_sc, const float* __restrict__ view_z, const float* __restrict__ zslices,
         BPParams p, BPTile bt, unsigned long long* __restrict__ count, int* __restrict__ err) {
  constexpr int TILE = BT_CWARPS * CPW;  // columns per CTA
  extern __shared__ __align__(128) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint8_t* slots = smem;  // [STAGES][nv_max][slot_bytes]
  int2* vinfo = reinterpret_cast<int2*>(slots + (size_t)BT_STAGES * bt.nv_max * bt.slot_bytes);  // [STAGES][nv_max]
  int* nvs = reinterpret_cast<int*>(vinfo + BT_STAGES * bt.nv_max);                             // [STAGES] (+pad)
  Geo* geo = reinterpret_cast<Geo*>(nvs + 4);                                                  // [warps][nv_max][CPW]
  uint64_t* full = reinterpret_cast<uint64_t*>(geo + BT_CWARPS * bt.nv_max * CPW);
  uint64_t* empty = full + BT_STAGES;
  __shared__ int s_fail;

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int ix0 = blockIdx.x * bt.tx, iy0 = blockIdx.y * bt.ty;
  const int s0 = blockIdx.z * 32;

  // slab z range (all warps compute the same values)
  const int my_s = s0 + lane;
  const float zl = my_s < p.nz ? zslices[my_s] : __int_as_float(0x7fc00000);
  float zmn = my_s < p.nz ? zl : 3.0e38f, zmx = my_s < p.nz ? zl : -3.0e38f;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    zmn = fminf(zmn, __shfl_xor_sync(0xffffffffu, zmn, o));
    zmx = fmaxf(zmx, __shfl_xor_sync(0xffffffffu, zmx, o));
  }

  if (threadIdx.x == 0) {
    s_fail = 0;
    for (int s = 0; s < BT_STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], BT_CWARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  const float nxm = 0.5f * ((float)p.nx - 1.0f), nym = 0.5f * ((float)p.ny - 1.0f);
  auto xcoord = [&](int ix) { return ((float)ix - nxm) * p.fov / (float)p.nx + p.x0; };
  auto ycoord = [&](int iy) { return ((float)iy - nym) * p.fov / (float)p.ny + p.y0; };
  const size_t slot_elems = (size_t)bt.slot_bytes / sizeof(T);

  if (warp == BT_CWARPS) {
    // ---------------- producer ----------------
    if (lane == 0) {
      const float zlo = zmn - bt.reach, zhi = zmx + bt.reach;
      const float xa = xcoord(ix0), xb = xcoord(min(ix0 + bt.tx - 1, p.nx - 1));
      const float ya = ycoord(iy0), yb = ycoord(min(iy0 + bt.ty - 1, p.ny - 1));
      const uint32_t view_bytes = (uint32_t)(bt.W * bt.nrp * sizeof(T));
      int issued_upto = 0;
      for (int t = 0; t < p.P2; t++) {
        const int s = t & 1, u = t >> 1;
        if (u >= 1 && !mbar_wait(&empty[s], (u - 1) & 1)) {
          atomicExch(&s_fail, 1);
          break;
        }
        if (*((volatile int*)&s_fail)) break;
        int nv = 0;
        for (int k = 0; k < p.K; k++) {
          const int j = t + k * p.P2;
          const float zt = __ldg(view_z + j);
          if (zt < zlo || zt > zhi) continue;
          if (nv == bt.nv_max) {
            atomicOr(err, 0x100);  // more views than slots: host sizing violated
            break;
          }
          const float2 sc = __ldg(view_sc + j);
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
          if (whi < zmn || wlo > zmx) continue;
          const float idx_min = p.kp - (pmax * p.ps + p.c0);  // p_idx decreases with p_hat
          int c_lo = (int)floorf(idx_min) - 1;
          c_lo = max(0, min(c_lo, p.nch - bt.W));
          vinfo[s * bt.nv_max + nv] = make_int2(j, c_lo);
          nv++;
        }
        nvs[s] = nv;
        mbar_arrive_tx(&full[s], (uint32_t)nv * view_bytes);
        for (int v = 0; v < nv; v++) {
          const int2 vi = vinfo[s * bt.nv_max + v];
          tma_load_3d(slots + ((size_t)s * bt.nv_max + v) * bt.slot_bytes, &map, &full[s], 0, vi.y, vi.x);
        }
        issued_upto = t + 1;
      }
      if (*((volatile int*)&s_fail)) {
        atomicExch(err, WFBP_ERR_TIMEOUT);
        // let copies already issued land before the CTA's shared memory goes away
        for (int t = max(0, issued_upto - BT_STAGES); t < issued_upto; t++) mbar_wait(&full[t & 1], (t >> 1) & 1);
      }
    }
    return;
  }

  // ---------------- consumers ----------------
  float vacc[CPW];
#pragma unroll
  for (int c = 0; c < CPW; c++) vacc[c] = 0.0f;
  unsigned long long cnt = 0;
  const float k1 = 2.5f / p.hn;
  Geo* wgeo = geo + (size_t)warp * bt.nv_max * CPW;
  constexpr int VPP = 32 / CPW;  // views per geometry pass
  const int gc = lane % CPW, gv = lane / CPW;
  const int gt = warp * CPW + gc;  // tile column handled by this lane in geometry passes
  const int gix = ix0 + gt % bt.tx, giy = iy0 + gt / bt.tx;
  const float gx = xcoord(gix), gy = ycoord(giy);
  const bool gactive = gix < p.nx && giy < p.ny && !(gx * gx + gy * gy > p.fov_half2);
  unsigned active_mask = 0;  // bit c: column c of this warp is inside the grid and the FOV
#pragma unroll
  for (int c = 0; c < CPW; c++) active_mask |= (__shfl_sync(0xffffffffu, gactive ? 1u : 0u, c) & 1u) << c;

  for (int t = 0; t < p.P2; t++) {
    const int s = t & 1, u = t >> 1;
    if (!mbar_wait(&full[s], u & 1)) {
      atomicExch(&s_fail, 1);
      atomicExch(err, WFBP_ERR_TIMEOUT);
      break;
    }
    const int nv = nvs[s];
    const T* stage = reinterpret_cast<const T*>(slots + (size_t)s * bt.nv_max * bt.slot_bytes);
    // geometry of (column gc, view v) for v = gv, gv + VPP, ...
    for (int v = gv; v < nv; v += VPP) {
      const int2 vi = vinfo[s * bt.nv_max + v];
      const float2 sc = __ldg(view_sc + vi.x);
      const float zt = __ldg(view_z + vi.x);
      const float p_hat = gx * sc.x - gy * sc.y;
      const float l_hat = sqrtf(p.R2 - p_hat * p_hat) - gx * sc.y - gy * sc.x;
      const float A = p.zr2pi * asinf(p.rR * p_hat);
      const float inv = 1.0f / (l_hat * p.tanc);
      const float p_idx = p.kp - (p_hat * p.ps + p.c0);
      const float pf = floorf(p_idx);
      bool valid = gactive && pf >= 0.0f && ceilf(p_idx) <= p.ncm2;
      const int cofs = (int)pf - vi.y;
      if (valid && (cofs < 0 || cofs > bt.W - 2)) {
        atomicOr(err, 0x200);  // channel window too narrow: host sizing violated
        valid = false;
      }
      Geo g;
      g.bq = inv * p.hn;
      g.cq = p.hn * fmaf(A - zt, inv, 1.0f);
      g.qlo = valid ? fmaxf(0.0f, fmaf(zt - p.z_rot, g.bq, g.cq)) : 3.0e38f;
      g.qhi = valid ? fminf(p.nrm2, fmaf(zt + p.z_rot, g.bq, g.cq)) : -3.0e38f;
      g.base = (int)((size_t)v * slot_elems) + (valid ? cofs : 0) * bt.nrp;
      g.wp = p_idx - pf;
      g.sv = std::is_same<T, float>::value ? 1.0f : __ldg(view_scale + vi.x);
      g.pad = 0.0f;
      wgeo[v * CPW + gc] = g;
    }
    __syncwarp();
    // CU columns per step: CU independent accumulation chains per view
    constexpr int CU = CPW >= 4 ? 4 : CPW;
    const unsigned nrm2u = (unsigned)(p.nr - 2);
#pragma unroll
    for (int c0 = 0; c0 < CPW; c0 += CU) {
      if (!((active_mask >> c0) & ((1u << CU) - 1u))) continue;
      float ag[CU], aw[CU];
#pragma unroll
      for (int u = 0; u < CU; u++) { ag[u] = 0.0f; aw[u] = 0.0f; }
      for (int v = 0; v < nv; v++) {
#pragma unroll
        for (int u = 0; u < CU; u++) {
          const Geo g = wgeo[v * CPW + c0 + u];
          const float q = fmaf(zl, g.bq, g.cq);
          const bool ok = (q >= g.qlo) && (q <= g.qhi);
          // any in-range row for invalid lanes (their weight is 0); NaN -> 0
          const unsigned r = min((unsigned)__float2int_rz(q), nrm2u);
          const float wq = q - (float)r;
          const T* e = stage + g.base + r;
          float top, bot;
          if constexpr (std::is_same<T, float>::value) {
            const float d00 = e[0], d01 = e[1], d10 = e[bt.nrp], d11 = e[bt.nrp + 1];
            top = fmaf(g.wp, d10 - d00, d00);
            bot = fmaf(g.wp, d11 - d01, d01);
          } else {
            const uint32_t u0 = e[0], u1 = e[bt.nrp];
            const float2 f0 = __half22float2(*reinterpret_cast<const __half2*>(&u0));
            const float2 f1 = __half22float2(*reinterpret_cast<const __half2*>(&u1));
            top = fmaf(g.wp, f1.x - f0.x, f0.x);
            bot = fmaf(g.wp, f1.y - f0.y, f0.y);
          }
          const float gval = fmaf(wq, bot - top, top);
          const float W = ok ? q_weight_row(q, p.hn, k1) : 0.0f;
          if constexpr (std::is_same<T, float>::value)
            ag[u] = fmaf(W, gval, ag[u]);
          else
            ag[u] = fmaf(W * g.sv, gval, ag[u]);
          aw[u] += W;
          if (COUNT) cnt += ok ? 1 : 0;
        }
      }
#pragma unroll
      for (int u = 0; u < CU; u++)
        if ((active_mask >> (c0 + u)) & 1u) vacc[c0 + u] += p.dtheta * (1.0f / aw[u]) * ag[u];  // cuda_kernels.cuh:283
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }

  // write the slab
  if (my_s < p.nz) {
    const size_t plane = (size_t)p.nx * p.ny;
#pragma unroll
    for (int c = 0; c < CPW; c++) {
      const int tt = warp * CPW + c;
      const int ix = ix0 + tt % bt.tx, iy = iy0 + tt / bt.tx;
      if (ix < p.nx && iy < p.ny) vol[(size_t)my_s * plane + (size_t)iy * p.nx + ix] = vacc[c];
    }
  }
  if (COUNT) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(count, cnt);
  }
}

template <typename T, int CPW>
cudaError_t launch_one(const CUtensorMap& map, const float* view_scale, float* vol, const float2* sc,
                       const float* vz, const float* zs, const BPParams& p, const BPTile& bt,
                       unsigned long long* count, int* err, cudaStream_t s) {
  dim3 grid((unsigned)((p.nx + bt.tx - 1) / bt.tx), (unsigned)((p.ny + bt.ty - 1) / bt.ty), (unsigned)((p.nz + 31) / 32));
  cudaError_t e;
  if (count) {
    e = cudaFuncSetAttribute(k_bp_tma<T, CPW, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bt.smem_bytes);
    if (e != cudaSuccess) return e;
    k_bp_tma<T, CPW, true><<<grid, BT_THREADS, bt.smem_bytes, s>>>(map, view_scale, vol, sc, vz, zs, p, bt, count, err);
  } else {
    e = cudaFuncSetAttribute(k_bp_tma<T, CPW, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bt.smem_bytes);
    if (e != cudaSuccess) return e;
    k_bp_tma<T, CPW, false><<<grid, BT_THREADS, bt.smem_bytes, s>>>(map, view_scale, vol, sc, vz, zs, p, bt, count, err);
  }
  return cudaGetLastError();
}

}  // namespace

// Shared-memory bytes of one launch configuration.
size_t bp_tma_smem_bytes(const BPTile& bt, int elem_bytes) {
  (void)elem_bytes;
  const int cpw = bt.tx * bt.ty / BT_CWARPS;
  return 128 + (size_t)BT_STAGES * bt.nv_max * bt.slot_bytes + (size_t)BT_STAGES * bt.nv_max * sizeof(int2) +
         4 * sizeof(int) + (size_t)BT_CWARPS * bt.nv_max * cpw * sizeof(Geo) + 2 * BT_STAGES * sizeof(uint64_t);
}

cudaError_t launch_backproject_tma(const void* D, int elem_half2, const float* view_scale, float* vol,
                                   const float2* sc, const float* vz, const float* zs, const BPParams& p,
                                   const BPTile& bt, unsigned long long* count, int* err, cudaStream_t s) {
  // 3-D map over [V][nch][nrp] 4-byte elements, box {nrp, W, 1}
  EncodeTiledFn fn = wfbp_encode_tiled_fn();
  if (!fn) return cudaErrorNotSupported;
  CUtensorMap map;
  cuuint64_t dims[3] = {(cuuint64_t)bt.nrp, (cuuint64_t)p.nch, (cuuint64_t)p.V};
  cuuint64_t strides[2] = {(cuuint64_t)bt.nrp * 4, (cuuint64_t)bt.nrp * 4 * p.nch};
  cuuint32_t box[3] = {(cuuint32_t)bt.nrp, (cuuint32_t)bt.W, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(&map, elem_half2 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                  const_cast<void*>(D), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  const int cpw = bt.tx * bt.ty / BT_CWARPS;
  if (elem_half2) {
    if (cpw == 16) return launch_one<uint32_t, 16>(map, view_scale, vol, sc, vz, zs, p, bt, count, err, s);
    if (cpw == 8) return launch_one<uint32_t, 8>(map, view_scale, vol, sc, vz, zs, p, bt, count, err, s);
    if (cpw == 4) return launch_one<uint32_t, 4>(map, view_scale, vol, sc, vz, zs, p, bt, count, err, s);
  } else {
    if (cpw == 16) return launch_one<float, 16>(map, view_scale, vol, sc, vz, zs, p, bt, count, err, s);
    if (cpw == 8) return launch_one<float, 8>(map, view_scale, vol, sc, vz, zs, p, bt, count, err, s);
    if (cpw == 4) return launch_one<float, 4>(map, view_scale, vol, sc, vz, zs, p, bt, count, err, s);
  }
  return cudaErrorInvalidValue;
}
