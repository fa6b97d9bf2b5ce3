// Ramp filter as a split-precision Toeplitz contraction on the 5th-generation
// tensor cores (tcgen05 / UMMA, sm_100a).
//
// The reference filters each zero-padded detector row with cuFFT
// (ReconstructionMachine.cu:206-290, cuda_kernels.cuh:41-58). With >= nch-1
// zeros of padding that circular convolution equals, on the data window, the
// linear convolution y[n] = sum_k h[|n-k|] x[k]: Y = X T with X the rebinned
// rows [M = V*nr][K = nch] and T the symmetric Toeplitz matrix of the taps.
//
// Precision: X = Xhi + Xlo and T = Thi + Tlo in FP16 (hi = f16(v),
// lo = f16(v - hi): 22 significant bits) after power-of-two scalings that keep
// every operand inside FP16's range (per view for X, o max|x| <= 16384; one for
// T); Y = Xhi Thi + Xhi Tlo + Xlo Thi accumulated in FP32 in tensor memory
// (the dropped Xlo Tlo term is ~2^-22 relative) and scaled back in the
// epilogue. A BF16 split (16 bits) measured 1.4 HU RMS against the FP64
// oracle on the flying-focal-spot scanner, whose fine channel sampling makes
// the ramp filter's cancellation severe; this split 0.03 HU.
//
// Tiling: 128 x BN output tiles (BN <= 256, a multiple of 16), the N tiles of
// one 128-row M tile consecutive (they share the A tile in L2). A persistent
// CTA per SM walks the tiles with three warp roles: warp 0 lane 0 issues the
// TMA loads (128B-swizzled, K-major) of the four operand tiles of each 64-wide
// K block into a 2-stage ring; warp 1 lane 0 issues the 3 x 4 UMMAs
// (M128 x N BN x K16) per K block into one of two FP32 accumulators in tensor
// memory and commits each stage back to the producer; warps 2-5 read the
// other accumulator out of tensor memory (tcgen05.ld 32x32b, one row per
// thread) and store FP32 rows, FP16 rows scaled by a per-row power of two, or
// half2 row pairs, while the next tile's MMAs run. Every mbarrier wait is
// bounded: on timeout the CTA records an error code, every role stops issuing
// work, and the CTA waits (bounded) for its copies and MMAs before freeing
// its tensor memory.
#include "wfbp_internal.h"
#include "wait.cuh"

#include <cuda.h>

#include <algorithm>

namespace {

constexpr int TC_BM = 128;
constexpr int TC_BK = 64;  // 64 FP16 = 128 bytes, one swizzle row
constexpr int TC_ACC = 2;            // accumulators in tensor memory (MMAs of tile i+1 overlap the epilogue of i)
constexpr int TC_EPI_THREADS = 128;  // warps 2-5
constexpr int TC_THREADS = 64 + TC_EPI_THREADS;
constexpr uint32_t TC_TMEM_COLS = 512;  // TC_ACC x BN (<= 256) columns, a power of two

struct TcParams {
  int M;          // rows of one operand plane of X (V * nrv)
  int mb, me;     // rows [mb, me) computed by this launch (mb a multiple of nrv)
  int nch;        // valid output channels
  int BN;         // N tile
  int kblocks;    // Kp / 64
  int np;         // padded N (rows of one B plane)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait on phase parity (wait.cuh); false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) { return wfbp_mbar_wait(bar, parity); }

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), LBO 16 bytes, descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::f16 instruction descriptor: D F32, A/B F16 (format 0), both K-major,
// M=128, N=bn.
__host__ __device__ constexpr uint32_t idesc_f16(int bn) {
  return (1u << 4) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Named barrier of the four epilogue warps (the CTA-wide barrier 0 is not
// used while the roles run).
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// One output tile's epilogue: the 32 rows of TMEM lane quarter `q` (rows
// 32q .. 32q+31 of the tile, one per lane) from accumulator columns `acc`.
__device__ __forceinline__ void tc_epilogue(const TcParams& p, const TcOutArgs& o, uint32_t tmem_acc, int q, int lane,
                                            int m0, int n0, float (*s_xchg)[16], int* err) {
  // row m of the tile: view v = m / nrv, row i = m % nrv (rows i >= nr are zero padding)
  const int m = m0 + q * 32 + lane;
  const int v = m / o.nrv, i = m % o.nrv;
  const bool row_ok = m < p.me && i < o.nr;
  // the accumulator holds (o_v x) . (t T): y = acc / (o_v t), all powers of two
  float inv = m < p.me ? 1.0f / (o.op_scale[v] * o.tap_scale) : 1.0f;
  if (o.mode == TC_OUT_F16_ROWS && row_ok) {
    inv /= o.row_scale_in[m];
    if (n0 == 0) o.row_scale_out[(size_t)v * o.nr + i] = o.row_scale_in[m];
  } else if (o.mode == TC_OUT_PAIRS && m < p.me) {
    inv /= o.pair_scale;
  }
  const uint32_t trow = tmem_acc + ((uint32_t)(q * 32) << 16);
  for (int c = 0; c < p.BN; c += 16) {
    float val[16];
    tmem_ld16(trow + (uint32_t)c, val);
    const int n = n0 + c;
    if (o.mode == TC_OUT_PAIRS) {
      // partner row i + 1 lives in the next lane, or in lane 0 of the next quarter
      if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 16; k++) s_xchg[q][k] = val[k];
      }
      epi_sync();
      float nxt[16];
#pragma unroll
      for (int k = 0; k < 16; k++) {
        const float dn = __shfl_down_sync(0xffffffffu, val[k], 1);
        nxt[k] = lane < 31 ? dn : (q < 3 ? s_xchg[q + 1][k] : 0.0f);
      }
      epi_sync();
      if (row_ok) {
        const bool last = (i == o.nr - 1);
        bool over = false;
        for (int k = 0; k < 16 && n + k < p.nch; k++) {
          const float a = val[k] * inv, b = last ? 0.0f : nxt[k] * inv;
          // |x| <= 16384 keeps the half2 differences of the backprojection's
          // channel interpolation finite
          over |= fabsf(a) > 16384.0f || fabsf(b) > 16384.0f;
          const __half2 h = __floats2half2_rn(a, b);
          o.pairs[((size_t)v * p.nch + (n + k)) * o.nrp + i] = *reinterpret_cast<const uint32_t*>(&h);
        }
        if (over) atomicOr(err, WFBP_ERRBIT_F16_RANGE);
      }
      continue;
    }
    if (!row_ok || n >= p.nch) continue;
    if (o.mode == TC_OUT_F16_ROWS) {
      __half* dst = o.y16 + ((size_t)v * o.nr + i) * p.nch + n;
      if (n + 16 <= p.nch && ((p.nch & 7) == 0)) {
        __align__(16) __half h[16];
#pragma unroll
        for (int k = 0; k < 16; k++) h[k] = __float2half_rn(val[k] * inv);
        reinterpret_cast<uint4*>(dst)[0] = reinterpret_cast<uint4*>(h)[0];
        reinterpret_cast<uint4*>(dst)[1] = reinterpret_cast<uint4*>(h)[1];
      } else {
        for (int k = 0; k < 16 && n + k < p.nch; k++) dst[k] = __float2half_rn(val[k] * inv);
      }
    } else {
      float* dst = o.y32 + (size_t)m * p.nch + n;
      for (int k = 0; k < 16 && n + k < p.nch; k++) dst[k] = val[k] * inv;
    }
  }
}

template <int TC_STAGES>
__global__ void __launch_bounds__(TC_THREADS, 1)
k_toeplitz_tc(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, TcParams p,
              TcOutArgs o, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t a_bytes = TC_BM * TC_BK * 2;          // 16 KB per plane
  const uint32_t b_bytes = (uint32_t)p.BN * TC_BK * 2; // BN x 128 B per plane
  const uint32_t stage_bytes = 2 * a_bytes + 2 * b_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + TC_STAGES * stage_bytes);
  uint64_t* empty = full + TC_STAGES;
  uint64_t* acc_full = empty + TC_STAGES;   // MMA -> epilogue: accumulator a holds a finished tile
  uint64_t* acc_empty = acc_full + TC_ACC;  // epilogue -> MMA: accumulator a has been read
  uint64_t* done = acc_empty + TC_ACC;      // every issued MMA has completed (teardown)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int s_fail;
  __shared__ float s_xchg[4][16];  // row 32q of each lane quarter, for the pairs of the quarter above
  __shared__ int s_epi_ok[4];

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int ntn = p.np / p.BN;                                   // N tiles
  const int mtiles = (p.me - p.mb + TC_BM - 1) / TC_BM;
  const int ntiles = mtiles * ntn;
  volatile int* fail = &s_fail;

  if (threadIdx.x == 0) {
    s_fail = 0;
    for (int s = 0; s < TC_STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < TC_ACC; a++) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], TC_EPI_THREADS);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  uint32_t issued = 0;  // K blocks whose loads the producer issued (over all tiles)
  if (warp == 0) {
    if (lane == 0) {
      uint32_t g = 0;
      for (int t = blockIdx.x; t < ntiles && !*fail; t += gridDim.x) {
        const int m0 = p.mb + (t / ntn) * TC_BM, n0 = (t % ntn) * p.BN;
        for (int kb = 0; kb < p.kblocks; kb++, g++) {
          const int s = (int)(g % TC_STAGES);
          const uint32_t u = g / TC_STAGES;
          if (u > 0 && !mbar_wait(&empty[s], (u - 1) & 1)) {
            atomicExch(&s_fail, 1);
            break;
          }
          if (*fail) break;
          uint8_t* st = smem + s * stage_bytes;
          mbar_expect_tx(&full[s], stage_bytes);
          const int kx = kb * TC_BK;
          tma_load_2d(st, &mapA, &full[s], kx, m0);
          tma_load_2d(st + a_bytes, &mapA, &full[s], kx, p.M + m0);
          tma_load_2d(st + 2 * a_bytes, &mapB, &full[s], kx, n0);
          tma_load_2d(st + 2 * a_bytes + b_bytes, &mapB, &full[s], kx, p.np + n0);
          issued = g + 1;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_f16(p.BN);
      uint32_t g = 0, it = 0;
      for (int t = blockIdx.x; t < ntiles && !*fail; t += gridDim.x, it++) {
        const int a = (int)(it % TC_ACC);
        const uint32_t ua = it / TC_ACC;
        if (ua > 0 && !mbar_wait(&acc_empty[a], (ua - 1) & 1)) {
          atomicExch(&s_fail, 1);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(a * p.BN);
        bool ok = true;
        for (int kb = 0; kb < p.kblocks; kb++, g++) {
          const int s = (int)(g % TC_STAGES);
          if (!mbar_wait(&full[s], (g / TC_STAGES) & 1) || *fail) {
            atomicExch(&s_fail, 1);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t st = smem_u32(smem + s * stage_bytes);
          const uint32_t ahi = st, alo = st + a_bytes, bhi = st + 2 * a_bytes, blo = bhi + b_bytes;
#pragma unroll
          for (int kk = 0; kk < TC_BK / 16; kk++) {
            const uint32_t off = kk * 32;  // 16 FP16 along K inside the swizzle row
            umma_f16(d, sw128_desc(ahi + off), sw128_desc(bhi + off), idesc, (kb | kk) ? 1u : 0u);
            umma_f16(d, sw128_desc(ahi + off), sw128_desc(blo + off), idesc, 1u);
            umma_f16(d, sw128_desc(alo + off), sw128_desc(bhi + off), idesc, 1u);
          }
          umma_commit(&empty[s]);
        }
        if (!ok) break;
        umma_commit(&acc_full[a]);  // arrives when the tile's MMAs have completed
      }
      umma_commit(done);  // arrives when every issued MMA has completed
    }
  } else {
    // epilogue warps 2-5: TMEM lane quarter q = warp % 4 (tcgen05.ld's access rule)
    const int q = warp % 4;
    uint32_t it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
      const int a = (int)(it % TC_ACC);
      int ok = 1;
      if (lane == 0) ok = mbar_wait(&acc_full[a], (it / TC_ACC) & 1) && !*fail;
      // the four epilogue warps agree before the named barriers inside the
      // epilogue, so that either all of them run it or none does
      if (lane == 0) s_epi_ok[q] = ok;
      epi_sync();
      ok = s_epi_ok[0] & s_epi_ok[1] & s_epi_ok[2] & s_epi_ok[3];
      epi_sync();  // every warp has read the flags before the next tile overwrites them
      if (!ok) {
        if (lane == 0) atomicExch(&s_fail, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      tc_epilogue(p, o, tmem + (uint32_t)(a * p.BN), q, lane, p.mb + (t / ntn) * TC_BM, (t % ntn) * p.BN, s_xchg, err);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&acc_empty[a]);
    }
  }
  __syncwarp();

  // teardown: every MMA and copy this CTA issued has landed before the tensor
  // memory and the shared memory go away
  if (warp == 1 && lane == 0) {
    if (!mbar_wait(done, 0)) atomicExch(&s_fail, 1);
  }
  __syncthreads();
  if (*fail && warp == 0 && lane == 0) {
    atomicExch(err, WFBP_ERR_TIMEOUT);
    for (uint32_t g = (issued > TC_STAGES ? issued - TC_STAGES : 0); g < issued; g++)
      mbar_wait(&full[g % TC_STAGES], (g / TC_STAGES) & 1);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
  }
}

}  // namespace

EncodeTiledFn wfbp_encode_tiled_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

namespace {

// 2-D FP16 map over `rows` rows of `kp` elements, box 64 x box_rows, 128B swizzle.
bool make_map(CUtensorMap* map, const void* base, uint64_t kp, uint64_t rows, uint32_t box_rows) {
  EncodeTiledFn fn = wfbp_encode_tiled_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {kp, rows};
  cuuint64_t strides[1] = {kp * 2};
  cuuint32_t box[2] = {TC_BK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

size_t tc_smem_bytes(int bn, int stages) { return (size_t)stages * (2 * TC_BM * TC_BK * 2 + 2 * bn * TC_BK * 2) + 1024 + 256; }

// Ring depth for an N tile: three stages when they fit in shared memory (N
// tiles of at most 144), else two.
int tc_stages(int bn) { return tc_smem_bytes(bn, 3) <= 227u * 1024u ? 3 : 2; }

// Chooses the N tile (multiple of 16, <= 256) that minimises padding of nch.
int tc_choose_bn(int nch) {
  int best = 256;
  long best_pad = -1;
  for (int bn = 256; bn >= 64; bn -= 16) {
    long np = ((long)(nch + bn - 1) / bn) * bn;
    if (best_pad < 0 || np < best_pad) { best_pad = np; best = bn; }
  }
  return best;
}

// a_planes: FP16 [2][M][kp] (hi then lo); b_planes: FP16 [2][np][kp].
cudaError_t launch_filter_tc(const void* a_planes, const void* b_planes, int M, int nch, int kp, int np, int bn,
                             const TcOutArgs& out, int* err, cudaStream_t s, int mb, int me) {
  if (me < 0) me = M;
  if (mb < 0 || mb >= me || me > M || mb % (out.nrv > 0 ? out.nrv : 1)) return cudaErrorInvalidValue;
  if (bn < 16 || bn > 256 || bn % 16 || kp % TC_BK || np % bn) return cudaErrorInvalidValue;
  CUtensorMap map_a, map_b;
  if (!make_map(&map_a, a_planes, (uint64_t)kp, 2ull * M, TC_BM)) return cudaErrorInvalidValue;
  if (!make_map(&map_b, b_planes, (uint64_t)kp, 2ull * np, (uint32_t)bn)) return cudaErrorInvalidValue;
  TcParams p;
  p.M = M;
  p.mb = mb;
  p.me = me;
  p.nch = nch;
  p.BN = bn;
  p.kblocks = kp / TC_BK;
  p.np = np;
  if (out.nrv < 1 || TC_BM % out.nrv != 0) return cudaErrorInvalidValue;  // views must not straddle M tiles
  if (2 * bn > (int)TC_TMEM_COLS) return cudaErrorInvalidValue;
  const int stages = tc_stages(bn);
  size_t smem = tc_smem_bytes(bn, stages);
  auto kern = stages == 3 ? k_toeplitz_tc<3> : k_toeplitz_tc<2>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  // persistent CTAs, one per SM (the shared memory of one ring fills an SM)
  const long tiles = (long)((me - mb + TC_BM - 1) / TC_BM) * (np / bn);
  const unsigned grid = (unsigned)std::max(1L, std::min<long>(tiles, sms));
  kern<<<grid, TC_THREADS, smem, s>>>(map_a, map_b, p, out, err);
  return cudaGetLastError();
}
