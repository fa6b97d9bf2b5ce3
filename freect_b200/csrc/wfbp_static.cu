// wfbp_run_static: the whole reconstruction with no device allocation.
//
// wfbp_run keeps its intermediates (rebinned rows, filtered rows, row scales,
// native-thickness volume) in context-owned scratch that it allocates with
// cudaMalloc on first use. Some callers cannot allow that: an application that
// gives all device memory to its own pool or caching allocator, a scanner
// pipeline that must run inside a fixed memory budget decided at start-up, or
// a latency-critical loop where cudaMalloc's implicit device synchronisation
// is not acceptable. This entry point serves them: its intermediates live in
// one file-scope device array of fixed size (WFBP_STATIC_SCRATCH_BYTES), which
// every GPU that loads this library holds until the process exits.
//
// It runs the stages of wfbp_run in wfbp_run's own layout (the backprojection
// layout and the TMA-staged backprojection whenever a launch fits), with the
// thickening as a separate pass instead of fused into the backprojection's
// write-back (the fused form would need the context's slab lists, which are
// allocated on first use); the two forms give the same volume bit for bit.
//
// The array's name is only a host-side stand-in for the device symbol, so the
// host code below never passes it to a kernel: with the device current, it
// asks the runtime for the array's device address (cudaGetSymbolAddress) and
// hands that address to the stage launches. The address is looked up once
// per device and CUDA context: after the application resets the device
// (cudaDeviceReset) the next call finds a new context and looks it up again.
#include "wfbp_internal.h"

#include <mutex>

#define WFBP_API extern "C" __attribute__((visibility("default")))

namespace {

static __device__ __align__(256) unsigned char g_static_scratch[WFBP_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct ScratchAddr {
  unsigned long long ctx_id = 0;  // CUDA context the address belongs to (0: none yet)
  void* addr = nullptr;
};
ScratchAddr g_scratch[kMaxDevices];

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points (the
// library does not link the driver library directly)
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
template <class F>
F driver_fn(const char* name) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
    return reinterpret_cast<F>(p);
  return nullptr;
}

// Device address of g_static_scratch on `device`, which is current. Looked up
// once per device and context; returns nullptr on failure.
void* scratch_address(int device, cudaError_t* err) {
  *err = cudaSuccess;
  if (device < 0 || device >= kMaxDevices) {
    *err = cudaErrorInvalidDevice;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  static const CtxGetCurrentFn get_current = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
  static const CtxGetIdFn get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
  if (!get_current || !get_id) {
    *err = cudaErrorNotSupported;
    return nullptr;
  }
  ScratchAddr& s = g_scratch[device];
  // the context current on this thread (cudaSetDevice binds the device's
  // primary context); none yet: the symbol lookup binds it
  CUcontext cu = nullptr;
  unsigned long long id = 0;
  void* p = nullptr;
  if (get_current(&cu) != CUDA_SUCCESS || !cu) {
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) {
      *err = e;
      return nullptr;
    }
    cu = nullptr;
    if (get_current(&cu) != CUDA_SUCCESS || !cu) {
      *err = cudaErrorDeviceUninitialized;
      return nullptr;
    }
  }
  if (get_id(cu, &id) != CUDA_SUCCESS) {
    *err = cudaErrorDeviceUninitialized;
    return nullptr;
  }
  if (s.ctx_id != id || !s.addr) {
    if (!p) {
      const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
      if (e != cudaSuccess) {
        *err = e;
        return nullptr;
      }
    }
    s.addr = p;
    s.ctx_id = id;
  }
  return s.addr;
}

}  // namespace

WFBP_API int wfbp_run_static(wfbp_ctx* ctx, const float* raw, float* volume, void* stream) {
  if (!ctx) return WFBP_ERR_INVALID_ARG;
  if (!raw || !volume) {
    ctx->err = "wfbp_run_static: null buffer";
    return WFBP_ERR_INVALID_ARG;
  }
  if (!ctx->views_set) {
    ctx->err = "wfbp_run_static: wfbp_set_views not called";
    return WFBP_ERR_STATE;
  }
  const int layout = wfbp_detail::run_layout_of(ctx);
  size_t reb = 0, filt = 0, scal = 0;
  wfbp_detail::buffer_bytes(ctx, layout, &reb, &filt, &scal);
  const size_t nat = sizeof(float) * (size_t)ctx->nz * ctx->ny * ctx->nx;
  // layout: [rebinned][filtered][row scales][native volume], 256-byte aligned
  const size_t off_filt = align256(reb);
  const size_t off_scal = off_filt + align256(filt);
  const size_t off_nat = off_scal + align256(scal);
  const size_t need = off_nat + align256(nat);
  if (need > (size_t)WFBP_STATIC_SCRATCH_BYTES) {
    ctx->err = "wfbp_run_static: this geometry needs " + std::to_string(need) +
               " bytes of intermediates, more than the static scratch of " +
               std::to_string((size_t)WFBP_STATIC_SCRATCH_BYTES) + " bytes; use wfbp_run";
    return WFBP_ERR_INVALID_ARG;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != ctx->device) cudaSetDevice(ctx->device);
  cudaError_t e;
  unsigned char* base = static_cast<unsigned char*>(scratch_address(ctx->device, &e));
  if (!base) {
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    ctx->err = std::string("wfbp_run_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
    return WFBP_ERR_CUDA;
  }
  // Every stage overwrites its whole output region, so nothing has to be
  // cleared between calls.
  void* rebinned = base;
  void* filtered = base + off_filt;
  float* scales = scal ? reinterpret_cast<float*>(base + off_scal) : nullptr;
  float* native = reinterpret_cast<float*>(base + off_nat);
  int st = wfbp_rebin(ctx, raw, rebinned, stream);
  if (!st) st = wfbp_detail::filter_stage(ctx, rebinned, filtered, scales, layout, stream);
  if (!st) st = wfbp_detail::backproject_stage(ctx, filtered, scales, native, layout, stream);
  if (!st) st = wfbp_thicken(ctx, native, volume, stream);
  if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
  return st;
}
