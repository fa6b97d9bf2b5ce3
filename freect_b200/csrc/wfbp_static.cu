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
// The array's name is only a host-side stand-in for the device symbol, so the
// host code below never passes it to a kernel: once per device, with that
// device current, it asks the runtime for the array's device address
// (cudaGetSymbolAddress) and hands that address to the stage launches.
#include "wfbp_internal.h"

#include <mutex>

#define WFBP_API extern "C" __attribute__((visibility("default")))

namespace {

static __device__ __align__(256) unsigned char g_static_scratch[WFBP_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Device address of g_static_scratch on `device` (looked up once per device,
// with that device current). Returns nullptr on failure.
void* scratch_address(int device, cudaError_t* err) {
  *err = cudaSuccess;
  if (device < 0 || device >= kMaxDevices) {
    *err = cudaErrorInvalidDevice;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) {
      *err = e;
      return nullptr;
    }
    g_scratch_addr[device] = p;
  }
  return g_scratch_addr[device];
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
  wfbp_dims d;
  int st = wfbp_query(ctx, &d);
  if (st) return st;
  // layout: [rebinned][filtered][row scales][native volume], 256-byte aligned
  const size_t off_filt = align256(d.rebinned_bytes);
  const size_t off_scal = off_filt + align256(d.filtered_bytes);
  const size_t off_nat = off_scal + align256(d.row_scale_bytes);
  const size_t need = off_nat + align256(d.native_volume_bytes);
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
  float* scales = d.row_scale_bytes ? reinterpret_cast<float*>(base + off_scal) : nullptr;
  float* native = reinterpret_cast<float*>(base + off_nat);
  if (!(st = wfbp_rebin(ctx, raw, rebinned, stream)) && !(st = wfbp_filter(ctx, rebinned, filtered, scales, stream)) &&
      !(st = wfbp_backproject(ctx, filtered, scales, native, nullptr, stream)))
    st = wfbp_thicken(ctx, native, volume, stream);
  if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
  return st;
}
