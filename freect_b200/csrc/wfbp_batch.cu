// Batched reconstruction of several scans (no counterpart in the reference,
// whose ReconstructionMachine reconstructs one scan per process run,
// main.cpp:60-66).
//
// Per scan the rebin and filter stages run as their own launches (their
// shapes differ from scan to scan); the backprojection of all scans is ONE
// persistent launch (k_bp_tma_batch) whose CTAs take work items -- a column
// tile and slab (32 or 16 native slices) of one scan -- from a list sorted by estimated
// cost, so uneven scans share the GPU without a tail per scan; thickening is
// again per scan. The whole chain is captured once into a CUDA graph and
// replayed while the caller's input and output pointers stay the same.
#include "wfbp_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#define WFBP_API extern "C" __attribute__((visibility("default")))

struct wfbp_batch {
  int device = 0;
  int precision = WFBP_PRECISION_FP32;
  std::vector<wfbp_ctx*> ctx;
  std::vector<void*> reb, filt;
  std::vector<float*> scales, native;
  wfbp_bp_config cfg{};
  std::vector<BPTile> tiles;
  BpScan* d_scans = nullptr;
  int4* d_items = nullptr;
  int n_items = 0;
  unsigned* d_next = nullptr;
  int* d_err = nullptr;
  int zc = 1;                       // record layout of the persistent launch (BPTile::zc of every scan)
  int smem = 0, grid = 0;
  cudaStream_t own = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<const void*> key;
  std::string err;
  std::vector<int4> h_items;          // the cost-sorted work list (host copy)
  // wfbp_batch_run_host: device copies of the readings and volumes, the copy
  // stream and its events, and the work list split into two launches
  std::vector<float*> raw_d, vol_d;
  cudaStream_t s_copy = nullptr;
  std::vector<cudaEvent_t> ev;
  int4* d_items_split = nullptr;
  int split_k = -1, split_na = 0;
};

namespace {

int bfail(wfbp_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  return code;
}

#define BCUDA(b, call)                                                                                \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess)                                                                            \
      return bfail((b), e_ == cudaErrorMemoryAllocation ? WFBP_ERR_OOM : WFBP_ERR_CUDA,               \
                   std::string(#call) + ": " + cudaGetErrorName(e_) + " " + cudaGetErrorString(e_)); \
  } while (0)

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DevGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

void drop_graph(wfbp_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->key.clear();
}

void free_plan(wfbp_batch* b) {
  cudaFree(b->d_scans);
  cudaFree(b->d_items);
  cudaFree(b->d_items_split);
  b->d_scans = nullptr;
  b->d_items = nullptr;
  b->d_items_split = nullptr;
  b->n_items = 0;
  b->split_k = -1;
}

// Views per theta~ reaching each slab (of `slab` native slices) of a scan, summed over
// theta~: the backprojection work of one column of that slab.
std::vector<double> slab_view_counts(const wfbp_ctx* c, const std::vector<float>& view_z, int slab) {
  const int nslab = (c->nz + slab - 1) / slab;
  std::vector<double> out(nslab, 0.0);
  for (int sl = 0; sl < nslab; sl++) {
    float zmn = 3e38f, zmx = -3e38f;
    for (int i = sl * slab; i < std::min(c->nz, sl * slab + slab); i++) {
      zmn = std::min(zmn, c->z_native[i]);
      zmx = std::max(zmx, c->z_native[i]);
    }
    long n = 0;
    for (int j = 0; j < c->K * c->P2; j++)
      if (!(view_z[j] < zmn - c->bp_reach || view_z[j] > zmx + c->bp_reach)) n++;
    out[sl] = (double)n;
  }
  return out;
}

// Lays out the persistent launch for configuration b->cfg: per-scan launch
// sizes, tensor maps and the cost-sorted work list.
int build_plan(wfbp_batch* b) {
  const int n = (int)b->ctx.size();
  std::vector<BpScan> hs(n);
  b->tiles.assign(n, BPTile{});
  int smem = 0;
  struct Item {
    int4 w;
    double cost;
  };
  std::vector<Item> items;
  // one launch, one record layout: with the table-position cull's row range
  // if any scan's cull can bind
  b->zc = 0;
  for (int i = 0; i < n; i++) b->zc |= b->ctx[i]->bp_zcull;
  for (int i = 0; i < n; i++) {
    wfbp_ctx* c = b->ctx[i];
    BPTile bt;
    if (!wfbp_detail::size_backprojection(c, b->cfg.tile_x, b->cfg.tile_y, b->cfg.cols_per_step,
                                          b->cfg.consumer_warps, b->cfg.slab, &bt))
      return bfail(b, WFBP_ERR_UNSUPPORTED, "backprojection configuration " + std::to_string(b->cfg.tile_x) + "x" +
                                                std::to_string(b->cfg.tile_y) + "/" +
                                                std::to_string(b->cfg.cols_per_step) + " does not fit scan " +
                                                std::to_string(i));
    if (bt.zc != b->zc) {
      bt.zc = b->zc;
      bt.smem_bytes = (int)bp_tma_smem_bytes(bt, 4);
      if (bt.smem_bytes > 220 * 1024)
        return bfail(b, WFBP_ERR_UNSUPPORTED, "backprojection configuration does not fit scan " + std::to_string(i));
    }
    b->tiles[i] = bt;
    smem = std::max(smem, bt.smem_bytes);
    memset(&hs[i], 0, sizeof(BpScan));
    hs[i].p = wfbp_detail::backprojection_params(c);
    hs[i].bt = bt;
    if (bp_tma_encode_map(b->filt[i], b->precision == WFBP_PRECISION_MIXED ? 1 : 0, hs[i].p, bt, &hs[i].map) !=
        cudaSuccess)
      return bfail(b, WFBP_ERR_CUDA, "tensor map encoding failed for scan " + std::to_string(i));
    // FP16 row pairs hold the rows divided by the scan's pair_scale (a power
    // of two): the write-back's 2 pi / P takes it back, exactly
    if (b->precision == WFBP_PRECISION_MIXED) hs[i].p.dtheta *= c->pair_scale;
    hs[i].vol = b->native[i];
    hs[i].view_sc = c->d_view_sc;
    hs[i].view_z = c->d_view_z;
    hs[i].zslices = c->d_z_native;
    // view table positions for the cost estimate
    std::vector<float> vz(c->V);
    BCUDA(b, cudaMemcpy(vz.data(), c->d_view_z, sizeof(float) * c->V, cudaMemcpyDeviceToHost));
    const std::vector<double> nv = slab_view_counts(c, vz, bt.slab);
    const int tx = (c->nx + bt.tx - 1) / bt.tx, ty = (c->ny + bt.ty - 1) / bt.ty;
    const double vx = c->rp.recon_fov / c->nx, vy = c->rp.recon_fov / c->ny;
    const double r2 = 0.25 * c->cg.acquisition_field_of_view * c->cg.acquisition_field_of_view;
    for (int by = 0; by < ty; by++)
      for (int bx = 0; bx < tx; bx++) {
        int cols = 0;
        for (int yy = by * bt.ty; yy < std::min(c->ny, (by + 1) * bt.ty); yy++)
          for (int xx = bx * bt.tx; xx < std::min(c->nx, (bx + 1) * bt.tx); xx++) {
            const double x = (xx - 0.5 * (c->nx - 1)) * vx + c->rp.x_origin;
            const double y = (yy - 0.5 * (c->ny - 1)) * vy + c->rp.y_origin;
            if (x * x + y * y <= r2) cols++;
          }
        for (int sl = 0; sl < (int)nv.size(); sl++)
          items.push_back({make_int4(i, bx, by, sl), (double)cols * nv[sl] + 1.0});
      }
  }
  std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& c) { return a.cost > c.cost; });
  std::vector<int4> hw(items.size());
  for (size_t k = 0; k < items.size(); k++) hw[k] = items[k].w;
  free_plan(b);
  BCUDA(b, cudaMalloc(&b->d_scans, sizeof(BpScan) * n));
  BCUDA(b, cudaMemcpy(b->d_scans, hs.data(), sizeof(BpScan) * n, cudaMemcpyHostToDevice));
  BCUDA(b, cudaMalloc(&b->d_items, sizeof(int4) * std::max<size_t>(hw.size(), 1)));
  BCUDA(b, cudaMemcpy(b->d_items, hw.data(), sizeof(int4) * hw.size(), cudaMemcpyHostToDevice));
  b->n_items = (int)hw.size();
  b->h_items = hw;
  b->smem = smem;
  int sms = 0;
  BCUDA(b, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  b->grid = std::max(1, std::min(sms, b->n_items));
  return WFBP_OK;
}

}  // namespace

WFBP_API int wfbp_batch_destroy(wfbp_batch* b) {
  if (!b) return WFBP_ERR_INVALID_ARG;
  {
    DevGuard g(b->device);
    drop_graph(b);
    free_plan(b);
    for (void* p : b->reb) cudaFree(p);
    for (void* p : b->filt) cudaFree(p);
    for (float* p : b->scales) cudaFree(p);
    for (float* p : b->native) cudaFree(p);
    cudaFree(b->d_next);
    cudaFree(b->d_err);
    for (float* p : b->raw_d) cudaFree(p);
    for (float* p : b->vol_d) cudaFree(p);
    for (auto e : b->ev) cudaEventDestroy(e);
    if (b->s_copy) cudaStreamDestroy(b->s_copy);
    if (b->own) cudaStreamDestroy(b->own);
  }
  delete b;
  return WFBP_OK;
}

WFBP_API int wfbp_batch_create(wfbp_ctx* const* ctxs, int n, wfbp_batch** out) {
  if (!ctxs || n < 1 || !out) return WFBP_ERR_INVALID_ARG;
  *out = nullptr;
  for (int i = 0; i < n; i++) {
    if (!ctxs[i]) return WFBP_ERR_INVALID_ARG;
    if (!ctxs[i]->views_set) return WFBP_ERR_STATE;
    if (ctxs[i]->device != ctxs[0]->device || ctxs[i]->ext.precision != ctxs[0]->ext.precision)
      return WFBP_ERR_INVALID_ARG;
    if (!ctxs[i]->bp_tma_ok) return WFBP_ERR_UNSUPPORTED;
  }
  wfbp_batch* b = new wfbp_batch;
  b->device = ctxs[0]->device;
  b->precision = ctxs[0]->ext.precision;
  b->ctx.assign(ctxs, ctxs + n);
  DevGuard g(b->device);
  auto bad = [&](int code) {
    wfbp_batch_destroy(b);
    return code;
  };
  for (int i = 0; i < n; i++) {
    size_t reb = 0, filt = 0, scal = 0;
    wfbp_detail::buffer_bytes(b->ctx[i], WFBP_LAYOUT_BACKPROJECTION, &reb, &filt, &scal);
    void *r = nullptr, *f = nullptr, *s = nullptr, *v = nullptr;
    const size_t nat = sizeof(float) * (size_t)b->ctx[i]->nz * b->ctx[i]->nx * b->ctx[i]->ny;
    cudaError_t e = cudaMalloc(&r, reb);
    if (!e) e = cudaMalloc(&f, filt);
    if (!e && scal) e = cudaMalloc(&s, scal);
    if (!e) e = cudaMalloc(&v, nat);
    b->reb.push_back(r);
    b->filt.push_back(f);
    b->scales.push_back(static_cast<float*>(s));
    b->native.push_back(static_cast<float*>(v));
    if (e) return bad(e == cudaErrorMemoryAllocation ? WFBP_ERR_OOM : WFBP_ERR_CUDA);
  }
  if (cudaMalloc(&b->d_next, sizeof(unsigned)) || cudaMalloc(&b->d_err, sizeof(int)) ||
      cudaMemset(b->d_err, 0, sizeof(int)) || cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking))
    return bad(WFBP_ERR_CUDA);
  // default configuration: the first candidate every scan fits
  int st = WFBP_ERR_UNSUPPORTED;
  for (int k = 0; k < wfbp_detail::n_bp_candidates() && st; k++) {
    wfbp_detail::bp_candidate(k, &b->cfg.tile_x, &b->cfg.tile_y, &b->cfg.cols_per_step, &b->cfg.consumer_warps,
                              &b->cfg.slab);
    bool fits = true;
    for (int i = 0; i < n && fits; i++) {
      BPTile bt;
      fits = wfbp_detail::size_backprojection(b->ctx[i], b->cfg.tile_x, b->cfg.tile_y, b->cfg.cols_per_step,
                                              b->cfg.consumer_warps, b->cfg.slab, &bt);
    }
    if (fits) st = build_plan(b);
  }
  if (st) return bad(st);
  *out = b;
  return WFBP_OK;
}

WFBP_API const char* wfbp_batch_last_error(const wfbp_batch* b) { return b ? b->err.c_str() : "null batch"; }

WFBP_API int wfbp_batch_size(const wfbp_batch* b, int* n_scans, int* n_items) {
  if (!b) return WFBP_ERR_INVALID_ARG;
  if (n_scans) *n_scans = (int)b->ctx.size();
  if (n_items) *n_items = b->n_items;
  return WFBP_OK;
}

WFBP_API int wfbp_batch_bp_configs(const wfbp_batch* b, wfbp_bp_config* out, int cap, int* n) {
  if (!b || !n || cap < 0 || (cap > 0 && !out)) return WFBP_ERR_INVALID_ARG;
  int k = 0;
  for (int c = 0; c < wfbp_detail::n_bp_candidates(); c++) {
    wfbp_bp_config cfg{};
    wfbp_detail::bp_candidate(c, &cfg.tile_x, &cfg.tile_y, &cfg.cols_per_step, &cfg.consumer_warps, &cfg.slab);
    bool fits = true;
    for (size_t i = 0; i < b->ctx.size() && fits; i++) {
      BPTile bt;
      fits = wfbp_detail::size_backprojection(b->ctx[i], cfg.tile_x, cfg.tile_y, cfg.cols_per_step, cfg.consumer_warps,
                                              cfg.slab, &bt);
    }
    if (!fits) continue;
    if (k < cap) out[k] = cfg;
    k++;
  }
  *n = k;
  return WFBP_OK;
}

WFBP_API int wfbp_batch_get_bp_config(const wfbp_batch* b, wfbp_bp_config* cfg) {
  if (!b || !cfg) return WFBP_ERR_INVALID_ARG;
  *cfg = b->cfg;
  return WFBP_OK;
}

WFBP_API int wfbp_batch_set_bp_config(wfbp_batch* b, const wfbp_bp_config* cfg) {
  if (!b || !cfg) return WFBP_ERR_INVALID_ARG;
  DevGuard g(b->device);
  const wfbp_bp_config old = b->cfg;
  b->cfg = *cfg;
  if (b->cfg.consumer_warps == 0) b->cfg.consumer_warps = BT_CWARPS;
  if (b->cfg.slab == 0) b->cfg.slab = 32;
  int st = build_plan(b);
  if (st) {
    const std::string msg = b->err;
    b->cfg = old;
    build_plan(b);
    b->err = msg;
    return st;
  }
  drop_graph(b);
  return WFBP_OK;
}

WFBP_API int wfbp_batch_run(wfbp_batch* b, const float* const* raws, float* const* volumes, void* stream) {
  if (!b) return WFBP_ERR_INVALID_ARG;
  const int n = (int)b->ctx.size();
  if (!raws || !volumes) return bfail(b, WFBP_ERR_INVALID_ARG, "wfbp_batch_run: null pointer array");
  for (int i = 0; i < n; i++)
    if (!raws[i] || !volumes[i]) return bfail(b, WFBP_ERR_INVALID_ARG, "wfbp_batch_run: null buffer for scan " +
                                                                           std::to_string(i));
  DevGuard g(b->device);
  // a graph cannot be captured on the legacy default stream: run on the
  // batch's own stream then, ordered after the caller's earlier work
  const bool legacy = stream == nullptr;
  cudaStream_t s = legacy ? b->own : (cudaStream_t)stream;
  if (legacy) BCUDA(b, cudaStreamSynchronize(0));
  std::vector<const void*> key(2 * n);
  for (int i = 0; i < n; i++) {
    key[i] = raws[i];
    key[n + i] = volumes[i];
  }
  if (!b->exec || key != b->key) {
    drop_graph(b);
    BCUDA(b, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int st = WFBP_OK;
    for (int i = 0; i < n && !st; i++) {
      st = wfbp_rebin(b->ctx[i], raws[i], b->reb[i], s);
      if (!st) st = wfbp_detail::filter_stage(b->ctx[i], b->reb[i], b->filt[i], b->scales[i],
                                              WFBP_LAYOUT_BACKPROJECTION, s);
      if (st) b->err = "scan " + std::to_string(i) + ": " + wfbp_last_error(b->ctx[i]);
    }
    cudaError_t e = cudaSuccess;
    if (!st) e = cudaMemsetAsync(b->d_next, 0, sizeof(unsigned), s);
    if (!st && !e) {
      const int cpw = b->cfg.tile_x * b->cfg.tile_y / b->cfg.consumer_warps;
      e = launch_backproject_tma_batch(b->precision == WFBP_PRECISION_MIXED ? 1 : 0, cpw, b->cfg.cols_per_step,
                                       b->cfg.consumer_warps, b->cfg.slab, b->zc,
                                       b->d_scans, b->d_items, b->n_items, b->d_next, b->d_err, b->smem, b->grid, s);
    }
    for (int i = 0; i < n && !st && !e; i++) {
      st = wfbp_thicken(b->ctx[i], b->native[i], volumes[i], s);
      if (st) b->err = "scan " + std::to_string(i) + ": " + wfbp_last_error(b->ctx[i]);
    }
    cudaGraph_t graph = nullptr;
    cudaError_t ec = cudaStreamEndCapture(s, &graph);
    if (st || e || ec) {
      if (graph) cudaGraphDestroy(graph);
      if (st) return st;
      return bfail(b, WFBP_ERR_CUDA, std::string("wfbp_batch_run: capture failed: ") +
                                         cudaGetErrorString(e ? e : ec));
    }
    b->graph = graph;
    BCUDA(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->key = key;
  }
  BCUDA(b, cudaGraphLaunch(b->exec, s));
  if (legacy) BCUDA(b, cudaStreamSynchronize(s));
  return WFBP_OK;
}

WFBP_API int wfbp_batch_check_device_status(wfbp_batch* b) {
  if (!b) return WFBP_ERR_INVALID_ARG;
  DevGuard g(b->device);
  int h = 0;
  BCUDA(b, cudaMemcpy(&h, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) {
    cudaMemset(b->d_err, 0, sizeof(int));
    return bfail(b, h == WFBP_ERR_TIMEOUT ? WFBP_ERR_TIMEOUT : WFBP_ERR_CUDA,
                 "the batched backprojection reported device error word " + std::to_string(h));
  }
  // the scans' rebin and filter stages report through their contexts' words
  for (int i = 0; i < (int)b->ctx.size(); i++) {
    const int st = wfbp_check_device_status(b->ctx[i]);
    if (st) return bfail(b, st, "scan " + std::to_string(i) + ": " + wfbp_last_error(b->ctx[i]));
  }
  return WFBP_OK;
}

// ---------------------------------------------------------------------------
// host buffers in, host buffers out
// ---------------------------------------------------------------------------
//
// The readings are copied scan by scan on a copy stream. The scans split in
// two groups in copy order: group A, the leading scans holding at least a
// quarter of the readings' bytes, is rebinned, filtered and backprojected (one
// persistent launch over its work items) as soon as its copies land, while
// group B's copies continue; A's volumes are thickened and copied back while
// group B is rebinned, filtered and backprojected (a second persistent
// launch). Same kernels and per-voxel sums as wfbp_batch_run: the volumes are
// identical. Synchronous, like wfbp_run_host.
WFBP_API int wfbp_batch_run_host(wfbp_batch* b, const float* const* raws_host, float* const* volumes_host,
                                 void* stream) {
  if (!b) return WFBP_ERR_INVALID_ARG;
  const int n = (int)b->ctx.size();
  if (!raws_host || !volumes_host) return bfail(b, WFBP_ERR_INVALID_ARG, "wfbp_batch_run_host: null pointer array");
  for (int i = 0; i < n; i++)
    if (!raws_host[i] || !volumes_host[i])
      return bfail(b, WFBP_ERR_INVALID_ARG, "wfbp_batch_run_host: null buffer for scan " + std::to_string(i));
  DevGuard g(b->device);
  const bool legacy = stream == nullptr;
  cudaStream_t s = legacy ? b->own : (cudaStream_t)stream;
  if (legacy) BCUDA(b, cudaStreamSynchronize(0));
  std::vector<wfbp_dims> d(n);
  double total = 0.0;
  for (int i = 0; i < n; i++) {
    wfbp_query(b->ctx[i], &d[i]);
    total += (double)d[i].raw_bytes;
  }
  if (b->raw_d.empty()) {
    b->raw_d.assign(n, nullptr);
    b->vol_d.assign(n, nullptr);
    for (int i = 0; i < n; i++) {
      BCUDA(b, cudaMalloc(&b->raw_d[i], d[i].raw_bytes));
      BCUDA(b, cudaMalloc(&b->vol_d[i], d[i].volume_bytes));
    }
  }
  if (!b->s_copy) BCUDA(b, cudaStreamCreateWithFlags(&b->s_copy, cudaStreamNonBlocking));
  if (b->ev.empty()) {
    b->ev.assign(n + 2, nullptr);  // per scan copy, caller order, group A thickened
    for (auto& e : b->ev) BCUDA(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  // group A: the shortest prefix with at least a quarter of the bytes
  int k = 0;
  for (double acc = 0.0; k < n && (k == 0 || acc < 0.25 * total); k++) acc += (double)d[k].raw_bytes;
  if (k >= n) k = n;
  if (k != b->split_k) {
    std::vector<int4> split;
    split.reserve(b->h_items.size());
    for (const int4& w : b->h_items)
      if (w.x < k) split.push_back(w);  // stable: each group keeps the cost order
    const int na = (int)split.size();
    for (const int4& w : b->h_items)
      if (w.x >= k) split.push_back(w);
    cudaFree(b->d_items_split);
    b->d_items_split = nullptr;
    BCUDA(b, cudaMalloc(&b->d_items_split, sizeof(int4) * std::max<size_t>(split.size(), 1)));
    BCUDA(b, cudaMemcpy(b->d_items_split, split.data(), sizeof(int4) * split.size(), cudaMemcpyHostToDevice));
    b->split_k = k;
    b->split_na = na;
  }
  // copies in scan order, after the caller's earlier work on its stream. From
  // pinned memory all are queued at once; from pageable memory (a copy holds
  // the host until it is staged) each just before its scan's work, so the
  // work queued earlier keeps the GPU busy meanwhile.
  bool pinned = true;
  for (int i = 0; i < n && pinned; i++) {
    cudaPointerAttributes pa;
    pinned = cudaPointerGetAttributes(&pa, raws_host[i]) == cudaSuccess && pa.type == cudaMemoryTypeHost;
  }
  cudaGetLastError();
  BCUDA(b, cudaEventRecord(b->ev[n], s));
  BCUDA(b, cudaStreamWaitEvent(b->s_copy, b->ev[n], 0));
  auto copy_in = [&](int i) -> int {
    BCUDA(b, cudaMemcpyAsync(b->raw_d[i], raws_host[i], d[i].raw_bytes, cudaMemcpyHostToDevice, b->s_copy));
    BCUDA(b, cudaEventRecord(b->ev[i], b->s_copy));
    return WFBP_OK;
  };
  if (pinned)
    for (int i = 0; i < n; i++)
      if (int e = copy_in(i)) return e;
  const int cpw = b->cfg.tile_x * b->cfg.tile_y / b->cfg.consumer_warps;
  auto group = [&](int i0, int i1, const int4* items, int n_items) -> int {
    for (int i = i0; i < i1; i++) {
      if (!pinned)
        if (int e = copy_in(i)) return e;
      BCUDA(b, cudaStreamWaitEvent(s, b->ev[i], 0));
      int st = wfbp_rebin(b->ctx[i], b->raw_d[i], b->reb[i], s);
      if (!st)
        st = wfbp_detail::filter_stage(b->ctx[i], b->reb[i], b->filt[i], b->scales[i], WFBP_LAYOUT_BACKPROJECTION, s);
      if (st) return bfail(b, st, "scan " + std::to_string(i) + ": " + wfbp_last_error(b->ctx[i]));
    }
    if (n_items > 0) {
      BCUDA(b, cudaMemsetAsync(b->d_next, 0, sizeof(unsigned), s));
      BCUDA(b, launch_backproject_tma_batch(b->precision == WFBP_PRECISION_MIXED ? 1 : 0, cpw, b->cfg.cols_per_step,
                                            b->cfg.consumer_warps, b->cfg.slab, b->zc, b->d_scans, items, n_items,
                                            b->d_next, b->d_err, b->smem, b->grid, s));
    }
    for (int i = i0; i < i1; i++) {
      int st = wfbp_thicken(b->ctx[i], b->native[i], b->vol_d[i], s);
      if (st) return bfail(b, st, "scan " + std::to_string(i) + ": " + wfbp_last_error(b->ctx[i]));
    }
    return WFBP_OK;
  };
  int st = group(0, k, b->d_items_split, b->split_na);
  if (st) return st;
  // group A's volumes go back on the copy stream while group B runs (issued
  // after group B's work is queued: a copy to pageable memory holds the host)
  BCUDA(b, cudaEventRecord(b->ev[n + 1], s));
  if (k < n) {
    st = group(k, n, b->d_items_split + b->split_na, b->n_items - b->split_na);
    if (st) return st;
  }
  BCUDA(b, cudaStreamWaitEvent(b->s_copy, b->ev[n + 1], 0));
  for (int i = 0; i < k; i++)
    BCUDA(b, cudaMemcpyAsync(volumes_host[i], b->vol_d[i], d[i].volume_bytes, cudaMemcpyDeviceToHost, b->s_copy));
  for (int i = k; i < n; i++)
    BCUDA(b, cudaMemcpyAsync(volumes_host[i], b->vol_d[i], d[i].volume_bytes, cudaMemcpyDeviceToHost, s));
  BCUDA(b, cudaStreamSynchronize(b->s_copy));
  BCUDA(b, cudaStreamSynchronize(s));
  return wfbp_batch_check_device_status(b);
}
