"""Benchmark of the helical WFBP path on B200.

One step = one full reconstruction (rebin -> filter -> backprojection ->
thickening) of one synthetic scan of the `rows64` workload (888 channels x 64
rows, 984 views/rotation, 10 rotations, 512 x 512 x 300 slices @ 1 mm),
through the C ABI. Metric: contributing backprojection voxel-view updates per
second over the whole step (whole job over all ranks), with s/volume beside
it. Inputs (2.2 GB raw frames) are larger than L2, so no flush is needed.
By default both precision forms run: the mixed form is the headline line,
the FP32 form is reported beside it ("fp32", "mixed_speedup_vs_fp32"), and
each form's volume is checked in HU against the FP64 oracle on one slab.
The rows64 line also carries "batch24": the 24 seeded uneven scans
reconstructed as one batch (mixed form, one persistent backprojection launch,
CUDA graph) against per-scan FP32 launches, with each scan's HU error against
the FP64 oracle on its middle slab (--no-batch skips it).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision both|fp32|mixed] [--workload rows64|small|ffs|batch24|...]

Under torchrun each rank reconstructs its own independently seeded scan
(weak scaling, no collective on the data path).
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "backproj voxel-view updates/s & s/volume at <=1 HU RMSE vs FP64; mixed vs FP32"
# DRAM read + write bytes and warp instructions per contributing update of one backprojection
# launch, from the ncu captures of rows64_short (2.3819501378e10 updates; profiles/
# k_bp_tma_rows64_short.md), by precision form and slab height (16-slice slabs stage each view
# window in twice as many CTAs); the kernel's binding limit is instruction issue
# ncu captures of k_bp_tma on rows64_short (2.3819501378e10 updates per launch;
# profiles/k_bp_tma_rows64_short.md): DRAM bytes and warp instructions per
# update, keyed by (form, configuration) for the shapes the autotuner picks on
# rows64, else by (form, slab height)
_SHORT_UPDATES = 2.3819501378e10
DRAM_BYTES_PER_UPDATE = {("fp32", 32): 14.42e9 / _SHORT_UPDATES,
                         ("mixed", 16): 14.39e9 / _SHORT_UPDATES,
                         ("fp32", 16): 21.08e9 / _SHORT_UPDATES,
                         ("mixed", 32): 13.18e9 / _SHORT_UPDATES,
                         ("mixed", "16x8/4w8s16"): 34.96e9 / _SHORT_UPDATES,
                         ("fp32", "16x8/8w8s32"): 15.38e9 / _SHORT_UPDATES,
                         ("fp32", "8x16/8w8s16"): 22.55e9 / _SHORT_UPDATES}
WARP_INST_PER_UPDATE = {("fp32", 32): 3.537e10 / _SHORT_UPDATES, ("mixed", 16): 3.428e10 / _SHORT_UPDATES,
                        ("fp32", 16): 3.475e10 / _SHORT_UPDATES, ("mixed", 32): 3.631e10 / _SHORT_UPDATES,
                        ("mixed", "16x8/4w8s16"): 3.6336e10 / _SHORT_UPDATES,
                        ("fp32", "16x8/8w8s32"): 3.4076e10 / _SHORT_UPDATES,
                        ("fp32", "8x16/8w8s16"): 3.4219e10 / _SHORT_UPDATES}
SMS, SCHEDULERS_PER_SM = 148, 4
UNIT = "voxel-view updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "fp32", "mixed"],
                    help="both: the mixed form is the headline line, the FP32 form is reported beside it")
    ap.add_argument("--workload", default="rows64")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-slices", type=int, default=8,
                    help="native slices the CPU baseline backprojects (spread over one rotation's feed)")
    ap.add_argument("--no-tune", action="store_true", help="keep the default backprojection configuration")
    ap.add_argument("--no-hu", action="store_true", help="skip the HU check against the FP64 oracle")
    ap.add_argument("--no-batch", action="store_true",
                    help="rows64: skip the batch24 summary (24 uneven scans, one persistent launch)")
    ap.add_argument("--batch-hu-scans", type=int, default=24,
                    help="batch24 summary: scans checked against the FP64 oracle on their middle slab")
    ap.add_argument("--bp-config", default=None,
                    help="fixed backprojection configuration, e.g. 16x20/8w20s16 (no tuning)")
    return ap.parse_args()


def load_peaks():
    """(HBM GB/s, BF16 TFLOP/s burst, BF16 TFLOP/s sustained, source)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return (d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0),
                "measured")
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def baseline_positions(spec, cg, rp, n=8):
    """n native slice indices spread evenly over one rotation's table feed
    centred on the middle of the native slice list: where the CPU baseline
    samples the backprojection."""
    from oracle import oracle as O
    zn, _ = O.slice_locations(cg, rp)
    mid = zn.size // 2
    span = max(1, int(round(spec.feed / max(1e-6, abs(float(zn[1] - zn[0]))))))  # native slices per rotation
    lo = max(0, mid - span // 2)
    hi = min(zn.size, lo + span)
    step = max(1, (hi - lo) // n)
    return [int(lo + step * i) for i in range(n) if lo + step * i < hi]


def cpu_baseline(spec, raw_host_fn, positions):
    """The reference's path on the host cores (the oracle's FP32 transcript,
    all threads): rebin+filter of the window of views the sampled native
    slices need, and the backprojection of those slices at full
    resolution; scaled to the full volume linearly in views (rebin+filter)
    and in slices (backprojection)."""
    import numpy as np
    from freect_b200 import scans  # noqa: F401
    from oracle import oracle as O
    nthreads = os.cpu_count() or 1
    O.set_threads(nthreads)
    tube, table = spec.views()
    cg, gp = O.configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    zn, zr = O.slice_locations(cg, rp)
    zs = zn[np.asarray(positions)]
    # views that pass the z cull for these slices, plus the rebin's view reach
    sel = np.nonzero((table >= zs.min() - cg.z_rot - 1.0) & (table <= zs.max() + cg.z_rot + 1.0))[0]
    reach = int(math.ceil(0.5 * spec.nch * spec.dbeta / (2 * math.pi / spec.P))) + 2
    v0 = max(0, sel[0] - reach)
    v0 -= v0 % (spec.P // 2)  # keep half-turn alignment of theta~
    v1 = min(spec.V, sel[-1] + reach + 1)
    sub = scans.ScanSpec(**{**spec.__dict__})
    sub.rotations = (v1 - v0) / spec.P
    raw = raw_host_fn(v0, v1)
    stube, stable = tube[v0:v1], table[v0:v1]
    scg, sgp = O.configure_geometry(sub.meta(), stable)
    scg.z_rot = cg.z_rot
    sgp.z_rot_over_2_pi = gp.z_rot_over_2_pi
    t0 = time.perf_counter()
    taps = O.taps_fft_from_half(scg, O.taps_f64(scg, spec.window).astype(np.float32))
    filt = O.rebin_filter_ref32(scg, raw, taps, q8=True)
    t1 = time.perf_counter()
    vn = O.backproject_ref32(scg, rp, sgp, filt, stube, stable, zs)
    t2 = time.perf_counter()
    # updates in the sample (FP64 oracle's count on the same views and slices)
    _, n_sample = O.backproject_f64(scg, rp, filt.astype(np.float64), stube.astype(np.float64),
                                    stable.astype(np.float64), zs.astype(np.float64))
    t_rf_full = (t1 - t0) * spec.V / float(v1 - v0)
    t_bp_full = (t2 - t1) * zn.size / float(zs.size)
    return {"t_rf_sample": t1 - t0, "t_bp_sample": t2 - t1, "views": int(v1 - v0), "slices": int(zs.size),
            "positions": [int(x) for x in positions], "native_slices": int(zn.size),
            "updates_sample": int(n_sample), "t_full_est": t_rf_full + t_bp_full, "cores": nthreads,
            "bp_updates_per_s": n_sample / (t2 - t1), "updates_full_est": n_sample * zn.size / float(zs.size)}


def run_reference(args, rank):
    """--impl reference: the reference's path on host cores, bounded sample
    per step: step i rebins and filters the view window of native slice
    position i mod 8 (8 positions spread over one rotation's table feed at
    the centre of the volume) and backprojects that slice; each step's time
    is scaled to the full volume, the line reports the median."""
    import numpy as np
    from freect_b200 import scans
    from oracle import oracle as O
    spec = scans.WORKLOADS[args.workload]()
    tube, table = spec.views()
    cg, _ = O.configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    positions = baseline_positions(spec, cg, rp)
    cache = {}

    def raw_host(v0, v1):
        for (a, b), arr in cache.items():
            if a <= v0 and v1 <= b:
                return arr[v0 - a:v1 - a]
        s = spec.synth()
        s.n_readings = v1 - v0
        s.angle0 = s.angle0 + v0 * s.dangle
        s.z0 = s.z0 + v0 * s.dz
        cache[(v0, v1)] = O.synth_project(s, spec.ellipsoids())
        return cache[(v0, v1)]

    # one synthesis of the window all positions need (outside the timed steps)
    first = cpu_baseline(spec, raw_host, positions)
    times = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(spec, raw_host, [positions[i % len(positions)]])
        if i >= args.warmup:
            times.append(r)
    ests = sorted(t["t_full_est"] for t in times)
    est = ests[len(ests) // 2]
    full_updates = first["updates_full_est"]
    value = full_updates / est
    sample = ("oracle FP32 transcript (q8 texture weights) on %d host threads; each step: rebin+filter of the ~%d "
              "views one native slice needs (of %d) and the backprojection of that slice at %dx%d, scaled linearly "
              "to the full volume (%d native slices); the step's slice cycles through %d positions spread over one "
              "rotation's table feed; median over steps; updates from the FP64 count of all %d positions"
              % (times[0]["cores"], times[0]["views"], spec.V, spec.nx, spec.ny, first["native_slices"],
                 len(positions), len(positions)))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": est * 1000.0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ellipsoid phantom)",
            "config": {"workload": spec.name, "channels": spec.nch, "rows": spec.nr, "views": spec.V,
                       "volume": [spec.n_slices, spec.ny, spec.nx], "l2": "inputs larger than L2"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": times[0]["cores"], "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "s_per_volume": est, "sample_seconds_per_step": sorted(t["t_rf_sample"] + t["t_bp_sample"]
                                                                   for t in times)[len(times) // 2],
            "s_per_volume_range": [ests[0], ests[-1]]}
    print(json.dumps(line))


def autotune_name(key):
    from freect_b200 import autotune
    return autotune.config_name(key)


def run_diff(args, rank, world, local, dist):
    """--workload diff4: one training step of the differentiable WFBP on a
    batch of 4 scans of the small scanner (672 x 16, 1160 views/rotation, 3
    rotations, 256^2 x 16), independently seeded phantoms: forward through
    the four FP32 stages, MSE to a target volume, backward through the
    adjoint kernels to the raw readings and 64 learnable filter taps. The
    target is each scan's noiseless reconstruction (computed once on the GPU).
    Updates are counted for the forward and the adjoint backprojection.
    --workload diff1: the same step on one scan of the small scanner reduced
    to 2 rotations and 192^2 x 12 slices, a profiling-size case of the same
    kernels (about 2 GB on the device)."""
    import torch
    from freect_b200 import scans, wfbp
    from freect_b200.autograd import Reconstructor

    dev = torch.device("cuda", local)
    n_scans = 4 if args.workload == "diff4" else 1
    specs = [scans.small(seed=4 * rank + i) for i in range(n_scans)]
    if args.workload == "diff1":
        for sp in specs:
            sp.rotations = 2
            sp.nx = sp.ny = 192
            sp.n_slices = 12
    tube, table = specs[0].views()
    cg, gp = wfbp.configure_geometry(specs[0].meta(), table)
    rp = specs[0].recon_config()
    rec = Reconstructor(cg, rp, tube, table, n_taps=64, device=local)
    shape = rec.raw_shape
    raws, targets = [], []
    for sp in specs:
        r = torch.empty(shape, dtype=torch.float32, device=dev)
        wfbp.synth_project(sp.synth(), sp.ellipsoids(), r)
        raws.append(r)
        clean = torch.empty(shape, dtype=torch.float32, device=dev)
        wfbp.synth_project(sp.synth(i0=0), sp.ellipsoids(), clean)
        v = rec.ctx.alloc("volume")
        rec.ctx.run(clean, v)
        targets.append(v)
    raw = torch.stack(raws)
    tgt = torch.stack(targets)
    mask = torch.isfinite(tgt)
    del raws, targets
    # contributing updates of one forward backprojection (the adjoint visits the same pairs)
    reb, flt, vn = rec.buf("rebinned"), rec.buf("filtered"), rec.buf("native")
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    rec.ctx.rebin(raw[0], reb)
    rec.ctx.filter(reb, flt)
    rec.ctx.backproject(flt, vn, update_count=cnt)
    torch.cuda.synchronize()
    updates = 2 * n_scans * int(cnt.item())
    tuned = None
    if not args.no_tune:
        # forward backprojection launch shape from the autotuner (outside the timed region)
        from freect_b200 import autotune
        tuned = autotune.tune_backprojection(rec.ctx, flt, vn, use_cache=False)["config"]
    try:
        bp_name = autotune_name(rec.ctx.bp_config().key())
    except wfbp.WfbpError:  # the reference-layout kernel (no TMA launch fits)
        bp_name = "reference layout"
    taps = torch.nn.Parameter(rec.initial_taps())
    raw.requires_grad_(True)

    def step():
        vol = rec(raw, taps)
        m = mask & torch.isfinite(vol)
        loss = ((vol - tgt)[m] ** 2).mean()
        raw.grad = None
        taps.grad = None
        loss.backward()
        return loss

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    rec.ctx.check_device_status()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        loss = step()
    b.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = a.elapsed_time(b) / args.steps
    tm = torch.tensor([ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    ms = float(tm.item())
    # end to end: raw readings from pinned host memory, loss and tap gradient back to the host
    raw_h = raw.detach().cpu().pin_memory()
    g_h = torch.empty(64, dtype=torch.float32).pin_memory()

    copy_stream = torch.cuda.Stream(device=dev)
    ready = [torch.cuda.Event() for _ in range(n_scans)]

    def e2e_step():
        # scan b's readings are copied on a second stream while the forward
        # reconstructs scan b - 1 (the forward waits for each scan's event)
        copy_stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.no_grad(), torch.cuda.stream(copy_stream):
            for b in range(n_scans):
                raw[b].copy_(raw_h[b], non_blocking=True)
                ready[b].record(copy_stream)
        vol = rec(raw, taps, ready)
        m = mask & torch.isfinite(vol)
        l = ((vol - tgt)[m] ** 2).mean()
        raw.grad = None
        taps.grad = None
        l.backward()
        g_h.copy_(taps.grad, non_blocking=True)
        return l.item()

    e2e_step()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        e2e_step()
    b.record(stream)
    torch.cuda.synchronize()
    ems = a.elapsed_time(b) / args.steps
    line = {"metric": METRIC, "value": updates * world / (ms / 1000.0), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (%d seeded head-like ellipsoid phantoms per rank, Poisson noise)" % n_scans,
            "config": {"workload": args.workload, "scans": n_scans, "channels": specs[0].nch, "rows": specs[0].nr,
                       "views": specs[0].V, "volume": [specs[0].n_slices, specs[0].ny, specs[0].nx],
                       "learnable_taps": 64, "step": "forward + MSE + backward to raw readings and taps",
                       "updates_counted": "forward and adjoint backprojection",
                       "parallelism": "independent batch per GPU",
                       "l2": "inputs larger than L2 (%.2f GB raw)" % (raw.numel() * 4 / 1e9),
                       "bp_config": bp_name},
            "updates_per_step": updates, "loss": float(loss.item()),
            # per step and scan: (rebin, filter, backprojection, thickening) forward and
            # (thickening, backprojection, filter, rebin adjoints + 2 tap-gradient kernels) backward
            "gpu_launches": n_scans * (4 + 6) * args.steps,
            "e2e": {"value": updates * world / (ems / 1000.0), "unit": UNIT, "ms_per_step": ems,
                    "h2d_bytes_per_step": int(raw.numel() * 4), "d2h_bytes_per_step": 4 + 64 * 4},
            "clocks": clk}
    if rank == 0:
        print(json.dumps(line))


def measure_batch(args, rank, world, local, dist, candidates=None, hu_scans=24, steps=None, warmup=None):
    """24 seeded uneven scans reconstructed as one batch (mixed form: per-scan
    rebin + tensor-core filter, ONE persistent backprojection launch over all
    scans, per-scan thickening, replayed as a CUDA graph), against the same
    scans as per-scan FP32 launches; each of the first `hu_scans` scans'
    mixed volume against the FP64 oracle on its middle slab. candidates:
    backprojection configuration names the batch autotuner may try (None:
    all that fit). Returns the summary dict."""
    import numpy as np
    import torch
    from freect_b200 import abi_types as T
    from freect_b200 import autotune, scans, wfbp

    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    dev = torch.device("cuda", local)
    specs = scans.batch_specs(seed=rank, n=24)
    ctxs, raws, vols, views = [], [], [], []
    for sp in specs:
        tube, table = sp.views()
        cg, gp = wfbp.configure_geometry(sp.meta(), table)
        c = wfbp.Context(cg, sp.recon_config(), wfbp.make_ext(precision=T.PRECISION_MIXED, filter_window=sp.window),
                         device=local)
        c.set_views(tube, table)
        ctxs.append(c)
        views.append((cg, tube, table))
        r = c.alloc("raw")
        wfbp.synth_project(sp.synth(), sp.ellipsoids(), r)
        raws.append(r)
        vols.append(c.alloc("volume"))
    torch.cuda.synchronize()
    batch = wfbp.Batch(ctxs)
    stream = torch.cuda.Stream(device=dev)
    tuned = None
    if not args.no_tune:
        tuned = autotune.tune_batch(batch, raws, vols, use_cache=False, candidates=candidates)

    # per-scan FP32 launches (the comparison) and the contributing updates
    # (counted once per scan by the FP32 form, outside every timed region)
    updates, fp32_ms, v32s = 0, 0.0, []
    for sp, r, v in zip(specs, raws, vols):
        tube, table = sp.views()
        cg, gp = wfbp.configure_geometry(sp.meta(), table)
        c32 = wfbp.Context(cg, sp.recon_config(), wfbp.make_ext(filter_window=sp.window, tex_weights=1,
                                                                filtered_layout=T.LAYOUT_BACKPROJECTION),
                           device=local)
        c32.set_views(tube, table)
        reb, flt, vn, v32 = c32.alloc("rebinned"), c32.alloc("filtered"), c32.alloc("native"), c32.alloc("volume")
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        c32.rebin(r, reb)
        c32.filter(reb, flt)
        c32.backproject(flt, vn, update_count=cnt)
        del reb, flt, vn
        c32.run(r, v32)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c32.run(r, v32)
        e1.record()
        torch.cuda.synchronize()
        fp32_ms += e0.elapsed_time(e1)
        updates += int(cnt.item())
        v32s.append(v32)
        c32.close()

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            batch.run(raws, vols)
        stream.synchronize()
        batch.check_device_status()
        hu_rms_fp32 = []
        for v, v32 in zip(vols, v32s):
            a, b = v.cpu().numpy(), v32.cpu().numpy()
            m = np.isfinite(a) & np.isfinite(b)
            hu_rms_fp32.append(float(np.sqrt(np.mean(((a[m] - b[m]) * 1000.0 / scans.MU_WATER) ** 2)))
                               if m.any() else None)
        del v32s
        clocks = ClockSampler(local)
        clocks.start()
        time.sleep(0.3)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(steps):
            batch.run(raws, vols)
        t1.record(stream)
        stream.synchronize()
        clk = clocks.stop()
    ms = t0.elapsed_time(t1) / steps
    tm = torch.tensor([ms], dtype=torch.float64, device=dev)
    ua = torch.tensor([float(updates)], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        dist.all_reduce(ua, op=dist.ReduceOp.SUM)
    ms = float(tm.item())
    value = float(ua.item()) / (ms / 1000.0)

    e2e = None
    if not args.no_e2e:
        hr = [torch.empty(r.shape, dtype=torch.float32, pin_memory=True) for r in raws]
        hv = [torch.empty(v.shape, dtype=torch.float32, pin_memory=True) for v in vols]
        for a, b in zip(hr, raws):
            a.copy_(b.cpu())
        h2d = sum(r.numel() * 4 for r in raws)
        d2h = sum(v.numel() * 4 for v in vols)
        with torch.cuda.stream(stream):
            batch.run_host(hr, hv, stream=stream)  # wfbp_batch_run_host: copies overlap the two launches
            stream.synchronize()
            if dist:
                dist.barrier()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(steps):
                batch.run_host(hr, hv, stream=stream)
            a1.record(stream)
            stream.synchronize()
        ems = a0.elapsed_time(a1) / steps
        te = torch.tensor([ems], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        ems = float(te.item())
        e2e = {"value": float(ua.item()) / (ems / 1000.0), "unit": UNIT, "ms_per_step": ems,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}
        del hr, hv

    # the checker: each scan's mixed volume against the FP64 oracle on its middle slab
    hu64 = []
    if rank == 0 and world == 1 and hu_scans and not args.no_hu:
        for sp, r, v, (cg, tube, table) in list(zip(specs, raws, vols, views))[:hu_scans]:
            try:
                h = hu_vs_fp64(sp, cg, sp.recon_config(), tube, table, r, v)
                hu64.append({"scan": sp.name, "rms": h["rms"], "max": h["max"], "voxels": h["voxels"]})
            except Exception as ex:  # reported, not fatal
                hu64.append({"scan": sp.name, "error": repr(ex)})
    n_scans, n_items = batch.size()
    out = {"value": value, "ms": ms, "updates": updates, "fp32_per_scan_launches_ms": fp32_ms,
           "speedup_vs_fp32_per_scan": fp32_ms / ms, "hu_rms_mixed_vs_fp32_per_scan": hu_rms_fp32,
           "hu_vs_fp64_per_scan": hu64,
           "hu_vs_fp64_rms_max": max((h["rms"] for h in hu64 if "rms" in h), default=None),
           "scans": n_scans, "work_items": n_items,
           "shapes": ["%dx%dx%d/%d->%dx%dx%d" % (sp.nch, sp.nr, sp.P, sp.V, sp.nx, sp.ny, sp.n_slices)
                      for sp in specs],
           "bp_config": autotune.config_name(batch.bp_config().key()),
           "bp_tuning_ms": tuned["times_ms"] if tuned else None,
           "raw_gb": sum(r.numel() for r in raws) * 4 / 1e9,
           "gpu_launches": (3 * n_scans + 1) * steps, "e2e": e2e, "clocks": clk}
    batch.close()
    for c in ctxs:
        c.close()
    return out


def run_batch(args, rank, world, local, dist):
    """--workload batch24: the batch as the bench's headline line."""
    b = measure_batch(args, rank, world, local, dist)
    line = {"metric": METRIC, "value": b["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": b["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f16-storage/f32-accumulate",
            "data": "synthetic (24 seeded uneven helical scans, ellipsoid phantoms, Poisson noise)",
            "config": {"workload": "batch24", "scans": b["scans"], "work_items": b["work_items"],
                       "shapes": b["shapes"],
                       "precision": "mixed, one persistent backprojection launch, CUDA graph replay",
                       "parallelism": "independent batch per GPU",
                       "l2": "inputs larger than L2 (%.1f GB raw frames)" % b["raw_gb"],
                       "bp_config": b["bp_config"], "bp_tuning_ms": b["bp_tuning_ms"]},
            "updates_per_step": b["updates"], "fp32_per_scan_launches_ms": b["fp32_per_scan_launches_ms"],
            "speedup_vs_fp32_per_scan": b["speedup_vs_fp32_per_scan"],
            "hu_rms_mixed_vs_fp32_per_scan": b["hu_rms_mixed_vs_fp32_per_scan"],
            "hu_vs_fp64_per_scan": b["hu_vs_fp64_per_scan"],
            "gpu_launches": b["gpu_launches"], "e2e": b["e2e"], "clocks": b["clocks"]}
    if rank == 0:
        print(json.dumps(line))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args, rank)
        return

    import numpy as np
    import torch
    from freect_b200 import abi_types as T
    from freect_b200 import scans, wfbp

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    if args.workload in ("batch24", "diff4", "diff1"):
        (run_batch if args.workload == "batch24" else run_diff)(args, rank, world, local, dist)
        if dist:
            dist.destroy_process_group()
        return

    spec = scans.WORKLOADS[args.workload](seed=rank)
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    raw = torch.empty((spec.V, spec.nr, spec.nch), dtype=torch.float32, device=dev)
    wfbp.synth_project(spec.synth(), spec.ellipsoids(), raw)
    torch.cuda.synchronize()
    forms = ["mixed", "fp32"] if args.precision == "both" else [args.precision]
    res = {f: measure_form(args, f, spec, cg, rp, tube, table, raw, dev, stream, dist, local) for f in forms}
    head = res[forms[0]]
    line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": head["dtype"],
            "data": "synthetic (seeded ellipsoid phantom, Poisson noise)",
            "config": {"workload": spec.name, "channels": spec.nch, "rows": spec.nr, "views": spec.V,
                       "volume": [head["dims"].n_slices_requested, head["dims"].ny, head["dims"].nx],
                       "native_slices": head["dims"].n_slices_native, "precision": forms[0],
                       "parallelism": "independent scan per GPU",
                       "l2": "inputs larger than L2 (%.2f GB raw frames, %.2f GB filtered rows)"
                             % (head["dims"].raw_bytes / 1e9, head["dims"].filtered_bytes / 1e9),
                       "bp_config": head["bp_config"], "bp_tuning_ms": head["tuning"]},
            "s_per_volume": head["ms"] / 1000.0, "updates_per_volume": head["updates"],
            "stage_ms": head["stage"], "roofline": head["roofline"], "stage_rooflines": head["stages"],
            "gpu_launches": 4 * args.steps,
            "e2e": head["e2e"], "clocks": head["clocks"]}
    if len(forms) == 2:
        f32 = res["fp32"]
        line["fp32"] = {k: f32[k] for k in ("value", "ms", "stage", "roofline", "stages", "e2e", "bp_config",
                                            "clocks", "updates") if k in f32}
        line["mixed_speedup_vs_fp32"] = {"device": f32["ms"] / head["ms"],
                                         "e2e": (f32["e2e"]["ms_per_step"] / head["e2e"]["ms_per_step"])
                                         if head["e2e"] and f32["e2e"] else None}
    if args.workload == "rows64" and not args.no_batch:
        # the batched uneven scans (24 scans, one persistent launch): the batch
        # autotuner tries the three fastest rows64 mixed shapes that fit
        tms = head["tuning"] or {}
        cands = sorted(tms, key=tms.get)[:3] if tms else None
        try:
            line["batch24"] = measure_batch(args, rank, world, local, dist, candidates=cands,
                                            hu_scans=args.batch_hu_scans, steps=min(args.steps, 3), warmup=1)
        except Exception as ex:  # reported, not fatal
            line["batch24"] = {"error": repr(ex)}
    if rank == 0 and world == 1 and not args.no_cpu and not args.no_hu:
        # the checker, on the host cores: each form's volume against the FP64 oracle on one slab
        for f in forms:
            try:
                hu = hu_vs_fp64(spec, cg, rp, tube, table, raw, res[f]["volume"])
            except Exception as ex:  # reported, not fatal
                hu = {"error": repr(ex)}
            if f == forms[0]:
                line["hu_vs_fp64"] = hu
            else:
                line["fp32"]["hu_vs_fp64"] = hu
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            from oracle import oracle as O
            pos = baseline_positions(spec, O.configure_geometry(spec.meta(), table)[0], rp, n=args.cpu_slices)
            cb = cpu_baseline(spec, lambda v0, v1: raw[v0:v1].cpu().numpy(), pos)
            full = head["updates"] / cb["t_full_est"]
            line["cpu_baseline"] = {
                "value": full, "unit": UNIT, "cores": cb["cores"], "kind": "port",
                "sample": "oracle FP32 transcript (q8 texture weights): rebin+filter of the %d of %d views that %d "
                          "native slices spread over one rotation's table feed need, backprojection of those %d "
                          "of %d native slices (%d updates) in %.1f s + %.1f s; scaled linearly to the full volume"
                          % (cb["views"], spec.V, cb["slices"], cb["slices"], head["dims"].n_slices_native,
                             cb["updates_sample"], cb["t_rf_sample"], cb["t_bp_sample"]),
                "s_per_volume_est": cb["t_full_est"], "positions": cb["positions"]}
        except Exception as ex:  # reported, not fatal
            line["cpu_baseline"] = {"error": repr(ex)}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def hu_vs_fp64(spec, cg, rp, tube, table, raw, vol):
    """HU error of `vol` against the FP64 oracle on the slab of the middle
    requested slice (oracle/slab_check.py). Returns rms, max, voxels."""
    from oracle.slab_check import hu_vs_fp64_slab
    return hu_vs_fp64_slab(spec, cg, rp, tube, table, lambda a0, a1: raw[a0:a1].cpu().numpy(),
                           lambda r0, r1: vol[r0:r1].cpu().numpy())


def stage_rooflines(form, ctx, d, updates, stage, clk):
    """Per-stage roofline fractions of one step, from the library's stage
    events of the timed steps (ms per stage), the measured peaks and the
    SM clock sampled during the timed region.

    backproject: instruction issue (the binding limit; ncu: 71-76 % issue
    active, no memory pipe near its peak): warp instructions per update from
    the ncu capture of the same kernel x updates / time, against one warp
    instruction per scheduler per clock. DRAM traffic per launch (the same
    capture, scaled by updates) is reported against the compulsory bytes
    (filtered rows read once, native volume written once).
    rebin: HBM, raw frames read once + rebinned output written once.
    filter: tensor pipe (mixed: 3 split-FP16 products of 2 (V nr) nch^2
    FLOP each, against the sustained cuBLAS BF16 rate, the same tensor rate
    as FP16) or FP32 FFMA (FP32
    form: 2 (V nr) nch^2 FLOP against 148 SMs x 128 lanes x 2 x clock)."""
    hbm, bf16, bf16_sus, peak_src = load_peaks()
    mhz = (clk or {}).get("sm_mhz") or 1965.0
    bpc = ctx.bp_config()
    slab, shape = bpc.slab, autotune_name(bpc.key())
    t_bp = stage["backproject"] / 1000.0
    wipu = WARP_INST_PER_UPDATE.get((form, shape), WARP_INST_PER_UPDATE.get((form, slab)))
    ipeak = SMS * SCHEDULERS_PER_SM * mhz * 1e6
    dram_per_update = DRAM_BYTES_PER_UPDATE.get((form, shape), DRAM_BYTES_PER_UPDATE.get((form, slab)))
    src = "configuration %s" % shape if (form, shape) in WARP_INST_PER_UPDATE else "slab height %d" % slab
    traffic = dram_per_update * updates if dram_per_update else None
    compulsory = d.filtered_bytes + d.native_volume_bytes
    bp = {"bound": "issue", "kernel": "backproject", "achieved": wipu * updates / t_bp if wipu else None,
          "peak": ipeak, "unit": "warp instructions/s",
          "frac": (wipu * updates / t_bp / ipeak) if wipu else None,
          "traffic": traffic, "compulsory_bytes": compulsory,
          "traffic_over_compulsory": traffic / compulsory if traffic else None,
          "dram_gbs": traffic / t_bp / 1e9 if traffic else None,
          "dram_frac_of_hbm": traffic / t_bp / 1e9 / hbm if traffic else None,
          "updates_per_s": updates / t_bp,
          "warp_inst_per_update": wipu,
          "note": "warp instructions per update and DRAM bytes per update from the ncu capture of the same "
                  "kernel and %s on rows64_short (profiles/), scaled by this launch's updates; peak = "
                  "%d SMs x %d schedulers x %.0f MHz (sampled); taps are shared-memory reads after one TMA "
                  "staging per view window" % (src, SMS, SCHEDULERS_PER_SM, mhz)}
    samples = d.n_views * d.n_rows * d.n_channels
    rebin_bytes = d.raw_bytes + samples * 4  # FP32 rows, or the two FP16 operand planes
    t_rb = stage["rebin"] / 1000.0
    rebin = {"bound": "hbm", "kernel": "rebin", "achieved": rebin_bytes / t_rb / 1e9, "peak": hbm, "unit": "GB/s",
             "frac": rebin_bytes / t_rb / 1e9 / hbm, "algorithmic_bytes": rebin_bytes,
             "note": "raw frames read once + %d output samples x 4 B written" % samples}
    rows = d.n_views * d.n_rows
    t_f = stage["filter"] / 1000.0
    if form == "mixed":
        flop = 3 * 2.0 * rows * d.n_channels * d.n_channels
        filt = {"bound": "tensor", "kernel": "toeplitz_tc", "achieved": flop / t_f / 1e12, "peak": bf16_sus,
                "unit": "TFLOP/s", "frac": flop / t_f / 1e12 / bf16_sus, "algorithmic_flop": flop,
                "note": "3 split-FP16 products (hi*hi, hi*lo, lo*hi) of 2 M K N, M = views x rows, K = N = "
                        "channels, against the sustained cuBLAS BF16 rate (FP16 runs at the same tensor rate)"}
    else:
        flop = 2.0 * rows * d.n_channels * d.n_channels
        fpk = SMS * 128 * 2 * mhz * 1e6 / 1e12
        filt = {"bound": "fp32", "kernel": "toeplitz_f32", "achieved": flop / t_f / 1e12, "peak": fpk,
                "unit": "TFLOP/s", "frac": flop / t_f / 1e12 / fpk, "algorithmic_flop": flop,
                "note": "FP32 FFMA Toeplitz, peak = 148 SMs x 128 lanes x 2 FLOP x sampled clock"}
    for r in (bp, rebin, filt):
        r["peak_source"] = peak_src if r is not filt or form == "mixed" else "nominal"
        r["ms"] = {"backproject": stage["backproject"], "rebin": stage["rebin"], "toeplitz_tc": stage["filter"],
                   "toeplitz_f32": stage["filter"]}[r["kernel"]]
    return bp, {"backproject": bp, "rebin": rebin, "filter": filt}


def measure_form(args, form, spec, cg, rp, tube, table, raw, dev, stream, dist, local):
    import torch
    from freect_b200 import abi_types as T
    from freect_b200 import autotune, wfbp
    prec = T.PRECISION_MIXED if form == "mixed" else T.PRECISION_FP32
    ext = wfbp.make_ext(precision=prec, filter_window=spec.window, tex_weights=1 if prec == T.PRECISION_FP32 else 0,
                        filtered_layout=T.LAYOUT_BACKPROJECTION)
    ctx = wfbp.Context(cg, rp, ext, device=local)
    ctx.set_views(tube, table)
    d = ctx.dims
    reb = ctx.alloc("rebinned")
    filt = ctx.alloc("filtered")
    scales = ctx.alloc("row_scales")
    vn = ctx.alloc("native")
    vol = ctx.alloc("volume")
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)

    def step(count=None):
        ctx.rebin(raw, reb)
        ctx.filter(reb, filt, scales)
        ctx.backproject(filt, vn, scales, update_count=count)
        ctx.thicken(vn, vol)

    tuned = None
    if not args.no_tune and not args.bp_config:
        # backprojection launch configuration from the autotuner (outside the timed region)
        ctx.rebin(raw, reb)
        ctx.filter(reb, filt, scales)
        tuned = autotune.tune_backprojection(ctx, filt, vn, row_scales=scales, use_cache=False)
    if args.bp_config:
        ctx.set_bp_config(autotune.parse_config_name(args.bp_config))
    step(cnt)  # counts the contributing updates once, outside the timed region
    torch.cuda.synchronize()
    updates = int(cnt.item())
    for _ in range(args.warmup):
        ctx.run(raw, vol)
    torch.cuda.synchronize()

    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # one step = wfbp_run (rebin, filter, backprojection with the thickening of
    # the slices inside a slab fused into its write-back, the remaining
    # slices' thickening), with the library's own stage events
    stage = {"rebin": 0.0, "filter": 0.0, "backproject": 0.0, "thicken": 0.0}
    start.record(stream)
    for i in range(args.steps):
        for k, v in ctx.run_timed(raw, vol).items():
            stage[k] += v
    stop.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    total_ms = start.elapsed_time(stop)
    stage = {k: v / args.steps for k, v in stage.items()}
    ms = total_ms / args.steps
    t_max = torch.tensor([ms], dtype=torch.float64, device=dev)
    u_all = torch.tensor([float(updates)], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.all_reduce(u_all, op=dist.ReduceOp.SUM)
    ms = float(t_max.item())
    value = float(u_all.item()) / (ms / 1000.0)

    # end to end through the public API with host buffers (pinned)
    e2e = None
    if not args.no_e2e:
        raw_h = torch.empty(raw.shape, dtype=torch.float32, pin_memory=True)
        raw_h.copy_(raw.cpu())
        vol_h = torch.empty(vol.shape, dtype=torch.float32, pin_memory=True)
        ctx.run_host(raw_h, vol_h)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            ctx.run_host(raw_h, vol_h)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / args.steps
        te = torch.tensor([ems], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        ems = float(te.item())
        e2e = {"value": float(u_all.item()) / (ems / 1000.0), "unit": UNIT, "ms_per_step": ems,
               "h2d_bytes_per_step": int(d.raw_bytes), "d2h_bytes_per_step": int(d.volume_bytes)}

    roofline, stages = stage_rooflines(form, ctx, d, updates, stage, clk)
    out = {"value": value, "ms": ms, "stage": stage, "updates": updates, "e2e": e2e, "clocks": clk,
           "roofline": roofline, "stages": stages, "dims": d, "tuning": tuned["times_ms"] if tuned else None,
           "bp_config": autotune.config_name(ctx.bp_config().key()),
           "dtype": "f32" if prec == T.PRECISION_FP32 else "f16-storage/f32-accumulate"}
    out["volume"] = vol
    ctx.close()
    return out


if __name__ == "__main__":
    main()
