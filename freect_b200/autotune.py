"""Autotuner for the backprojection launch configuration.

The reference launches backproject_kernel with one fixed block shape
(ReconstructionMachine.cu:347-351). Here the column tile and the number of
columns accumulated per pass over a view window are chosen per geometry:
every configuration the library reports as fitting (wfbp_bp_configs) is
timed with CUDA events on the caller's filtered projections, the fastest is
set on the context (wfbp_set_bp_config), and the choice is cached in a JSON
file keyed by the geometry, so later contexts of the same shape skip the
timing.
"""
import json
import os

from . import abi_types as T

_DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "freect_b200", "bp_tune.json")


def cache_path():
    return os.environ.get("FREECT_B200_TUNE_CACHE", _DEFAULT_CACHE)


def signature(ctx):
    """Key of a tuning result: what the backprojection's cost depends on."""
    d = ctx.dims
    cg, gp = ctx.geometry()
    return "v3|V%d|nr%d|nch%d|P%d|%dx%dx%d|prec%d|fov%.3f|ps%.5f|zrot%.4f" % (
        d.n_views, d.n_rows, d.n_channels, int(cg.projections_per_rotation), d.nx, d.ny, d.n_slices_native,
        d.precision, ctx.rp.recon_fov, gp.pixel_scale, cg.z_rot)


def config_name(key):
    """'16x16/4w16s32': column tile, columns per pass, consumer warps, slab slices."""
    return "%dx%d/%dw%ds%d" % tuple(key)


def parse_config_name(name):
    """Inverse of config_name: '16x20/8w20s16' -> (16, 20, 8, 20, 16)."""
    import re
    m = re.fullmatch(r"(\d+)x(\d+)/(\d+)w(\d+)s(\d+)", name.strip())
    if not m:
        raise ValueError("backprojection configuration %r is not of the form TXxTY/CwNsS" % name)
    return tuple(int(g) for g in m.groups())


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp.%d" % os.getpid()
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune_backprojection(ctx, filtered, volume_native, row_scales=None, reps=2, use_cache=True, path=None):
    """Times each fitting configuration and sets the fastest on `ctx`.

    filtered / volume_native: device tensors of the context's backprojection
    input and output (the output is overwritten). Returns a dict with the
    chosen configuration, the per-configuration times (ms) and whether the
    result came from the cache.
    """
    import torch

    path = path or cache_path()
    key = signature(ctx)
    if use_cache:
        table = _load(path)
        hit = table.get(key)
        if hit:
            ctx.set_bp_config(tuple(hit["config"]))
            return {"config": tuple(hit["config"]), "times_ms": hit.get("times_ms", {}), "cached": True}
    times, keys = {}, {}
    for cfg in ctx.bp_configs():
        ctx.set_bp_config(cfg)
        ctx.backproject(filtered, volume_native, row_scales=row_scales)  # warm-up
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(reps):
            ctx.backproject(filtered, volume_native, row_scales=row_scales)
        t1.record()
        torch.cuda.synchronize()
        ctx.check_device_status()
        times[config_name(cfg.key())] = t0.elapsed_time(t1) / reps
        keys[config_name(cfg.key())] = cfg.key()
    if not times:
        raise RuntimeError("no backprojection configuration fits this geometry")
    choice = keys[min(times, key=times.get)]
    ctx.set_bp_config(choice)
    if use_cache:
        table = _load(path)
        table[key] = {"config": list(choice), "times_ms": times}
        _store(path, table)
    return {"config": choice, "times_ms": times, "cached": False}


def batch_signature(batch):
    parts = ["v2-batch"]
    for c in batch.contexts:
        parts.append(signature(c))
    return "||".join(parts)


def tune_batch(batch, raws, volumes, reps=1, use_cache=True, path=None, candidates=None):
    """Times the whole batch (graph replay) with each backprojection
    configuration that fits every scan (or, given `candidates`, each of those
    configuration names that fits) and keeps the fastest."""
    import torch

    path = path or cache_path()
    key = batch_signature(batch) + ("|cand:" + ",".join(sorted(candidates)) if candidates else "")
    if use_cache:
        hit = _load(path).get(key)
        if hit:
            batch.set_bp_config(tuple(hit["config"]))
            return {"config": tuple(hit["config"]), "times_ms": hit.get("times_ms", {}), "cached": True}
    times, keys = {}, {}
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        cfgs = batch.bp_configs()
        if candidates:
            picked = [c for c in cfgs if config_name(c.key()) in candidates]
            cfgs = picked or cfgs
        for cfg in cfgs:
            batch.set_bp_config(cfg)
            batch.run(raws, volumes)  # capture + first replay
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(reps):
                batch.run(raws, volumes)
            t1.record(stream)
            stream.synchronize()
            batch.check_device_status()
            times[config_name(cfg.key())] = t0.elapsed_time(t1) / reps
            keys[config_name(cfg.key())] = cfg.key()
    choice = keys[min(times, key=times.get)]
    batch.set_bp_config(choice)
    if use_cache:
        table = _load(path)
        table[key] = {"config": list(choice), "times_ms": times}
        _store(path, table)
    return {"config": choice, "times_ms": times, "cached": False}
