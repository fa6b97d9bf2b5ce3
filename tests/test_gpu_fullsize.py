"""Parity at the benchmark configurations' own sizes.

* small scanner (672 ch x 16 rows x 3480 readings -> 256^2 x 16 slices,
  Ram-Lak): the FP32 form against the reference's OWN kernels
  (cuda_kernels.cuh run on a B200 through oracle/ref_shim; the committed
  fixture holds the seed, the SHA-256 of the raw frames and the reference's
  volume), gate 0.5 HU RMS / 2 HU max; both forms against the FP64 oracle.
* rows64 (888 x 64 x 9840 -> 512^2 x 300), the flying-focal-spot scan
  (736 x 32 PhiZ, 18432 readings -> 512^2 x 200) and the 24-scan uneven batch
  (mixed form, one persistent launch): against the FP64 oracle on the slab of
  the middle requested slice, gate 1 HU RMS (the mixed form's bar) and, for
  the FP32 form, 0.5 HU RMS.

HU = 1000 (mu - mu_water) / mu_water with mu_water = 0.019 / mm, over voxels
with full coverage (finite in both volumes).
"""
import hashlib
import os

import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans, wfbp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda", 0)
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _ctx(spec, precision, **ext):
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    e = wfbp.make_ext(precision=precision, filter_window=spec.window,
                      tex_weights=1 if precision == T.PRECISION_FP32 else 0, **ext)
    ctx = wfbp.Context(cg, spec.recon_config(), e, device=0)
    ctx.set_views(tube, table)
    return ctx, cg, tube, table


def _slab_hu(spec, cg, tube, table, raw, vol, which=None):
    from oracle.slab_check import hu_vs_fp64_slab
    return hu_vs_fp64_slab(spec, cg, spec.recon_config(), tube, table,
                           lambda a0, a1: raw[a0:a1].cpu().numpy(),
                           lambda r0, r1: vol[r0:r1].cpu().numpy(), which)


def test_small_full_fp32_vs_reference_kernels(orc):
    d = np.load(os.path.join(GOLDEN, "full_ref_small.npz"))
    spec = scans.small(seed=int(d["seed"]))
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    # the raw frames are regenerated from the seed: they must be the ones the
    # reference reconstructed
    assert hashlib.sha256(np.ascontiguousarray(raw).tobytes()).hexdigest() == str(d["raw_sha256"])
    ctx, cg, tube, table = _ctx(spec, T.PRECISION_FP32)
    assert np.array_equal(ctx.slices()[1], d["z_req"])
    raw_d = torch.from_numpy(raw).to(DEV)
    vol = ctx.alloc("volume")
    ctx.run(raw_d, vol)
    torch.cuda.synchronize()
    got = vol.cpu().numpy()
    rms, mx, n = orc.hu_error(got, d["volume"])
    assert np.array_equal(np.isnan(got), np.isnan(d["volume"]))
    assert n == np.isfinite(d["volume"]).sum() and n > 0.9 * got.size
    assert rms <= 0.5 and mx <= 2.0, (rms, mx)
    ctx.close()


@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
def test_small_full_vs_fp64(orc, precision):
    spec = scans.small(seed=3)
    raw = torch.from_numpy(orc.synth_project(spec.synth(), spec.ellipsoids())).to(DEV)
    ctx, cg, tube, table = _ctx(spec, precision)
    vol = ctx.alloc("volume")
    ctx.run(raw, vol)
    torch.cuda.synchronize()
    hu = _slab_hu(spec, cg, tube, table, raw, vol)
    assert hu["voxels"] > 0
    assert hu["rms"] <= (0.5 if precision == T.PRECISION_FP32 else 1.0), hu
    ctx.close()


@pytest.mark.parametrize("workload", ["rows64", "ffs"])
def test_full_size_vs_fp64(workload):
    spec = scans.WORKLOADS[workload](seed=0)
    raw = torch.empty((spec.V, spec.nr, spec.nch), dtype=torch.float32, device=DEV)
    wfbp.synth_project(spec.synth(), spec.ellipsoids(), raw)
    res = {}
    for precision in (T.PRECISION_MIXED, T.PRECISION_FP32):
        ctx, cg, tube, table = _ctx(spec, precision, filtered_layout=T.LAYOUT_BACKPROJECTION)
        vol = ctx.alloc("volume")
        ctx.run(raw, vol)
        torch.cuda.synchronize()
        ctx.check_device_status()
        res[precision] = _slab_hu(spec, cg, tube, table, raw, vol)
        del vol
        ctx.close()
    for precision, hu in res.items():
        assert hu["voxels"] > 0.5 * spec.nx * spec.ny, hu
        assert hu["rms"] <= (0.5 if precision == T.PRECISION_FP32 else 1.0), (workload, res)


def test_batch24_full_size_vs_fp64_per_scan():
    # the 24 uneven scans reconstructed as ONE batch (mixed form, persistent
    # backprojection launch), each scan against the FP64 oracle on its middle slab
    specs = scans.batch_specs(seed=0, n=24)
    ctxs, raws, vols, meta = [], [], [], []
    for sp in specs:
        c, cg, tube, table = _ctx(sp, T.PRECISION_MIXED)
        r = c.alloc("raw")
        wfbp.synth_project(sp.synth(), sp.ellipsoids(), r)
        ctxs.append(c)
        raws.append(r)
        vols.append(c.alloc("volume"))
        meta.append((cg, tube, table))
    batch = wfbp.Batch(ctxs)
    batch.run(raws, vols)
    torch.cuda.synchronize()
    batch.check_device_status()
    worst = []
    for sp, r, v, (cg, tube, table) in zip(specs, raws, vols, meta):
        hu = _slab_hu(sp, cg, tube, table, r, v)
        assert hu["voxels"] > 0, sp.name
        worst.append(hu["rms"])
    assert max(worst) <= 1.0, worst
    batch.close()
    for c in ctxs:
        c.close()
