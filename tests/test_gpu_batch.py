"""Batched reconstruction of uneven scans (wfbp_batch): one persistent
backprojection launch over all scans, the chain captured into a CUDA graph.

Every scan of the batch must come out exactly as its own wfbp_run (same
kernels, the per-voxel sums in the same order), on the first call (graph
capture) and on replays, after a change of the output pointers (recapture)
and of the launch configuration; and each scan is judged against the FP64
oracle (<= 1 HU RMS for the mixed form)."""
import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans, wfbp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda", 0)


def build(specs, precision, orc):
    ctxs, raws = [], []
    for s in specs:
        tube, table = s.views()
        cg, gp = wfbp.configure_geometry(s.meta(), table)
        ext = wfbp.make_ext(precision=precision, filter_window=s.window,
                            tex_weights=1 if precision == T.PRECISION_FP32 else 0)
        c = wfbp.Context(cg, s.recon_config(), ext, device=0)
        c.set_views(tube, table)
        ctxs.append(c)
        raws.append(torch.from_numpy(orc.synth_project(s.synth(), s.ellipsoids())).to(DEV))
    return ctxs, raws


@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
def test_batch_equals_per_scan_runs(orc, precision):
    specs = scans.batch_specs(seed=3, n=6, reduced=True)
    ctxs, raws = build(specs, precision, orc)
    refs = []
    for c, r in zip(ctxs, raws):
        v = c.alloc("volume")
        c.run(r, v)
        refs.append(v)
    torch.cuda.synchronize()
    batch = wfbp.Batch(ctxs)
    n_scans, n_items = batch.size()
    assert n_scans == 6 and n_items > 6
    vols = [c.alloc("volume") for c in ctxs]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        for it in range(3):  # capture, then two replays
            for v in vols:
                v.fill_(-7.0)
            batch.run(raws, vols)
            stream.synchronize()
            batch.check_device_status()
            for i, (v, ref) in enumerate(zip(vols, refs)):
                assert np.array_equal(v.cpu().numpy(), ref.cpu().numpy(), equal_nan=True), (it, i)
    # new output pointers: recaptured; another launch configuration: same volumes
    vols2 = [c.alloc("volume") for c in ctxs]
    cfgs = batch.bp_configs()
    assert len(cfgs) >= 2
    batch.set_bp_config(cfgs[-1])
    assert batch.bp_config().key() == cfgs[-1].key()
    batch.run(raws, vols2)  # legacy stream: synchronous
    batch.check_device_status()
    for v, ref in zip(vols2, refs):
        assert np.array_equal(v.cpu().numpy(), ref.cpu().numpy(), equal_nan=True)
    batch.close()


@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
def test_batch_run_host_equals_per_scan_runs(orc, precision):
    # host buffers in and out: the copies overlap the two backprojection
    # launches (the leading quarter of the readings' bytes, then the rest);
    # the volumes equal each scan's own wfbp_run, on two calls in a row
    specs = scans.batch_specs(seed=5, n=7, reduced=True)
    ctxs, raws = build(specs, precision, orc)
    refs = []
    for c, r in zip(ctxs, raws):
        v = c.alloc("volume")
        c.run(r, v)
        refs.append(v.cpu())
    batch = wfbp.Batch(ctxs)
    raws_h = [r.cpu().pin_memory() for r in raws]
    for it in range(2):
        vols_h = [torch.full(tuple(ref.shape), -7.0, dtype=torch.float32).pin_memory() for ref in refs]
        batch.run_host(raws_h, vols_h)
        for i, (v, ref) in enumerate(zip(vols_h, refs)):
            assert torch.equal(torch.nan_to_num(v, nan=123.0), torch.nan_to_num(ref, nan=123.0)), (it, i)
    # pageable host arrays: the copies are issued scan by scan, same volumes
    raws_n = [r.numpy().copy() for r in raws_h]
    vols_n = [np.full(tuple(ref.shape), -7.0, np.float32) for ref in refs]
    batch.run_host(raws_n, vols_n)
    for i, (v, ref) in enumerate(zip(vols_n, refs)):
        assert np.array_equal(v, ref.numpy(), equal_nan=True), i
    with pytest.raises(ValueError):
        batch.run_host(raws_h[:-1], vols_h)
    batch.close()


def test_batch_mixed_vs_fp64(orc):
    specs = scans.batch_specs(seed=4, n=5, reduced=True)
    ctxs, raws = build(specs, T.PRECISION_MIXED, orc)
    batch = wfbp.Batch(ctxs)
    vols = [c.alloc("volume") for c in ctxs]
    batch.run(raws, vols)
    batch.check_device_status()
    for s, r, v in zip(specs, raws, vols):
        ref = orc.reconstruct_f64(s, r.cpu().numpy())["volume"]
        got = v.cpu().numpy()
        rms, mx, n = orc.hu_error(got, ref)
        assert n == np.isfinite(ref).sum() and n > 0
        assert rms <= 1.0, (s.name, rms, mx)


def test_batch_rejects_mixed_forms(orc):
    specs = scans.batch_specs(seed=5, n=2, reduced=True)
    a, _ = build(specs[:1], T.PRECISION_FP32, orc)
    b, _ = build(specs[1:], T.PRECISION_MIXED, orc)
    with pytest.raises(wfbp.WfbpError) as e:
        wfbp.Batch(a + b)
    assert e.value.status == 1
    tube, table = specs[0].views()
    cg, gp = wfbp.configure_geometry(specs[0].meta(), table)
    c = wfbp.Context(cg, specs[0].recon_config(), device=0)  # views not set
    with pytest.raises(wfbp.WfbpError) as e:
        wfbp.Batch([c])
    assert e.value.status == 6
