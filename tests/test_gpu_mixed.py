"""Mixed-precision form on the GPU: rebin with FP64 sample coordinates,
split-FP16 (hi + lo) tcgen05 Toeplitz filter with FP32 accumulation, FP16
filtered rows with power-of-two scales, backprojection with FP64 per-view
geometry and FP32 accumulation. Judged against the FP64 oracle: <= 1 HU RMSE."""
import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans, wfbp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda", 0)


def make_ctx(spec, **ext):
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    e = wfbp.make_ext(precision=T.PRECISION_MIXED, filter_window=spec.window, **ext)
    ctx = wfbp.Context(cg, spec.recon_config(), e, device=0)
    ctx.set_views(tube, table)
    return ctx, cg, gp


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(DEV)


@pytest.mark.parametrize("shape", [(96, 8, 96, 3.0), (90, 5, 100, 2.57), (672, 16, 1160, 2.1)])
def test_tc_filter_matches_fp64(orc, shape):
    nch, nr, P, rot = shape
    spec = scans.tiny(nch=nch, nr=nr, P=P, rotations=rot)
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    ctx, cg, gp = make_ctx(spec)
    reb = ctx.alloc("rebinned")
    filt = ctx.alloc("filtered")
    sc = ctx.alloc("row_scales")
    ctx.rebin(dev(raw), reb)
    ctx.filter(reb, filt, sc)
    torch.cuda.synchronize()
    ctx.check_device_status()
    got = filt.float().cpu().numpy() * sc.cpu().numpy()[: spec.V * spec.nr].reshape(spec.V, spec.nr, 1)
    x = orc.rebin_f64(cg, raw)  # exact weights and FP64 coordinates, like the mixed rebin
    taps = wfbp.filter_taps(cg).astype(np.float64)
    ref = orc.filter_f64(x, taps)
    err = np.abs(got - ref)
    # FP16 storage: round to nearest, <= 2^-11 relative to each value (half
    # an ulp); the split FP16 operands (22 bits each), the dropped Xlo*Tlo
    # term and FP32 accumulation: ~2^-20 of sum|h| max|x| (bound with a 4x
    # margin)
    l1 = taps[0] + 2 * np.abs(taps[1:]).sum()
    bound = 2.0 ** -11 * np.abs(ref) + 2.0 ** -18 * l1 * np.abs(x).max(axis=-1, keepdims=True)
    assert np.all(err <= bound), (err / bound).max()
    s = sc.cpu().numpy()[: spec.V * spec.nr]
    assert np.all(s > 0) and np.all(np.log2(s) == np.round(np.log2(s)))  # powers of two


@pytest.mark.parametrize("which", ["tiny", "small128"])
def test_mixed_vs_fp64_oracle(orc, which):
    if which == "tiny":
        spec = scans.tiny()
    else:
        spec = scans.small(seed=2)
        spec.nx = spec.ny = 128
        spec.n_slices = 4
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    ctx, cg, gp = make_ctx(spec)
    vol = ctx.alloc("volume")
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    ctx.check_device_status()
    got = vol.cpu().numpy()
    r64 = orc.reconstruct_f64(spec, raw)
    rms, mx, n = orc.hu_error(got, r64["volume"])
    assert n == got.size
    assert rms <= 1.0, (rms, mx)


def test_mixed_shepp_logan_window(orc):
    spec = scans.tiny(window=T.FILTER_SHEPP_LOGAN)
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    ctx, cg, gp = make_ctx(spec)
    vol = ctx.alloc("volume")
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    r64 = orc.reconstruct_f64(spec, raw)
    rms, mx, n = orc.hu_error(vol.cpu().numpy(), r64["volume"])
    assert n == vol.numel() and rms <= 1.0


def test_mixed_requires_row_scales(orc):
    spec = scans.tiny()
    ctx, cg, gp = make_ctx(spec)
    reb = ctx.alloc("rebinned")
    filt = ctx.alloc("filtered")
    with pytest.raises(wfbp.WfbpError) as e:
        ctx.filter(reb, filt, None)
    assert e.value.status == 1


@pytest.mark.parametrize("which", ["tiny", "odd", "lowpitch"])
def test_mixed_backprojection_layout_stages(orc, which):
    # split-FP16 filter writing FP16 row pairs with one scale per scan, read by
    # the TMA-staged backprojection; against the FP64 oracle ("lowpitch": the
    # table-position cull binds, 4 mm table feed per rotation)
    if which == "tiny":
        spec = scans.tiny()
    elif which == "lowpitch":
        spec = scans.tiny()
        spec.feed = 4.0
    else:
        spec = scans.tiny(nch=90, nr=5, P=100, rotations=2.57, nx=33, n_slices=3)
        spec.ny = 17
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    e = wfbp.make_ext(precision=T.PRECISION_MIXED, filter_window=spec.window, filtered_layout=T.LAYOUT_BACKPROJECTION)
    ctx = wfbp.Context(cg, spec.recon_config(), e, device=0)
    ctx.set_views(tube, table)
    reb, filt, sc, vn, vol = (ctx.alloc(k) for k in ("rebinned", "filtered", "row_scales", "native", "volume"))
    ctx.rebin(dev(raw), reb)
    ctx.filter(reb, filt, sc)
    ctx.backproject(filt, vn, sc)
    ctx.thicken(vn, vol)
    torch.cuda.synchronize()
    ctx.check_device_status()
    # one power of two for the whole scan, the smallest >= the taps' L1 norm
    s = sc.cpu().numpy()[: spec.V]
    taps = wfbp.filter_taps(cg).astype(np.float64)
    l1 = abs(taps[0]) + 2 * np.abs(taps[1:]).sum()
    assert np.all(s == s[0]) and s[0] >= l1 and s[0] / 2 < l1
    assert np.log2(s[0]) == np.round(np.log2(s[0]))
    r64 = orc.reconstruct_f64(spec, raw)
    got = vol.cpu().numpy()
    rms, mx, n = orc.hu_error(got, r64["volume"])
    assert n == np.isfinite(r64["volume"]).sum()
    assert rms <= 1.0, (rms, mx)


def test_mixed_pairs_range_is_reported(orc):
    # rebinned samples far above 16384 overflow the FP16 row pairs: the filter
    # records it and check_device_status reports it; the context stays usable
    spec = scans.tiny()
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    ctx, cg, gp = make_ctx(spec, filtered_layout=T.LAYOUT_BACKPROJECTION)
    vol = ctx.alloc("volume")
    ctx.run(dev(raw * 1.0e7), vol)
    torch.cuda.synchronize()
    with pytest.raises(wfbp.WfbpError) as e:
        ctx.check_device_status()
    assert e.value.status == 5 and "FP16" in str(e.value)  # WFBP_ERR_UNSUPPORTED
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    ctx.check_device_status()
    r64 = orc.reconstruct_f64(spec, raw)
    rms, mx, n = orc.hu_error(vol.cpu().numpy(), r64["volume"])
    assert rms <= 1.0, (rms, mx)
