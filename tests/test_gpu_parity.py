"""GPU parity: every stage of the sm_100a path, called through the C ABI,
against the oracle on the same seeded inputs.

Tolerances: stages are compared elementwise relative to the data's scale
(FP32 arithmetic in a different order); volumes in HU (1 HU = 1.9e-5 /mm):
the FP32 form must stay within 0.5 HU RMS / 2 HU max of the reference
transcript (the parity gate of the FP32 form against the reference's
algorithm).
"""
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
    ctx = wfbp.Context(cg, spec.recon_config(), wfbp.make_ext(filter_window=spec.window, **ext), device=0)
    ctx.set_views(tube, table)
    return ctx, cg, gp


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(DEV)


@pytest.fixture(scope="module")
def tiny(orc):
    spec = scans.tiny()
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    return spec, raw


@pytest.mark.parametrize("q8", [0, 1])
def test_rebin_matches_oracle(orc, tiny, q8):
    spec, raw = tiny
    ctx, cg, _ = make_ctx(spec, tex_weights=q8)
    out = ctx.alloc("rebinned")
    ctx.rebin(dev(raw), out)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(spec.V, spec.nr, spec.nch)
    ref = orc.rebin_ref32(cg, raw, q8=bool(q8))
    scale = np.abs(ref).max()
    d = np.abs(got - ref)
    # identical formula; contraction / asinf ulps can move a texel fraction,
    # which with 8-bit weights is a full 1/256 step
    assert np.mean(d < 1e-5 * scale) > (0.99 if q8 else 0.999)
    assert d.max() < (1.0 / 128 if q8 else 1e-3) * scale
    ref64 = orc.rebin_f64(cg, raw)
    if not q8:
        assert np.abs(got - ref64).max() < 1e-3 * scale


def test_filter_matches_oracle(orc, tiny):
    spec, raw = tiny
    ctx, cg, _ = make_ctx(spec)
    reb = orc.rebin_ref32(cg, raw)
    out = ctx.alloc("filtered")
    ctx.filter(dev(reb), out)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(reb.shape)
    half = wfbp.filter_taps(cg).astype(np.float64)
    ref = orc.filter_f64(reb, half)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() < 2e-5 * scale


def test_backproject_matches_oracle(orc, tiny):
    spec, raw = tiny
    ctx, cg, gp = make_ctx(spec)
    tube, table = spec.views()
    filt = orc.rebin_filter_ref32(cg, raw, orc.taps_ref_fft(cg))
    nat, _ = ctx.slices()
    vn = ctx.alloc("native")
    cnt = torch.zeros(1, dtype=torch.int64, device=DEV)
    ctx.backproject(dev(filt), vn, update_count=cnt)
    torch.cuda.synchronize()
    got = vn.cpu().numpy()
    ref = orc.backproject_ref32(cg, ctx.rp, gp, filt, tube, table, nat)
    rms, mx, n = orc.hu_error(got, ref)
    assert n == got.size
    assert rms < 0.05 and mx < 0.5
    v64, n64 = orc.backproject_f64(cg, ctx.rp, filt.astype(np.float64), tube.astype(np.float64),
                                   table.astype(np.float64), nat)
    assert abs(int(cnt.item()) - n64) <= 1e-4 * n64


def test_thicken_matches_oracle(orc, tiny):
    spec, _ = tiny
    ctx, cg, gp = make_ctx(spec)
    nat, req = ctx.slices()
    rng = np.random.default_rng(3)
    vn = rng.standard_normal((nat.size, spec.ny, spec.nx)).astype(np.float32)
    out = ctx.alloc("volume")
    ctx.thicken(dev(vn), out)
    torch.cuda.synchronize()
    ref = orc.thicken_ref32(ctx.rp, vn, nat, req)
    assert np.allclose(out.cpu().numpy(), ref, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("q8", [1, 0])
def test_full_path_vs_reference_transcript(orc, tiny, q8):
    spec, raw = tiny
    ctx, cg, gp = make_ctx(spec, tex_weights=q8)
    vol = ctx.alloc("volume")
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    got = vol.cpu().numpy()
    ref = orc.reconstruct_ref32(spec, raw, q8=bool(q8))
    rms, mx, n = orc.hu_error(got, ref["volume"])
    assert n == got.size
    assert rms <= 0.5 and mx <= 2.0
    r64 = orc.reconstruct_f64(spec, raw)
    rms64, mx64, _ = orc.hu_error(got, r64["volume"])
    assert rms64 <= (0.5 if q8 else 0.1)


def test_small_config_vs_reference_transcript(orc):
    # the small scanner (672 x 16, 1160 views/rot, 3 rotations) on a 128^2 grid
    spec = scans.small(seed=1)
    spec.nx = spec.ny = 128
    spec.n_slices = 6
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    ctx, cg, gp = make_ctx(spec, tex_weights=1)
    vol = ctx.alloc("volume")
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    got = vol.cpu().numpy()
    ref = orc.reconstruct_ref32(spec, raw, q8=True)
    rms, mx, n = orc.hu_error(got, ref["volume"])
    assert n == got.size, "NaN voxels"
    assert rms <= 0.5 and mx <= 2.0, (rms, mx)


def test_odd_sizes(orc):
    # sizes no launch divides evenly: nx=33, ny=17, V % 8 != 0, nch % 4 != 0
    spec = scans.tiny(nch=90, nr=5, P=100, rotations=2.57, nx=33, n_slices=3)
    spec.ny = 17
    assert spec.V % 8 != 0
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    ctx, cg, gp = make_ctx(spec)
    tube, table = spec.views()
    reb = ctx.alloc("rebinned")
    ctx.rebin(dev(raw), reb)
    filt = ctx.alloc("filtered")
    ctx.filter(reb, filt)
    vn = ctx.alloc("native")
    ctx.backproject(filt, vn)
    torch.cuda.synchronize()
    ref_reb = orc.rebin_ref32(cg, raw)
    scale = np.abs(ref_reb).max()
    assert np.abs(reb.cpu().numpy().reshape(ref_reb.shape) - ref_reb).max() < 1e-3 * scale
    ref_f = orc.filter_f64(ref_reb, wfbp.filter_taps(cg).astype(np.float64))
    got_f = filt.cpu().numpy().reshape(ref_f.shape)
    assert np.abs(got_f - ref_f).max() < 1e-4 * np.abs(ref_f).max()
    nat, _ = ctx.slices()
    ref_v = orc.backproject_ref32(cg, ctx.rp, gp, got_f, tube, table, nat)
    rms, mx, n = orc.hu_error(vn.cpu().numpy(), ref_v)
    assert rms < 0.05 and mx < 0.5


def test_synth_gpu_matches_cpu(orc):
    spec = scans.tiny()
    scan = spec.synth(i0=0)
    ref = orc.synth_project(scan, spec.ellipsoids())
    out = torch.empty(ref.shape, dtype=torch.float32, device=DEV)
    wfbp.synth_project(scan, spec.ellipsoids(), out)
    torch.cuda.synchronize()
    assert np.allclose(out.cpu().numpy(), ref, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
@pytest.mark.parametrize("which", ["tiny", "small"])
def test_run_host_matches_run(orc, tiny, which, precision):
    # wfbp_run_host pipelines the copies of reading chunks with the rebin,
    # filter and the backprojection of the slabs whose views are ready; the
    # volume must equal wfbp_run's bit for bit
    if which == "tiny":
        spec, raw = tiny
    else:
        spec = scans.small(seed=9)
        spec.nx = spec.ny = 64
        spec.n_slices = 40  # several 32-slice slabs
        raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    ctx, cg, gp = make_ctx(spec, tex_weights=1 if precision == T.PRECISION_FP32 else 0, precision=precision)
    assert ctx.dims.n_slices_native > 32 or which == "tiny"
    vol = ctx.alloc("volume")
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    pinned = torch.from_numpy(np.ascontiguousarray(raw)).pin_memory()
    for _ in range(2):
        host = ctx.run_host(pinned)
        assert np.array_equal(host, vol.cpu().numpy(), equal_nan=True)
    # a pinned destination: the slices thickened inside a slab are copied
    # back while later slabs run
    out = torch.full(tuple(vol.shape), -7.0, dtype=torch.float32).pin_memory()
    for _ in range(2):
        ctx.run_host(pinned, out)
        assert np.array_equal(out.numpy(), vol.cpu().numpy(), equal_nan=True)


@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
def test_run_fused_thickening_matches_stages(orc, precision):
    # wfbp_run thickens the requested slices that lie inside one slab in the
    # backprojection's write-back and the slices that straddle slabs
    # afterwards; the volume must equal the stage chain's (backproject, then
    # wfbp_thicken) bit for bit, for both slab heights
    spec = scans.small(seed=11)
    spec.nx = spec.ny = 64
    spec.n_slices = 50
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ctx = wfbp.Context(cg, spec.recon_config(), wfbp.make_ext(precision=precision, filter_window=spec.window,
                                                             filtered_layout=T.LAYOUT_BACKPROJECTION), device=0)
    ctx.set_views(tube, table)
    assert ctx.dims.n_slices_native > 64
    reb, filt, sc, vn = ctx.alloc("rebinned"), ctx.alloc("filtered"), ctx.alloc("row_scales"), ctx.alloc("native")
    staged, fused = ctx.alloc("volume"), ctx.alloc("volume")
    seen = set()
    for c in ctx.bp_configs():
        if c.slab in seen:
            continue
        seen.add(c.slab)
        ctx.set_bp_config(c)
        ctx.rebin(dev(raw), reb)
        ctx.filter(reb, filt, sc)
        ctx.backproject(filt, vn, sc)
        ctx.thicken(vn, staged)
        fused.fill_(-7.0)
        ctx.run(dev(raw), fused)
        torch.cuda.synchronize()
        ctx.check_device_status()
        a, b = staged.cpu().numpy(), fused.cpu().numpy()
        assert np.isfinite(a).any()
        assert np.array_equal(a, b, equal_nan=True), c.key()
    assert seen == {16, 32}


def test_state_and_argument_errors(tiny):
    spec, raw = tiny
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ctx = wfbp.Context(cg, spec.recon_config())
    f = ctx.alloc("filtered")
    vn = ctx.alloc("native")
    with pytest.raises(wfbp.WfbpError) as e:
        ctx.backproject(f, vn)  # views not set
    assert e.value.status == T.WFBP_OK + 6
    bad = tube.copy()
    bad[5] = np.nan
    with pytest.raises(wfbp.WfbpError) as e:
        ctx.set_views(bad, table)
    assert e.value.status == 1
    assert "reading 5" in str(e.value)


def _golden_files():
    import glob
    import os
    return sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_*.npz")))


@pytest.mark.parametrize("path", _golden_files(), ids=lambda p: p.rsplit("/", 1)[-1])
def test_fp32_form_vs_reference_kernels(orc, path):
    # The parity gate against the reference's own fct_wfbp kernels (run on a
    # B200 via the shim): the FP32 form within 0.5 HU RMS / 2 HU max.
    from tests.golden.make_reference_fixtures import cases
    name = path.rsplit("/", 1)[-1][4:-4]
    spec = dict(cases())[name]
    d = np.load(path)
    ctx, cg, gp = make_ctx(spec, tex_weights=1)
    vol = ctx.alloc("volume")
    ctx.run(dev(d["raw"]), vol)
    torch.cuda.synchronize()
    got = vol.cpu().numpy()
    rms, mx, n = orc.hu_error(got, d["volume"])
    assert np.array_equal(np.isnan(got), np.isnan(d["volume"]))
    assert n == np.isfinite(d["volume"]).sum()
    assert rms <= 0.5 and mx <= 2.0, (rms, mx)


@pytest.mark.parametrize("which", ["tiny", "odd", "small128", "lowpitch"])
def test_backprojection_layout_stages(orc, which):
    # FP32 form through the stage API with the backprojection layout: the
    # transposed filter output equals the reference-layout one, and the
    # TMA-staged backprojection equals the transcript on the same rows.
    # "lowpitch": a table feed (4 mm per rotation) below the detector cone's
    # height, so the table-position cull (cuda_kernels.cuh:232) removes
    # samples the rows would admit and the records carry its row range.
    if which == "tiny":
        spec = scans.tiny()
    elif which == "lowpitch":
        spec = scans.tiny()
        spec.feed = 4.0
    elif which == "odd":
        spec = scans.tiny(nch=90, nr=5, P=100, rotations=2.57, nx=33, n_slices=3)
        spec.ny = 17
    else:
        spec = scans.small(seed=5)
        spec.nx = spec.ny = 128
        spec.n_slices = 6
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ctx = wfbp.Context(cg, spec.recon_config(), wfbp.make_ext(filter_window=spec.window, tex_weights=1,
                                                             filtered_layout=T.LAYOUT_BACKPROJECTION), device=0)
    ctx.set_views(tube, table)
    reb = ctx.alloc("rebinned")
    ctx.rebin(dev(raw), reb)
    filt = ctx.alloc("filtered")
    ctx.filter(reb, filt)
    vn = ctx.alloc("native")
    cnt = torch.zeros(1, dtype=torch.int64, device=DEV)
    ctx.backproject(filt, vn, update_count=cnt)
    torch.cuda.synchronize()
    ctx.check_device_status()
    nrp = (spec.nr + 3) // 4 * 4
    ft = filt.cpu().numpy().reshape(spec.V, spec.nch, nrp)[:, :, :spec.nr].transpose(0, 2, 1)
    ref_reb = orc.rebin_ref32(cg, raw, q8=True)
    ref_f = orc.filter_f64(ref_reb, wfbp.filter_taps(cg, spec.window).astype(np.float64))
    # 8-bit weights: a last-ulp difference can move a weight by 1/256
    assert np.abs(ft - ref_f).max() < 5e-3 * np.abs(ref_f).max()
    nat, _ = ctx.slices()
    ref_v = orc.backproject_ref32(cg, ctx.rp, gp, np.ascontiguousarray(ft), tube, table, nat)
    got = vn.cpu().numpy()
    rms, mx, n = orc.hu_error(got, ref_v)
    assert np.array_equal(np.isnan(got), np.isnan(ref_v))
    # the z cull |z - z_j| <= z_rot is evaluated in row space (q range per
    # column and view): a slice exactly on the boundary can fall the other
    # way, which moves that voxel by a fraction of a HU
    assert rms < 0.05 and mx < 1.0, (rms, mx)
    _, n64 = orc.backproject_f64(cg, ctx.rp, ft.astype(np.float64), tube.astype(np.float64),
                                 table.astype(np.float64), nat)
    assert abs(int(cnt.item()) - n64) <= 1e-4 * n64 + 2


@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
def test_bp_configs_identical_and_tuner(orc, tmp_path, precision):
    # every launch configuration computes the same per-voxel sums in the same
    # order, so the volumes are bit-identical; the autotuner picks one of them
    from freect_b200 import autotune
    spec = scans.small(seed=7)
    spec.nx = spec.ny = 96
    spec.n_slices = 40
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ctx = wfbp.Context(cg, spec.recon_config(), wfbp.make_ext(precision=precision, filter_window=spec.window,
                                                             filtered_layout=T.LAYOUT_BACKPROJECTION), device=0)
    ctx.set_views(tube, table)
    reb, filt, sc = ctx.alloc("rebinned"), ctx.alloc("filtered"), ctx.alloc("row_scales")
    ctx.rebin(dev(raw), reb)
    ctx.filter(reb, filt, sc)
    cfgs = ctx.bp_configs()
    assert len(cfgs) >= 4
    vols = []
    for c in cfgs:
        ctx.set_bp_config(c)
        assert ctx.bp_config().key() == c.key()
        vn = ctx.alloc("native")
        ctx.backproject(filt, vn, sc)
        torch.cuda.synchronize()
        ctx.check_device_status()
        vols.append(vn.cpu().numpy())
    assert np.isfinite(vols[0]).any()
    for c, v in zip(cfgs[1:], vols[1:]):
        assert np.array_equal(v, vols[0], equal_nan=True), c.key()
    assert {c.slab for c in cfgs} == {16, 32}
    with pytest.raises(wfbp.WfbpError):
        ctx.set_bp_config((16, 16, 16))
    # ext.bp_slab admits only the configurations with that slab height
    c16 = wfbp.Context(cg, spec.recon_config(), wfbp.make_ext(precision=precision, filter_window=spec.window,
                                                             filtered_layout=T.LAYOUT_BACKPROJECTION, bp_slab=16),
                       device=0)
    c16.set_views(tube, table)
    assert c16.bp_config().slab == 16 and {c.slab for c in c16.bp_configs()} == {16}
    with pytest.raises(wfbp.WfbpError):
        c16.set_bp_config((16, 16, 4, 16, 32))
    with pytest.raises(wfbp.WfbpError):
        wfbp.Context(cg, spec.recon_config(), wfbp.make_ext(bp_slab=8), device=0)
    path = str(tmp_path / "tune.json")
    vn = ctx.alloc("native")
    r1 = autotune.tune_backprojection(ctx, filt, vn, row_scales=sc, path=path)
    assert not r1["cached"] and r1["config"] in [c.key() for c in cfgs]
    assert len(r1["times_ms"]) == len(cfgs)
    r2 = autotune.tune_backprojection(ctx, filt, vn, row_scales=sc, path=path)
    assert r2["cached"] and r2["config"] == r1["config"] and ctx.bp_config().key() == r1["config"]


def test_run_timed_matches_run(orc, tiny):
    spec, raw = tiny
    ctx, cg, gp = make_ctx(spec, tex_weights=1)
    a, b = ctx.alloc("volume"), ctx.alloc("volume")
    ctx.run(dev(raw), a)
    ms = ctx.run_timed(dev(raw), b)
    torch.cuda.synchronize()
    assert set(ms) == {"rebin", "filter", "backproject", "thicken"} and all(v > 0 for v in ms.values())
    assert np.array_equal(a.cpu().numpy(), b.cpu().numpy(), equal_nan=True)


@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
def test_descending_slices_and_origin_offset(orc, precision):
    # start_pos > end_pos (slice lists run downwards, ReconstructionMachine.cu:116-132)
    # and a reconstruction grid centred off the isocentre (x_origin, y_origin)
    spec = scans.tiny(nch=96, nr=8, P=96, rotations=3, nx=32, n_slices=4)
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    rp.start_pos, rp.end_pos = rp.end_pos - 0.5 * rp.slice_pitch, rp.start_pos - 0.5 * rp.slice_pitch
    rp.x_origin, rp.y_origin = 7.5, -4.25
    ext = wfbp.make_ext(precision=precision, filter_window=spec.window,
                        tex_weights=1 if precision == T.PRECISION_FP32 else 0)
    ctx = wfbp.Context(cg, rp, ext, device=0)
    ctx.set_views(tube, table)
    nat, req = ctx.slices()
    assert nat[1] < nat[0] and req[1] < req[0]
    vol = ctx.alloc("volume")
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    ctx.check_device_status()
    got = vol.cpu().numpy()
    # the same reconstruction through the FP64 oracle's stages with these slice lists
    zn, zr = orc.slice_locations(cg, rp)
    assert np.array_equal(zn, nat) and np.array_equal(zr, req)
    x = orc.rebin_f64(cg, raw)
    y = orc.filter_f64(x, orc.taps_f64(cg, spec.window))
    vn, _ = orc.backproject_f64(cg, rp, y, tube.astype(np.float64), table.astype(np.float64), zn)
    ref = orc.thicken_f64(rp, vn, zn, zr)
    rms, mx, n = orc.hu_error(got, ref)
    assert n == np.isfinite(ref).sum() and n > 0
    assert rms <= (0.5 if precision == T.PRECISION_FP32 else 1.0), (rms, mx)


@pytest.mark.parametrize("rk", [T.RECON_KERNEL_SHEPP_LOGAN, T.RECON_KERNEL_HANN, T.RECON_KERNEL_HAMMING])
def test_recon_kernel_from_yaml(orc, tmp_path, rk):
    # a recon YAML with recon_kernel set, read by wfbp_parse_recon_config; the
    # context (no filter in the extension) filters with that window, checked
    # against the reference transcript given the same window's taps
    spec = scans.tiny(seed=21)
    ref_rp = spec.recon_config()
    p = tmp_path / "recon.yaml"
    p.write_text("raw_data_dir: synthetic\noutput_dir: .\nstart_pos: %r\nend_pos: %r\nrecon_fov: %r\n"
                 "slice_thickness: %r\nslice_pitch: %r\nnx: %d\nny: %d\nrecon_kernel: %d\n"
                 % (ref_rp.start_pos, ref_rp.end_pos, ref_rp.recon_fov, ref_rp.slice_thickness, ref_rp.slice_pitch,
                    ref_rp.nx, ref_rp.ny, rk))
    rp = wfbp.parse_recon_config(str(p))
    assert rp.recon_kernel == rk
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ctx = wfbp.Context(cg, rp, wfbp.make_ext(tex_weights=1), device=0)
    ctx.set_views(tube, table)
    vol = ctx.alloc("volume")
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    w, c, a = wfbp.recon_kernel_filter(rk)
    half = wfbp.filter_taps(cg, w, c, a)
    ref = orc.reconstruct_ref32(spec, raw, taps_half=half, q8=True)
    got = vol.cpu().numpy()
    rms, mx, n = orc.hu_error(got, ref["volume"])
    assert n == got.size
    assert rms <= 0.5 and mx <= 2.0, (rms, mx)
    # and it differs from the Ram-Lak reconstruction (the window took effect)
    ramlak = orc.reconstruct_ref32(spec, raw, q8=True)
    assert orc.hu_error(got, ramlak["volume"])[0] > 5.0 * max(rms, 0.01)
    ctx.close()


def test_adaptive_filtration(orc):
    # ReconConfig.adaptive_filtration_s > 0: the raw readings are smoothed
    # (attenuation-adaptive, k_adaptive_filter) before the rebin. FP32 form
    # against the reference transcript fed with the oracle's filtered readings;
    # mixed form against the FP64 oracle on the same; the pipelined host path
    # (filtration chunk by chunk as the readings arrive) equals wfbp_run; the
    # adjoints refuse it
    spec = scans.tiny(seed=23)
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    s = 0.35
    raw_af = orc.adaptive_filter_f64(raw, s).astype(np.float32)
    assert not np.array_equal(raw_af, raw)
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    rp.adaptive_filtration_s = s
    ctx = wfbp.Context(cg, rp, wfbp.make_ext(tex_weights=1), device=0)
    ctx.set_views(tube, table)
    vol = ctx.alloc("volume")
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    got = vol.cpu().numpy()
    ref = orc.reconstruct_ref32(spec, raw_af, q8=True)
    rms, mx, n = orc.hu_error(got, ref["volume"])
    assert n == got.size and rms <= 0.5 and mx <= 2.0, (rms, mx)
    plain = orc.reconstruct_ref32(spec, raw, q8=True)
    assert orc.hu_error(got, plain["volume"])[0] > 5.0 * max(rms, 0.01)  # the filtration took effect
    vh = np.zeros_like(got)
    ctx.run_host(raw, vh)
    assert np.array_equal(vh, got)
    g = ctx.alloc("rebinned")
    with pytest.raises(wfbp.WfbpError):
        ctx.rebin_adjoint(g, ctx.alloc("raw"))
    ctx.close()
    ctx = wfbp.Context(cg, rp, wfbp.make_ext(precision=T.PRECISION_MIXED), device=0)
    ctx.set_views(tube, table)
    vol = ctx.alloc("volume")
    ctx.run(dev(raw), vol)
    torch.cuda.synchronize()
    r64 = orc.reconstruct_f64(spec, raw_af)
    rms, mx, n = orc.hu_error(vol.cpu().numpy(), r64["volume"])
    assert n == np.isfinite(r64["volume"]).sum() and rms <= 1.0, (rms, mx)
    ctx.close()
