"""Adjoint kernels and the autograd wrapper on the GPU.

Each adjoint is checked twice: against its own GPU forward by the
dot-product identity <F x, y> = <x, F^T y> (which any transpose satisfies),
and elementwise against the FP64 oracle's adjoint of the same stage. The
differentiable reconstruction (a batch of scans of the small scanner, MSE to
the voxelised phantom) is checked against the FP64 oracle's gradient with
respect to the raw readings and the 64 learnable filter taps; the oracle's
gradient itself is pinned by central finite differences in
test_adjoint_oracle.py (exact there, the loss being quadratic).
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


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(DEV)


def make(spec, tex_weights=0, adjoint_scale_table=0):
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ext = wfbp.make_ext(filter_window=spec.window, tex_weights=tex_weights, adjoint_scale_table=adjoint_scale_table)
    ctx = wfbp.Context(cg, spec.recon_config(), ext, device=0)
    ctx.set_views(tube, table)
    return ctx, cg, tube, table


def dot_ok(a, b, na, nb, tol=2e-5):
    # |<Fx, y> - <x, F^T y>| against the Cauchy-Schwarz scale of the products
    assert abs(a - b) <= tol * na * nb, (a, b, na * nb)


@pytest.fixture(scope="module")
def tiny():
    return scans.tiny(nch=96, nr=8, P=96, rotations=3, nx=32, n_slices=4)


@pytest.mark.parametrize("q8", [0, 1])
def test_rebin_adjoint(orc, tiny, q8):
    ctx, cg, _, _ = make(tiny, tex_weights=q8)
    d = ctx.dims
    rng = np.random.default_rng(1)
    x = rng.standard_normal((d.n_readings, d.raw_rows, d.raw_channels)).astype(np.float32)
    y = rng.standard_normal((d.n_views, d.n_rows, d.n_channels)).astype(np.float32)
    fx = ctx.alloc("rebinned")
    ctx.rebin(dev(x), fx)
    gx = torch.empty(x.shape, dtype=torch.float32, device=DEV)
    ctx.rebin_adjoint(dev(y), gx)
    torch.cuda.synchronize()
    ctx.check_device_status()
    fx, gx = fx.cpu().numpy().reshape(y.shape).astype(np.float64), gx.cpu().numpy().astype(np.float64)
    dot_ok(np.vdot(fx, y), np.vdot(x, gx), np.linalg.norm(x), np.linalg.norm(gx))
    if not q8:
        ref = orc.rebin_adjoint_f64(cg, y)
        assert np.abs(gx - ref).max() < 1e-4 * np.abs(ref).max()


def test_filter_adjoint(tiny):
    ctx, cg, _, _ = make(tiny)
    d = ctx.dims
    rng = np.random.default_rng(2)
    shape = (d.n_views, d.n_rows, d.n_channels)
    x = rng.standard_normal(shape).astype(np.float32)
    y = rng.standard_normal(shape).astype(np.float32)
    fx, gy = ctx.alloc("filtered"), torch.empty(shape, dtype=torch.float32, device=DEV)
    ctx.filter(dev(x), fx)
    ctx.filter_adjoint(dev(y), gy)
    torch.cuda.synchronize()
    fx, gy = fx.cpu().numpy().astype(np.float64), gy.cpu().numpy().astype(np.float64)
    dot_ok(np.vdot(fx, y), np.vdot(x, gy), np.linalg.norm(fx), np.linalg.norm(y))


@pytest.mark.parametrize("table_mode", [0, -1])  # with the scale table, and recomputing the weight sums
@pytest.mark.parametrize("which", ["tiny", "odd"])
def test_backproject_adjoint(orc, tiny, which, table_mode):
    spec = tiny
    if which == "odd":
        spec = scans.tiny(nch=90, nr=5, P=100, rotations=2.57, nx=33, n_slices=3)
        spec.ny = 17
    ctx, cg, tube, table = make(spec, adjoint_scale_table=table_mode)
    d = ctx.dims
    rng = np.random.default_rng(3)
    f = rng.standard_normal((d.n_views, d.n_rows, d.n_channels)).astype(np.float32)
    vn = ctx.alloc("native")
    ctx.backproject(dev(f), vn)
    torch.cuda.synchronize()
    vn = vn.cpu().numpy().astype(np.float64)
    fin = np.isfinite(vn)
    assert fin.mean() > 0.3
    y = rng.standard_normal(vn.shape)
    y[~fin] = 0.0
    gf = torch.empty(f.shape, dtype=torch.float32, device=DEV)
    ctx.backproject_adjoint(dev(y), gf)
    torch.cuda.synchronize()
    gf = gf.cpu().numpy().astype(np.float64)
    dot_ok(np.vdot(vn[fin], y[fin]), np.vdot(f, gf), np.linalg.norm(vn[fin]), np.linalg.norm(y))
    nat, _ = ctx.slices()
    ref = orc.backproject_adjoint_f64(cg, ctx.rp, y, tube.astype(np.float64), table.astype(np.float64), nat)
    err = np.abs(gf - ref)
    # FP32 geometry: a sample on a bounds / cull boundary can fall the other way
    assert np.mean(err < 1e-4 * np.abs(ref).max()) > 0.999
    assert np.linalg.norm(gf - ref) < 1e-3 * np.linalg.norm(ref)


def test_backproject_adjoint_table_reuse(tiny):
    # the weight table depends on the geometry alone: one context computes it
    # once and reuses it for every gradient, and again after its views or
    # slices change; each result must match a context that recomputes the
    # weight sums
    ctx_t, cg, tube, table = make(tiny, adjoint_scale_table=0)
    ctx_r, _, _, _ = make(tiny, adjoint_scale_table=-1)
    d = ctx_t.dims
    rng = np.random.default_rng(6)

    def check():
        y = dev(rng.standard_normal((d.n_slices_native, d.ny, d.nx)))
        a = torch.empty((d.n_views, d.n_rows, d.n_channels), dtype=torch.float32, device=DEV)
        b = torch.empty_like(a)
        ctx_t.backproject_adjoint(y, a)
        ctx_r.backproject_adjoint(y, b)
        torch.cuda.synchronize()
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(a).max() > 0
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()

    check()
    check()
    table2 = (table + 0.37).astype(np.float32)  # views moved by a fraction of a slice
    ctx_t.set_views(tube, table2)
    ctx_r.set_views(tube, table2)
    check()
    nat, req = ctx_t.slices()
    for c in (ctx_t, ctx_r):
        c.set_slices(nat + 0.21, req + 0.21)
    check()
    with pytest.raises(wfbp.WfbpError):
        wfbp.Context(cg, tiny.recon_config(), wfbp.make_ext(adjoint_scale_table=2), device=0)


def test_thicken_adjoint(orc, tiny):
    ctx, cg, _, _ = make(tiny)
    d = ctx.dims
    rng = np.random.default_rng(4)
    v = rng.standard_normal((d.n_slices_native, d.ny, d.nx)).astype(np.float32)
    y = rng.standard_normal((d.n_slices_requested, d.ny, d.nx)).astype(np.float32)
    tv, gv = ctx.alloc("volume"), ctx.alloc("native")
    ctx.thicken(dev(v), tv)
    ctx.thicken_adjoint(dev(y), gv)
    torch.cuda.synchronize()
    tv, gv = tv.cpu().numpy().astype(np.float64), gv.cpu().numpy().astype(np.float64)
    dot_ok(np.vdot(tv, y), np.vdot(v, gv), np.linalg.norm(tv), np.linalg.norm(y))
    nat, req = ctx.slices()
    ref = orc.thicken_adjoint_f64(ctx.rp, y, nat, req)
    assert np.allclose(gv, ref, rtol=1e-5, atol=1e-6)


def test_taps_gradient(orc, tiny):
    ctx, cg, _, _ = make(tiny)
    d = ctx.dims
    rng = np.random.default_rng(5)
    raw = rng.standard_normal((d.n_readings, d.raw_rows, d.raw_channels)).astype(np.float32)
    g = rng.standard_normal((d.n_views, d.n_rows, d.n_channels)).astype(np.float32)
    n = 16
    gt = torch.empty(n, dtype=torch.float32, device=DEV)
    ctx.taps_gradient(dev(raw), dev(g), gt)
    reb = ctx.alloc("rebinned")
    ctx.rebin(dev(raw), reb)
    torch.cuda.synchronize()
    x = reb.cpu().numpy().reshape(g.shape).astype(np.float64)
    gt = gt.cpu().numpy().astype(np.float64)
    ref = orc.taps_gradient_f64(g.reshape(-1, d.n_channels), x.reshape(-1, d.n_channels), n)
    assert np.allclose(gt, ref, rtol=1e-4, atol=1e-4 * np.abs(ref).max())
    # <filter_dh(x), g> = <dh, gradient>: filter with taps dh (zero beyond n)
    base = ctx.get_taps()
    dh = np.zeros(d.n_channels, np.float32)
    dh[:n] = rng.standard_normal(n)
    ctx.set_taps(dev(dh))
    fy = ctx.alloc("filtered")
    ctx.filter(reb, fy)
    ctx.set_taps(base)
    torch.cuda.synchronize()
    lhs = np.vdot(fy.cpu().numpy().astype(np.float64), g)
    assert lhs == pytest.approx(np.vdot(dh[:n].astype(np.float64), gt), rel=1e-4, abs=1e-6 * np.abs(gt).sum())


def test_adjoint_errors(tiny):
    ctx, cg, _, _ = make(tiny)
    with pytest.raises(wfbp.WfbpError):
        ctx.taps_gradient(torch.zeros(1, device=DEV), torch.zeros(1, device=DEV),
                          torch.zeros(ctx.dims.n_channels + 1, device=DEV))
    tube, table = tiny.views()
    cgm, _ = wfbp.configure_geometry(tiny.meta(), table)
    mixed = wfbp.Context(cgm, tiny.recon_config(), wfbp.make_ext(precision=T.PRECISION_MIXED), device=0)
    mixed.set_views(tube, table)
    with pytest.raises(wfbp.WfbpError) as e:
        mixed.backproject_adjoint(torch.zeros(1, device=DEV), torch.zeros(1, device=DEV))
    assert e.value.status == 5
    ffs = scans.tiny_ffs()
    tube, table = ffs.views()
    cgf, _ = wfbp.configure_geometry(ffs.meta(), table)
    cf = wfbp.Context(cgf, ffs.recon_config(), device=0)
    cf.set_views(tube, table)
    with pytest.raises(wfbp.WfbpError) as e:
        cf.rebin_adjoint(torch.zeros(1, device=DEV), torch.zeros(1, device=DEV))
    assert e.value.status == 5


def test_autograd_batch_vs_fp64_gradient(orc):
    # a batch of 4 scans of the small scanner (672 x 16, 1160 views/rotation,
    # pitch 1), independently seeded phantoms, 64 learnable taps; the volume
    # is reduced (96^2 x 6 slices, 2 rotations) so the FP64 oracle's gradient
    # stays within a test's time
    from freect_b200.autograd import Reconstructor
    specs = []
    for seed in range(4):
        s = scans.small(seed=seed)
        s.rotations = 2
        s.nx = s.ny = 96
        s.n_slices = 6
        specs.append(s)
    tube, table = specs[0].views()
    cg, gp = wfbp.configure_geometry(specs[0].meta(), table)
    rp = specs[0].recon_config()
    rec = Reconstructor(cg, rp, tube, table, n_taps=64)
    raws = [orc.synth_project(s.synth(), s.ellipsoids()) for s in specs]
    _, req = rec.ctx.slices()
    targets = [orc.voxelize(s.ellipsoids(), rp, req, 1.0) for s in specs]
    raw = torch.stack([dev(r) for r in raws]).requires_grad_(True)
    taps = torch.nn.Parameter(rec.initial_taps())
    vol = rec(raw, taps)
    tgt = torch.stack([dev(t) for t in targets])
    losses = []
    for b in range(4):
        m = torch.isfinite(vol[b])
        losses.append(((vol[b] - tgt[b])[m] ** 2).mean())
    loss = torch.stack(losses).sum()
    loss.backward()
    torch.cuda.synchronize()
    rec.ctx.check_device_status()
    full_taps = rec.base_taps.cpu().numpy().astype(np.float64)
    g_taps_ref = np.zeros(64)
    rng = np.random.default_rng(11)
    for b in range(4):
        L, g_raw, g_t, v64 = orc.loss_and_grad_f64(specs[b], raws[b], full_taps, targets[b], 64)
        assert float(losses[b].detach()) == pytest.approx(L, rel=1e-3)
        gr = raw.grad[b].cpu().numpy().astype(np.float64)
        assert np.linalg.norm(gr - g_raw) < 2e-3 * np.linalg.norm(g_raw)
        # 32 seeded sinogram entries (among those the loss depends on)
        nz = np.flatnonzero(np.abs(g_raw) > 1e-3 * np.abs(g_raw).max())
        idx = rng.choice(nz, 32, replace=False)
        assert np.allclose(gr.ravel()[idx], g_raw.ravel()[idx], rtol=1e-2, atol=1e-3 * np.abs(g_raw).max())
        g_taps_ref += g_t
    gt = taps.grad.cpu().numpy().astype(np.float64)
    assert np.allclose(gt, g_taps_ref, rtol=2e-3, atol=2e-3 * np.abs(g_taps_ref).max())
    # scans copied in on another stream, the forward waiting per scan: the same volumes
    raw_h = raw.detach().cpu().pin_memory()
    raw2 = torch.zeros_like(raw.detach())
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    ready = [torch.cuda.Event() for _ in range(4)]
    with torch.cuda.stream(side):
        for b in range(4):
            raw2[b].copy_(raw_h[b], non_blocking=True)
            ready[b].record(side)
    with torch.no_grad():
        vol2 = rec(raw2, taps, ready)
    torch.cuda.synchronize()
    assert torch.equal(torch.nan_to_num(vol2, nan=7.0), torch.nan_to_num(vol.detach(), nan=7.0))
    with pytest.raises(ValueError):
        rec(raw2, taps, ready[:2])
