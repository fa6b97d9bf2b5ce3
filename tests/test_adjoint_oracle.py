"""The FP64 oracle's adjoints (the transposes of its forward loops) and its
gradient of an image loss: dot-product identities, and central finite
differences (eps = 1e-3) on 32 seeded sinogram entries and all 64
learnable taps. The reconstruction is linear in the raw readings and in the
taps, so the MSE loss is quadratic in each and the central difference
equals the directional derivative up to rounding: the tolerances are tight.
These pin the reference gradient the GPU adjoints are checked against."""
import numpy as np
import pytest

from freect_b200 import scans


@pytest.fixture(scope="module")
def geo(orc):
    spec = scans.tiny(nch=96, nr=6, P=96, rotations=3, nx=24, n_slices=3)
    tube, table = spec.views()
    cg, gp = orc.configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    zn, zr = orc.slice_locations(cg, rp)
    return spec, cg, rp, tube.astype(np.float64), table.astype(np.float64), zn, zr


def test_adjoint_dot_products(orc, geo):
    spec, cg, rp, tube, table, zn, zr = geo
    rng = np.random.default_rng(0)
    V, nr, nch = spec.V, spec.nr, spec.nch
    # rebin
    raw = rng.standard_normal((V, nr, nch)).astype(np.float32)
    gx = rng.standard_normal((V, nr, nch))
    a = np.vdot(orc.rebin_f64(cg, raw), gx)
    b = np.vdot(raw.astype(np.float64), orc.rebin_adjoint_f64(cg, gx))
    assert a == pytest.approx(b, rel=1e-10)
    # backprojection (linear in the filtered rows)
    y = rng.standard_normal((V, nr, nch))
    gn = rng.standard_normal((zn.size, spec.ny, spec.nx))
    vn, _ = orc.backproject_f64(cg, rp, y, tube, table, zn)
    fin = np.isfinite(vn)
    gn[~fin] = 0.0
    a = np.vdot(np.where(fin, vn, 0.0), gn)
    b = np.vdot(y, orc.backproject_adjoint_f64(cg, rp, gn, tube, table, zn))
    assert a == pytest.approx(b, rel=1e-10)
    # thickening
    v = rng.standard_normal((zn.size, spec.ny, spec.nx))
    gv = rng.standard_normal((zr.size, spec.ny, spec.nx))
    a = np.vdot(orc.thicken_f64(rp, v, zn, zr), gv)
    b = np.vdot(v, orc.thicken_adjoint_f64(rp, gv, zn, zr))
    assert a == pytest.approx(b, rel=1e-10)
    # filter: symmetric Toeplitz, and the tap gradient
    taps = orc.taps_f64(cg)
    x = rng.standard_normal((V * nr, nch))
    g = rng.standard_normal((V * nr, nch))
    assert np.vdot(orc.filter_f64(x, taps), g) == pytest.approx(np.vdot(x, orc.filter_f64(g, taps)), rel=1e-10)
    dh = np.zeros(nch)
    dh[:8] = rng.standard_normal(8)
    lin = np.vdot(orc.filter_f64(x, dh), g)  # filter is linear in the taps
    assert lin == pytest.approx(np.vdot(dh[:8], orc.taps_gradient_f64(g, x, 8)), rel=1e-10)


def test_loss_gradient_finite_differences(orc, geo):
    spec, cg, rp, tube, table, zn, zr = geo
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    taps = orc.taps_f64(cg)
    target = orc.voxelize(spec.ellipsoids(), rp, zr, 1.0)
    L, g_raw, g_taps, vol = orc.loss_and_grad_f64(spec, raw, taps, target, 64)
    assert np.isfinite(vol).all()
    assert L == pytest.approx(orc.loss_f64(spec, raw, taps, target), rel=1e-12)
    eps = 1e-3
    # 32 seeded sinogram entries the loss depends on; the perturbation is
    # applied in float32 (the raw readings' type), so divide by the step
    # actually taken
    rng = np.random.default_rng(1)
    nz = np.flatnonzero(np.abs(g_raw) > 1e-3 * np.abs(g_raw).max())
    scale = np.abs(g_raw).max()
    for flat in rng.choice(nz, 32, replace=False):
        idx = np.unravel_index(flat, raw.shape)
        rp_, rm_ = raw.copy(), raw.copy()
        rp_[idx] += np.float32(eps)
        rm_[idx] -= np.float32(eps)
        step = float(rp_[idx]) - float(rm_[idx])
        fd = (orc.loss_f64(spec, rp_, taps, target) - orc.loss_f64(spec, rm_, taps, target)) / step
        assert fd == pytest.approx(g_raw[idx], rel=1e-5, abs=1e-7 * scale)
    # all 64 learnable taps
    tscale = np.abs(g_taps).max()
    for d in range(64):
        tp, tm = taps.copy(), taps.copy()
        tp[d] += eps
        tm[d] -= eps
        fd = (orc.loss_f64(spec, raw, tp, target) - orc.loss_f64(spec, raw, tm, target)) / (2 * eps)
        assert fd == pytest.approx(g_taps[d], rel=1e-6, abs=1e-8 * tscale)
