"""The oracle against outputs of the reference's own kernels.

tests/golden/ref_*.npz and tex_probe.npz were produced by
tests/golden/make_reference_fixtures.py, which runs the reference's
cuda_kernels.cuh (compiled unmodified from its source tree with a texture
object standing in for the removed texture-reference API) on a B200.
"""
import glob
import os

import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_FILES = sorted(glob.glob(os.path.join(GOLD, "ref_*.npz")))


def tex_emulate(img, xy, rounding):
    """tex2D, linear filter, clamp addressing, unnormalised coordinates, with
    the fractional weights reduced to 8 bits by `rounding`."""
    h, w = img.shape
    xb = xy[:, 0].astype(np.float32) - np.float32(0.5)
    yb = xy[:, 1].astype(np.float32) - np.float32(0.5)
    fx, fy = np.floor(xb), np.floor(yb)
    ax, ay = (xb - fx).astype(np.float32), (yb - fy).astype(np.float32)
    if rounding == "nearest":
        ax = np.rint(ax * 256) / 256
        ay = np.rint(ay * 256) / 256
    elif rounding == "truncate":
        ax = np.floor(ax * 256) / 256
        ay = np.floor(ay * 256) / 256
    x0 = np.clip(fx.astype(int), 0, w - 1)
    x1 = np.clip(fx.astype(int) + 1, 0, w - 1)
    y0 = np.clip(fy.astype(int), 0, h - 1)
    y1 = np.clip(fy.astype(int) + 1, 0, h - 1)
    return ((1 - ax) * (1 - ay) * img[y0, x0] + ax * (1 - ay) * img[y0, x1] + (1 - ax) * ay * img[y1, x0]
            + ax * ay * img[y1, x1])


def test_fixtures_present():
    assert len(REF_FILES) >= 4, "run tests/golden/make_reference_fixtures.py on a GPU"
    assert os.path.exists(os.path.join(GOLD, "tex_probe.npz"))


def test_texture_unit_weights_closest_to_8bit_round_to_nearest():
    # Among simple models of the texture unit's linear filter, 8-bit
    # round-to-nearest fractional weights are closest to the hardware; none
    # is exact (residual ~2e-3 RMS on unit-variance texels).
    d = np.load(os.path.join(GOLD, "tex_probe.npz"))
    img, xy, hw = d["img"], d["xy"], d["out"]
    rms = {r: float(np.sqrt(np.mean((tex_emulate(img, xy, r) - hw) ** 2))) for r in ("nearest", "truncate", "exact")}
    assert rms["nearest"] < rms["exact"] < rms["truncate"], rms
    assert rms["nearest"] < 3e-3, rms


def _spec_for(name):
    from tests.golden.make_reference_fixtures import cases
    return dict(cases())[name]


@pytest.mark.parametrize("path", REF_FILES, ids=[os.path.basename(p) for p in REF_FILES])
def test_oracle_transcript_matches_reference_kernels(orc, path):
    name = os.path.basename(path)[4:-4]
    spec = _spec_for(name)
    d = np.load(path)
    raw = d["raw"]
    cg, gp = orc.configure_geometry(spec.meta(), d["table"])
    tube, table = spec.views()
    assert np.array_equal(tube, d["tube"]) and np.array_equal(table, d["table"])
    # (1) backprojection transcript on the reference's own filtered rows:
    #     equal to the reference kernel to FP32 rounding
    rp = spec.recon_config()
    zn, zr = orc.slice_locations(cg, rp)
    assert np.array_equal(zn, d["z_native"]) and np.array_equal(zr, d["z_req"])
    gp.n_slices_native, gp.n_slices_requested = zn.size, zr.size
    vn = orc.backproject_ref32(cg, rp, gp, d["filtered"], tube, table, zn)
    rms, mx, n = orc.hu_error(vn, d["native"])
    assert np.array_equal(np.isnan(vn), np.isnan(d["native"]))  # same voxels without coverage
    assert n == np.isfinite(vn).sum() and rms < 0.005 and mx < 0.05, (rms, mx)
    vol = orc.thicken_ref32(rp, d["native"], zn, zr)
    assert np.allclose(vol, d["volume"], rtol=1e-5, atol=1e-7, equal_nan=True)
    # (2) rebin + filter: the texture unit's filter is modelled by 8-bit
    #     round-to-nearest weights (not exact; see the probe test above)
    filt = orc.rebin_filter_ref32(cg, raw, d["taps_fft"], q8=True)
    scale = np.abs(d["filtered"]).max()
    rel = np.abs(filt - d["filtered"]) / scale
    assert rel.max() < 5e-3 and np.percentile(rel, 99) < 1e-3
    # (3) whole path within a fraction of the parity budget (0.5 HU RMS / 2 HU max)
    ref = orc.reconstruct_ref32(spec, raw, taps_half=None, q8=True)
    rms, mx, n = orc.hu_error(ref["volume"], d["volume"])
    assert n == np.isfinite(d["volume"]).sum()
    assert rms < 0.25 and mx < 1.0, (rms, mx)
    # exact weights (the FP64 oracle) miss the 2 HU max budget on some inputs
    r64 = orc.reconstruct_f64(spec, raw)
    rms64, mx64, _ = orc.hu_error(r64["volume"], d["volume"])
    assert rms64 < 0.5, (rms64, mx64)


def test_oracle_transcript_matches_reference_kernels_full_size(orc):
    # the small scanner at its full size (672 ch x 16 rows x 3480 readings ->
    # 256^2 x 16 slices, Ram-Lak): the reference's own kernels ran on a B200
    # (full_ref_small.npz: seed, SHA-256 of the raw frames, final volume); the
    # oracle's FP32 transcript reproduces that volume from the regenerated frames
    import hashlib
    from freect_b200 import scans
    d = np.load(os.path.join(GOLD, "full_ref_small.npz"))
    spec = scans.small(seed=int(d["seed"]))
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    assert hashlib.sha256(np.ascontiguousarray(raw).tobytes()).hexdigest() == str(d["raw_sha256"])
    ref = orc.reconstruct_ref32(spec, raw, q8=True)
    assert np.array_equal(ref["z_req"], d["z_req"]) and np.array_equal(ref["z_native"], d["z_native"])
    rms, mx, n = orc.hu_error(ref["volume"], d["volume"])
    assert np.array_equal(np.isnan(ref["volume"]), np.isnan(d["volume"]))
    assert n == np.isfinite(d["volume"]).sum() and n > 0.9 * d["volume"].size
    assert rms < 0.25 and mx < 1.0, (rms, mx)
