"""CPU checks of the oracle (no GPU): known answers, identities, geometry.

The reference ships no tests or golden vectors for this path; these pin the
oracle to the formulas in the reference's sources and to the analytic
phantom. tests/test_golden.py pins it to outputs of the reference's own
kernels.
"""
import math

import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans


def _geom(orc, spec):
    tube, table = spec.views()
    cg, gp = orc.configure_geometry(spec.meta(), table)
    return cg, gp, tube, table


def test_ramp_taps_known_answers(orc):
    # resources/ramp.m:1-15 with c = a = 1 (Ram-Lak): h[0] = 1/(4 ds),
    # h[odd n] = -1/(pi^2 n^2 ds), h[even n != 0] = 0.
    spec = scans.small()
    cg, _, _, _ = _geom(orc, spec)
    ds = cg.detector_pixel_size_col * cg.distance_source_to_isocenter / cg.distance_source_to_detector
    taps = orc.taps_ref_fft(cg)  # fftshifted: taps[j] = h[j] for j < N/2
    N = taps.size
    assert N == 2048
    assert taps[0] == pytest.approx(1.0 / (4 * ds), rel=1e-6)
    for n in (1, 3, 5, 11, 101, 671):
        # float pi*n in the reference's r(t) perturbs sin(t) at large n
        assert abs(taps[n] + 1.0 / (math.pi ** 2 * n * n * ds)) < 2e-4 * abs(taps[n]) + 2e-7 * taps[0]
        assert taps[N - n] == taps[n]  # h[-n] after fftshift
    for n in (2, 4, 10, 100):
        assert abs(taps[n]) < 1e-5 * taps[0]
    half = orc.taps_f64(cg)
    assert np.allclose(taps[:672], half, rtol=2e-4, atol=1e-6 * taps[0])


def test_shepp_logan_taps(orc):
    spec = scans.rows64()
    cg, _, _, _ = _geom(orc, spec)
    ds = cg.detector_pixel_size_col * cg.distance_source_to_isocenter / cg.distance_source_to_detector
    h = orc.taps_f64(cg, T.FILTER_SHEPP_LOGAN)
    assert h[0] == pytest.approx(2.0 / (math.pi ** 2 * ds))
    assert h[3] == pytest.approx(-2.0 / (math.pi ** 2 * ds * 35.0))
    # DC gain of the discrete kernel is zero (sum over all n of h[n] = 0)
    n = np.arange(1, 200000, dtype=np.float64)
    dc = h[0] + 2 * np.sum(-2.0 / (math.pi ** 2 * ds * (4 * n * n - 1)))
    assert abs(dc) < 1e-5 * h[0]


def test_geometry_matches_reference_formulas(orc):
    spec = scans.small()
    cg, gp, tube, table = _geom(orc, spec)
    assert cg.num_detector_cols_padded_fft == 2048
    assert cg.z_rot == pytest.approx(9.6, rel=1e-5)
    csw = 595.0 * (spec.drow / 1085.6)
    assert cg.collimated_slice_width == pytest.approx(csw, rel=1e-6)
    assert cg.collimated_slice_width == pytest.approx(0.6, rel=1e-5)
    assert cg.theta_cone == pytest.approx(2 * math.atan(7.5 * csw / 595.0), rel=1e-6)
    afov = 2 * 595.0 * math.sin(335.5 * spec.dcol / 1085.6)
    assert cg.acquisition_field_of_view == pytest.approx(afov, rel=1e-6)
    assert gp.projections_per_half_turn == 580 and gp.n_half_turns == 6
    assert gp.pixel_scale == pytest.approx(1085.6 / (595.0 * spec.dcol), rel=1e-6)
    assert gp.two_pi_over_projections_per_rotation == pytest.approx(2 * math.pi / 1160, rel=1e-6)


def test_slice_lists_float_accumulation(orc):
    spec = scans.small()
    cg, _, _, _ = _geom(orc, spec)
    rp = spec.recon_config()
    zn, zr = orc.slice_locations(cg, rp)
    assert zr.size == 16 and zn.size == 26
    # float accumulation loc += delta (ReconstructionMachine.cu:115-119)
    loc = np.float32(rp.start_pos)
    for i in range(zn.size):
        assert zn[i] == loc
        loc = np.float32(loc + np.float32(cg.collimated_slice_width))
    # reversed direction
    rp.start_pos, rp.end_pos = rp.end_pos, rp.start_pos
    zn2, zr2 = orc.slice_locations(cg, rp)
    assert zr2.size == 16 and np.all(np.diff(zr2) < 0)
    # single slice
    rp.end_pos = rp.start_pos
    zn3, zr3 = orc.slice_locations(cg, rp)
    assert zn3.size == 1 and zr3.size == 1


def test_fft_filter_equals_toeplitz_on_data_window(orc):
    # The zero padding of the reference's FFT filter is >= nch - 1, so its
    # data window equals the linear (Toeplitz) convolution -- except the left
    # pad of view 0, which the rebin never rewrites after the first row.
    spec = scans.tiny(nch=64, nr=4, P=64, rotations=2.5)
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    cg, _, _, _ = _geom(orc, spec)
    taps_fft = orc.taps_ref_fft(cg)
    faithful = orc.rebin_filter_ref32(cg, raw, taps_fft)
    reb = orc.rebin_ref32(cg, raw)
    half = taps_fft[:64].astype(np.float64)
    lin = orc.filter_f32(reb, half)
    V = int(cg.total_number_of_projections)
    scale = np.abs(lin).max()
    assert V % 8 == 0
    d = np.abs(faithful - lin)
    assert d[1:].max() < 1e-5 * scale          # every view but 0
    assert d[0, 0].max() < 1e-5 * scale        # view 0, first row: pads still zero
    assert d[0, 1:].max() > 1e-5 * scale       # view 0, later rows: stale left pad


def test_views_beyond_rebin_grid_are_stale(orc):
    # rebin grid covers 8*floor(V/8) views (ReconstructionMachine.cu:255)
    spec = scans.tiny(nch=64, nr=3, P=64, rotations=2.5)
    spec.rotations = (64 * 2 + 69) / 64.0  # V = 197, 5 views outside the grid
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    cg, _, _, _ = _geom(orc, spec)
    V = int(cg.total_number_of_projections)
    assert V == 197
    faithful = orc.rebin_filter_ref32(cg, raw, orc.taps_ref_fft(cg))
    lin = orc.filter_f32(orc.rebin_ref32(cg, raw), orc.taps_ref_fft(cg)[:64].astype(np.float64))
    assert np.abs(faithful[192:, 0]).max() < 1e-12  # first row: never rebinned, zeros
    assert np.abs(faithful[192:, 1] - lin[192:, 1]).max() > 1e-3


def test_oracle_reconstructs_analytic_phantom(orc):
    spec = scans.tiny(nch=128, nr=8, P=128, rotations=3, nx=32, n_slices=3)
    raw = orc.synth_project(spec.synth(i0=0), spec.ellipsoids())
    r64 = orc.reconstruct_f64(spec, raw)
    vox = orc.voxelize(spec.ellipsoids(), r64["rp"], r64["z_req"], 1.0)
    hu = r64["volume"] * 1000 / scans.MU_WATER - 1000
    hv = vox * 1000 / scans.MU_WATER - 1000
    # interior water voxels (away from edges): within 25 HU of the phantom
    interior = np.abs(hv) < 1.0
    from scipy import ndimage
    plane = np.zeros((3, 3, 3), bool)
    plane[1] = ndimage.generate_binary_structure(2, 1)
    interior &= ndimage.binary_erosion(interior, structure=plane, iterations=2)
    assert interior.sum() > 200
    err = np.abs(hu - hv)[interior]
    assert np.median(err) < 10.0 and np.percentile(err, 95) < 40.0
    # the skull (about +1000 HU) is where the phantom puts it
    bone = hv > 900
    assert bone.sum() > 10 and np.mean(hu[bone]) > 500


def test_ref32_close_to_f64(orc):
    spec = scans.tiny()
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    r32 = orc.reconstruct_ref32(spec, raw)
    r64 = orc.reconstruct_f64(spec, raw)
    rms, mx, n = orc.hu_error(r32["volume"], r64["volume"])
    assert n == r32["volume"].size
    assert rms < 0.1 and mx < 0.5
    assert r64["updates"] > 0


def test_texture_weight_quantisation_effect(orc):
    # 8-bit fractional weights (texture unit) vs exact weights: visible but small
    spec = scans.tiny()
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    a = orc.reconstruct_ref32(spec, raw, q8=False)
    b = orc.reconstruct_ref32(spec, raw, q8=True)
    rms, mx, _ = orc.hu_error(a["volume"], b["volume"])
    assert 0.0 < rms < 2.0


def test_nan_where_no_half_turn_contributes(orc):
    # a slice far outside the scanned range gets NaN (0 * (1/0)), like the reference
    spec = scans.tiny(n_slices=1)
    raw = orc.synth_project(spec.synth(i0=0), spec.ellipsoids())
    cg, gp, tube, table = _geom(orc, spec)
    rp = spec.recon_config()
    filt = orc.rebin_filter_ref32(cg, raw, orc.taps_ref_fft(cg))
    v = orc.backproject_ref32(cg, rp, gp, filt, tube, table, np.array([500.0], np.float32))
    inside = v[0] != 0
    assert np.isnan(v[0]).sum() > 0
    v64, n = orc.backproject_f64(cg, rp, filt.astype(np.float64), tube.astype(np.float64),
                                 table.astype(np.float64), np.array([500.0]))
    assert n == 0 and np.isnan(v64).sum() == np.isnan(v).sum()


def test_adaptive_filter_oracle(orc):
    # ReconConfig.adaptive_filtration_s (parsed, never applied by fct_wfbp):
    # attenuation-adaptive smoothing of the raw line integrals, restated here
    # in numpy from its definition and checked against the C oracle
    rng = np.random.default_rng(3)
    raw = rng.uniform(0.0, 6.0, (5, 3, 17)).astype(np.float32)
    raw[2] = 1.5  # a uniform reading: smoothing changes nothing
    raw[3] = -rng.uniform(0.0, 1.0, (3, 17))  # no attenuation: p_max <= 0, unchanged
    s = 0.4
    got = orc.adaptive_filter_f64(raw, s)
    x = raw.astype(np.float64)
    pmax = x.reshape(5, -1).max(1)[:, None, None]
    pt = (1.0 - s) * pmax
    left = np.concatenate([x[..., :1], x[..., :-1]], -1)
    right = np.concatenate([x[..., 1:], x[..., -1:]], -1)
    pb = 0.25 * (left + 2.0 * x + right)
    w = np.clip((x - pt) / (pmax - pt), 0.0, 1.0)
    ref = np.where(pmax > 0, x + w * (pb - x), x)
    assert np.allclose(got, ref, rtol=1e-14, atol=1e-14)
    assert np.array_equal(got[2], x[2]) and np.array_equal(got[3], x[3])
    # below the threshold nothing changes; the reading's maximum is fully smoothed
    assert np.array_equal(got[x < pt], x[x < pt])
    r, c = np.unravel_index(np.argmax(x[0]), x[0].shape)
    assert abs(got[0, r, c] - pb[0, r, c]) < 1e-12
    # s = 0 is the reference's behaviour (off)
    assert np.array_equal(orc.adaptive_filter_f64(raw, 0.0), x)
