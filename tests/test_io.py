"""Input files: the recon-parameter YAML of fct_wfbp (parse_config) and the
FreeCT 2-file scan format (meta.yaml + projections.dat), through the C ABI
(host only)."""
import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans, wfbp


def test_recon_yaml(tmp_path):
    p = tmp_path / "recon.yaml"
    p.write_text("# a recon file\nraw_data_dir: /data/scan_01\noutput_dir: './out'\nstart_pos: -12.5\n"
                 "end_pos: 37.25\nrecon_fov: 360\nslice_thickness: 1.5\nnx: 512\nny: 384\nrecon_kernel: 2\n"
                 "x_origin: -3.0   # offset\ny_origin: 4.5\ntube_angle_offset: 0.25\n")
    rp = wfbp.parse_recon_config(str(p))
    assert rp.raw_data_dir == b"/data/scan_01" and rp.output_dir == b"./out"
    assert rp.output_file == (str(p) + "_recon.dat").encode()
    assert (rp.start_pos, rp.end_pos, rp.recon_fov, rp.slice_thickness) == (-12.5, 37.25, 360.0, 1.5)
    assert rp.slice_pitch == 1.5  # absent: the slice thickness (parse_config.cpp:59-60)
    assert (rp.nx, rp.ny, rp.recon_kernel) == (512, 384, 2)
    assert (rp.x_origin, rp.y_origin, rp.tube_angle_offset, rp.adaptive_filtration_s) == (-3.0, 4.5, 0.25, 0.0)
    bad = tmp_path / "bad.yaml"
    bad.write_text("- a list item\n")
    with pytest.raises(wfbp.WfbpError):
        wfbp.parse_recon_config(str(bad))
    with pytest.raises(wfbp.WfbpError):
        wfbp.parse_recon_config(str(tmp_path / "missing.yaml"))


@pytest.mark.parametrize("ffs", [T.FFS_NONE, T.FFS_PHIZ])
def test_freect_scan_round_trip(orc, tmp_path, ffs):
    spec = scans.tiny(nch=40, nr=4, P=64, rotations=2, nx=16, n_slices=2)
    spec.ffs_mode = ffs
    tube, table = spec.views()
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    meta = spec.meta()
    wfbp.write_scan(str(tmp_path), meta, tube, table, raw)
    m = wfbp.read_meta(str(tmp_path))
    assert bytes(m) == bytes(meta)
    t, z, r = wfbp.read_frames(str(tmp_path), m)
    assert np.array_equal(t, tube) and np.array_equal(z, table) and np.array_equal(r, raw)
    # a window of readings with one seek
    t, z, r = wfbp.read_frames(str(tmp_path), m, first=17, count=9)
    assert np.array_equal(t, tube[17:26]) and np.array_equal(z, table[17:26]) and np.array_equal(r, raw[17:26])
    with pytest.raises(wfbp.WfbpError):
        wfbp.read_frames(str(tmp_path), m, first=spec.V - 2, count=3)
    # a file shorter than its metadata
    with open(tmp_path / "projections.dat", "r+b") as f:
        f.truncate(100)
    with pytest.raises(wfbp.WfbpError):
        wfbp.read_frames(str(tmp_path), m)


def test_meta_requires_geometry_keys(tmp_path):
    (tmp_path / "meta.yaml").write_text("detector_rows: 4\ndetector_channels: 8\n")
    with pytest.raises(wfbp.WfbpError):
        wfbp.read_meta(str(tmp_path))


@pytest.mark.parametrize("rk,window,c,a", [(T.RECON_KERNEL_RAMLAK, T.FILTER_REFERENCE, 1.0, 1.0),
                                           (T.RECON_KERNEL_SHEPP_LOGAN, T.FILTER_SHEPP_LOGAN, 1.0, 1.0),
                                           (T.RECON_KERNEL_HANN, T.FILTER_REFERENCE, 1.0, 0.5),
                                           (T.RECON_KERNEL_HAMMING, T.FILTER_REFERENCE, 1.0, 0.54)])
def test_recon_kernel_selects_filter(orc, tmp_path, rk, window, c, a):
    # recon_kernel from a recon YAML (parse_config.cpp:53) -> filter window and
    # generate_filter's (c, a) (resources/ramp.m); taps against the oracle's
    p = tmp_path / "recon.yaml"
    p.write_text("recon_fov: 250\nslice_thickness: 1\nnx: 32\nny: 32\nrecon_kernel: %d\n" % rk)
    rp = wfbp.parse_recon_config(str(p))
    w, cc, aa = wfbp.recon_kernel_filter(rp.recon_kernel)
    assert (w, cc) == (window, c) and abs(aa - a) < 1e-7
    spec = scans.small()
    tube, table = spec.views()
    cg, _ = wfbp.configure_geometry(spec.meta(), table)
    got = wfbp.filter_taps(cg, w, cc, aa)
    ref = orc.taps_f64(cg, w, cc, aa)
    # generate_filter in FP32 (ReconstructionMachine.cu:478-513) against the FP64 formula
    assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max()


def test_recon_kernel_rejects_unknown_values():
    for rk in (-1, 4, 100):
        with pytest.raises(wfbp.WfbpError):
            wfbp.recon_kernel_filter(rk)
