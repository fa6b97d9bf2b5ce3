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


# ---------------------------------------------------------------------------
# DICOM-CT-PD: files written here by an encoder of the test's own (DICOM Part
# 10 element encoding: tag, VR, length, value; little endian), read back
# through the C ABI
# ---------------------------------------------------------------------------
import struct

_LONG = {"OB", "OW", "OF", "SQ", "UT", "UN"}


def _el(tag, vr, value, explicit):
    g, e = tag >> 16, tag & 0xFFFF
    if len(value) % 2:
        value += b" " if vr in ("CS", "LO", "DS", "UI", "IS") else b"\0"
    if not explicit:
        return struct.pack("<HHI", g, e, len(value)) + value
    if vr in _LONG:
        return struct.pack("<HH2sHI", g, e, vr.encode(), 0, len(value)) + value
    return struct.pack("<HH2sH", g, e, vr.encode(), len(value)) + value


def _dicom_file(path, elems, explicit=True, with_sequence=False):
    ts = b"1.2.840.10008.1.2.1" if explicit else b"1.2.840.10008.1.2"
    meta = _el(0x00020010, "UI", ts + b"\0", True)
    body = b""
    if with_sequence:  # an undefined-length sequence the reader must skip
        item = _el(0x00081150, "UI", b"1.2.3\0", explicit)
        seq_hdr = struct.pack("<HH2sHI", 0x0008, 0x1140, b"SQ", 0, 0xFFFFFFFF) if explicit else \
            struct.pack("<HHI", 0x0008, 0x1140, 0xFFFFFFFF)
        body += seq_hdr + struct.pack("<HHI", 0xFFFE, 0xE000, 0xFFFFFFFF) + item + \
            struct.pack("<HHI", 0xFFFE, 0xE00D, 0) + struct.pack("<HHI", 0xFFFE, 0xE0DD, 0)
    for tag, vr, val in sorted(elems, key=lambda t: t[0]):
        body += _el(tag, vr, val, explicit)
    with open(path, "wb") as f:
        f.write(b"\0" * 128 + b"DICM" + meta + body)


def _write_ctpd(d, raw, angles, zs, explicit, transpose, ffs="FFSNONE"):
    n, nr, nch = raw.shape
    slope, icpt = 0.5, -1024.0
    for k in range(n):
        counts = np.round((raw[k] - icpt) / slope).astype(np.uint16)
        img = counts.T if transpose else counts  # [channels][rows] or [rows][channels]
        elems = [
            (0x00080070, "LO", b"SYNTH"),
            (0x00280010, "US", struct.pack("<H", img.shape[0])),
            (0x00280011, "US", struct.pack("<H", img.shape[1])),
            (0x00281052, "DS", b"%g" % icpt),
            (0x00281053, "DS", b"%g" % slope),
            (0x70291010, "US", struct.pack("<H", nr)),
            (0x70291011, "US", struct.pack("<H", nch)),
            (0x70291002, "FL", struct.pack("<f", 1.2858)),
            (0x70291006, "FL", struct.pack("<f", 1.0947)),
            (0x7029100B, "CS", b"CYLINDRICAL"),
            (0x70311001, "FL", struct.pack("<f", angles[k])),
            (0x70311002, "FL", struct.pack("<f", zs[k])),
            (0x70311003, "FL", struct.pack("<f", 595.0)),
            (0x70311031, "FL", struct.pack("<f", 1085.6)),
            (0x70311033, "FL", struct.pack("<ff", 366.25, 15.5)),
            (0x7033100B, "FL", struct.pack("<f", 0.0)),
            (0x7033100C, "FL", struct.pack("<f", 0.0)),
            (0x7033100D, "FL", struct.pack("<f", 0.0)),
            (0x7033100E, "CS", ffs.encode()),
            (0x70331013, "US", struct.pack("<H", 1152)),
            (0x70371009, "CS", b"AXIAL"),
            (0x7037100A, "CS", b"FANBEAM"),
            (0x7FE00010, "OW", np.ascontiguousarray(img).astype("<u2").tobytes()),
        ]
        _dicom_file(str(d / ("proj_%05d.dcm" % k)), elems, explicit, with_sequence=(k == 0))
    return slope, icpt


@pytest.mark.parametrize("explicit,transpose", [(True, False), (False, True), (True, True)])
def test_dicom_ctpd_reader(tmp_path, explicit, transpose):
    rng = np.random.default_rng(7)
    n, nr, nch = 5, 4, 12
    slope, icpt = 0.5, -1024.0
    counts = rng.integers(0, 4000, (n, nr, nch))
    raw = (counts * slope + icpt).astype(np.float32)
    angles = rng.uniform(-3, 3, n).astype(np.float32)
    zs = rng.uniform(-50, 50, n).astype(np.float32)
    _write_ctpd(tmp_path, raw, angles, zs, explicit, transpose, ffs="FFSXYZ")
    m = wfbp.dicom_read_meta(str(tmp_path))
    assert (m.total_num_projections, m.detector_rows, m.detector_channels, m.projections_per_rotation) == (n, nr, nch, 1152)
    assert m.ffs_mode == T.FFS_PHIZ
    assert np.float32(m.detector_transverse_spacing) == np.float32(1.2858)
    assert np.float32(m.detector_axial_spacing) == np.float32(1.0947)
    assert (m.dist_source_to_isocenter, m.dist_source_to_detector) == (np.float32(595.0), np.float32(1085.6))
    assert (m.detector_central_channel, m.detector_central_row) == (366.25, 15.5)
    a, z, got = wfbp.dicom_read_frames(str(tmp_path), m)
    assert np.array_equal(a, angles) and np.array_equal(z, zs) and np.array_equal(got, raw)
    a2, z2, got2 = wfbp.dicom_read_frames(str(tmp_path), m, first=2, count=2)
    assert np.array_equal(got2, raw[2:4]) and np.array_equal(a2, angles[2:4])


def test_dicom_ctpd_rejects_bad_input(tmp_path):
    (tmp_path / "a.dcm").write_bytes(b"\0" * 140)  # no DICM marker
    with pytest.raises(wfbp.WfbpError):
        wfbp.dicom_read_meta(str(tmp_path))
    d = tmp_path / "big"
    d.mkdir()
    raw = np.zeros((2, 2, 3), np.float32)
    _write_ctpd(d, raw, np.zeros(2, np.float32), np.zeros(2, np.float32), True, False)
    m = wfbp.dicom_read_meta(str(d))
    with pytest.raises(wfbp.WfbpError):
        wfbp.dicom_read_frames(str(d), m, first=1, count=5)  # past the last file
