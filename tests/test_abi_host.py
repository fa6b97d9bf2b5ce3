"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and its host-only entry points (geometry, slice lists,
taps, argument validation) agree with the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans, wfbp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"^\s*(?:int|const char\*|void)\s+(wfbp_\w+)\s*\(", txt, re.M))
    return names


def test_library_exports_every_declared_symbol(lib):
    declared = _declared()
    assert len(declared) >= 17
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(wfbp.exported_symbols())


def test_struct_layout_matches_reference_header():
    # tests/golden/struct_layout.json was produced by compiling the reference's
    # recon_structs.h (tests/golden/make_struct_layout.py); both the ctypes
    # mirror and include/freect_wfbp.h (compiled here) must match it.
    import json
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_struct_layout as msl
    gold = json.load(open(os.path.join(ROOT, "tests", "golden", "struct_layout.json")))
    for name, fields in msl.FIELDS.items():
        cls = getattr(T, name)
        assert C.sizeof(cls) == gold[name]["sizeof"], name
        for f in fields:
            assert getattr(cls, f).offset == gold[name][f], (name, f)
    ours = msl.run('#include "freect_wfbp.h"', [os.path.join(ROOT, "include")])
    assert ours == gold


@pytest.mark.parametrize("spec", [scans.small(), scans.rows64(), scans.tiny()])
def test_configure_geometry_matches_oracle(orc, spec):
    tube, table = spec.views()
    cg1, gp1 = wfbp.configure_geometry(spec.meta(), table)
    cg2, gp2 = orc.configure_geometry(spec.meta(), table)
    assert bytes(cg1) == bytes(cg2)
    assert bytes(gp1) == bytes(gp2)
    rp = spec.recon_config()
    n1, r1 = wfbp.slice_locations(cg1, rp)
    n2, r2 = orc.slice_locations(cg2, rp)
    assert np.array_equal(n1, n2) and np.array_equal(r1, r2)
    assert r1.size == spec.n_slices


def test_filter_taps_match_oracle(orc):
    spec = scans.small()
    tube, table = spec.views()
    cg, _ = wfbp.configure_geometry(spec.meta(), table)
    t = wfbp.filter_taps(cg)
    ref = orc.taps_ref_fft(cg)[:672]
    assert np.array_equal(t, ref)
    sl = wfbp.filter_taps(cg, T.FILTER_SHEPP_LOGAN)
    assert np.allclose(sl, orc.taps_f64(cg, T.FILTER_SHEPP_LOGAN), rtol=1e-6)


def test_invalid_arguments_are_rejected_without_a_device(lib):
    spec = scans.tiny()
    tube, table = spec.views()
    meta = spec.meta()
    bad = T.ScanMeta.from_buffer_copy(meta)
    bad.total_num_projections = bad.projections_per_rotation  # needs > P
    with pytest.raises(wfbp.WfbpError) as e:
        wfbp.configure_geometry(bad, table)
    assert e.value.status == 1
    cg, gp = wfbp.configure_geometry(meta, table)
    rp = spec.recon_config()
    for field, val in (("nx", 0), ("recon_fov", 0.0), ("slice_thickness", -1.0)):
        r2 = T.ReconConfig.from_buffer_copy(rp)
        setattr(r2, field, val)
        h = C.c_void_p()
        assert lib.wfbp_ctx_create(C.byref(cg), C.byref(r2), None, 0, C.byref(h)) == 1
        assert not h
    ext = wfbp.make_ext()
    ext.version = 99
    h = C.c_void_p()
    assert lib.wfbp_ctx_create(C.byref(cg), C.byref(rp), C.byref(ext), 0, C.byref(h)) == 1
    assert lib.wfbp_ctx_create(None, C.byref(rp), None, 0, C.byref(h)) == 1
    assert lib.wfbp_status_string(3) == b"WFBP_ERR_CUDA"
    assert lib.wfbp_query(None, None) == 1
    assert lib.wfbp_rebin(None, None, None, None) == 1


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(wfbp, "_lib", None)
    monkeypatch.setattr(wfbp, "_LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(ImportError):
        wfbp.load()


def test_ffs_geometry_and_validation(lib, orc):
    # FFS readings: the context derives the effective geometry; a reading
    # count that is not a multiple of the focal states is rejected before
    # any device work
    spec = scans.tiny_ffs(mode=T.FFS_PHIZ, nch=64, nr=8, P=256)
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    assert cg.ffs_phi and cg.ffs_z
    ce = orc.ffs_effective(cg)
    assert ce.num_detector_cols == 128 and ce.num_detector_rows == 16
    assert ce.total_number_of_projections == spec.V // 4 and ce.projections_per_rotation == 64
    assert ce.detector_central_col == pytest.approx(2 * spec.c0 + 0.5)
    bad = T.CTGeometry.from_buffer_copy(cg)
    bad.total_number_of_projections -= 1
    h = C.c_void_p()
    assert lib.wfbp_ctx_create(C.byref(bad), C.byref(spec.recon_config()), None, 0, C.byref(h)) == 1


def test_bp_config_names_round_trip():
    from freect_b200 import autotune
    for key in [(16, 16, 4, 16, 32), (16, 20, 8, 20, 16), (8, 16, 8, 8, 32)]:
        assert autotune.parse_config_name(autotune.config_name(key)) == key
    with pytest.raises(ValueError):
        autotune.parse_config_name("16x16/4w16")
