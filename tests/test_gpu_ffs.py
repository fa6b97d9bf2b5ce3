"""Flying focal spot on the GPU (no counterpart in the reference's WFBP,
whose fct_wfbp ignores CTGeometry's FFS fields): readings cycle through the
focal states of fct_icd's generate_ffs_offset and are merged onto an
effective detector with twice the channels / rows. Judged against the FP64
oracle of the same algorithm."""
import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans, wfbp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda", 0)
MODES = [T.FFS_PHI, T.FFS_Z, T.FFS_PHIZ]


def run(spec, raw, precision, layout=T.LAYOUT_REFERENCE):
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ext = wfbp.make_ext(precision=precision, filter_window=spec.window, filtered_layout=layout)
    ctx = wfbp.Context(cg, spec.recon_config(), ext, device=0)
    ctx.set_views(tube, table)
    vol = ctx.alloc("volume")
    ctx.run(torch.from_numpy(raw).to(DEV), vol)
    torch.cuda.synchronize()
    ctx.check_device_status()
    return ctx, vol.cpu().numpy()


@pytest.mark.parametrize("mode", MODES)
def test_ffs_effective_geometry_matches_oracle(orc, mode):
    spec = scans.tiny_ffs(mode=mode, nch=64, nr=8, P=256)
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ctx = wfbp.Context(cg, spec.recon_config(), device=0)
    ce, _ = ctx.geometry()
    assert bytes(ce) == bytes(orc.ffs_effective(cg))
    G = (2 if cg.ffs_phi else 1) * (2 if cg.ffs_z else 1)
    d = ctx.dims
    assert d.n_readings == spec.V and d.n_views == spec.V // G
    assert d.raw_channels == spec.nch and d.n_channels == spec.nch * (2 if cg.ffs_phi else 1)
    assert d.raw_rows == spec.nr and d.n_rows == spec.nr * (2 if cg.ffs_z else 1)


@pytest.mark.parametrize("mode", MODES)
def test_ffs_fp32_vs_fp64(orc, mode):
    spec = scans.tiny_ffs(mode=mode, nch=64, nr=8, P=256)
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    r64 = orc.reconstruct_f64(spec, raw)
    for layout in (T.LAYOUT_REFERENCE, T.LAYOUT_BACKPROJECTION):
        _, got = run(spec, raw, T.PRECISION_FP32, layout)
        rms, mx, n = orc.hu_error(got, r64["volume"])
        assert n == np.isfinite(r64["volume"]).sum()
        assert rms < 0.1 and mx < 1.0, (mode, layout, rms, mx)


@pytest.mark.parametrize("layout", [T.LAYOUT_REFERENCE, T.LAYOUT_BACKPROJECTION])
@pytest.mark.parametrize("mode", MODES)
def test_ffs_mixed_vs_fp64(orc, mode, layout):
    spec = scans.tiny_ffs(mode=mode, nch=64, nr=8, P=256)
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    r64 = orc.reconstruct_f64(spec, raw)
    _, got = run(spec, raw, T.PRECISION_MIXED, layout)
    rms, mx, n = orc.hu_error(got, r64["volume"])
    assert n == np.isfinite(r64["volume"]).sum()
    assert rms <= 1.0, (mode, layout, rms, mx)


def test_ffs_reconstructs_phantom(orc):
    # noiseless phi+z FFS scan: water within a few HU of the voxelised phantom
    spec = scans.tiny_ffs(mode=T.FFS_PHIZ, nch=64, nr=4, P=256, nx=32, n_slices=3)
    raw = orc.synth_project(spec.synth(i0=0), spec.ellipsoids())
    _, got = run(spec, raw, T.PRECISION_FP32)
    vox = orc.voxelize(spec.ellipsoids(), spec.recon_config(), orc.slice_locations(
        orc.ffs_effective(wfbp.configure_geometry(spec.meta(), spec.views()[1])[0]), spec.recon_config())[1], 1.0)
    hu, hv = got * 1000 / scans.MU_WATER - 1000, vox * 1000 / scans.MU_WATER - 1000
    water = np.abs(hv) < 1.0
    assert water.sum() > 100
    assert np.median(np.abs(hu - hv)[water]) < 10.0
