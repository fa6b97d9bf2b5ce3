"""Z-slab sharding on the GPU (one GPU, the slabs run one after another):
every slab is reconstructed by its own context from its own window of
readings, and the stitched slabs equal the whole-scan reconstruction bit for
bit (FP32 and mixed forms, with and without a flying focal spot). The
multi-process path (one rank per GPU, gather of the slabs) is covered on
CPU by tests/test_shard.py with gloo ranks."""
import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans, shard, wfbp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda", 0)


def _spec(name):
    if name == "small":
        s = scans.small(seed=2)
        s.rotations = 5
        s.nx = s.ny = 96
        s.n_slices = 30
        return s
    return scans.tiny_ffs(mode=T.FFS_PHIZ, nch=64, nr=4, P=128, rotations=6, nx=32, n_slices=12)


@pytest.mark.parametrize("name", ["small", "ffs"])
@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
def test_slabs_stitch_to_whole(orc, name, precision):
    spec = _spec(name)
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    ext = wfbp.make_ext(precision=precision, filter_window=spec.window,
                        tex_weights=1 if precision == T.PRECISION_FP32 else 0)
    raw = torch.from_numpy(orc.synth_project(spec.synth(), spec.ellipsoids())).to(DEV)
    whole_ctx = wfbp.Context(cg, rp, ext, device=0)
    whole_ctx.set_views(tube, table)
    whole = whole_ctx.alloc("volume")
    whole_ctx.run(raw, whole)
    torch.cuda.synchronize()
    whole = whole.cpu().numpy()
    assert np.isfinite(whole).mean() > 0.5
    for world in (2, 3):
        plans = shard.plan(cg, rp, table, world)
        parts = []
        for p in plans:
            a0, a1 = p.readings
            assert a1 - a0 < raw.shape[0] or world == 1
            ctx = shard.slab_context(cg, rp, ext, tube, table, p, device=0)
            slab = ctx.alloc("volume")
            ctx.run(raw[a0:a1].contiguous(), slab)
            torch.cuda.synchronize()
            ctx.check_device_status()
            parts.append(slab.cpu().numpy())
            ctx.close()
        got = np.concatenate(parts)
        assert np.array_equal(got, whole, equal_nan=True), (world, np.nanmax(np.abs(got - whole)))
