"""wfbp_run_static: the reconstruction with no device allocation.

Some callers cannot let the library call cudaMalloc -- their device memory
belongs to their own pool, or they run inside a fixed memory budget, or they
cannot afford cudaMalloc's synchronisation in their loop. wfbp_run_static
keeps the intermediates in a static device array instead. These tests call it
through the C ABI and check it against the same four stages run on
context-allocated buffers (the context's own layout, as wfbp_run_static
uses), twice in a row (the array keeps the previous call's contents), and
that oversized geometries are
rejected. This file is collected last so that a failure here does not stop a
run before the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans, wfbp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)


def _ctx(spec, precision):
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ext = wfbp.make_ext(precision=precision, filter_window=spec.window,
                        tex_weights=1 if precision == T.PRECISION_FP32 else 0)
    ctx = wfbp.Context(cg, spec.recon_config(), ext, device=0)
    ctx.set_views(tube, table)
    return ctx


@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
def test_run_static_matches_run_twice(orc, precision):
    lib = wfbp.load()
    dev = torch.device("cuda", 0)
    for seed in (3, 4):  # two different scans, back to back
        spec = scans.tiny(seed=seed)
        raw = torch.from_numpy(orc.synth_project(spec.synth(), spec.ellipsoids())).to(dev)
        ctx = _ctx(spec, precision)
        ref = ctx.alloc("volume")
        reb, filt, sc, vn = ctx.alloc("rebinned"), ctx.alloc("filtered"), ctx.alloc("row_scales"), ctx.alloc("native")
        ctx.rebin(raw, reb)
        ctx.filter(reb, filt, sc)
        ctx.backproject(filt, vn, sc)
        ctx.thicken(vn, ref)
        got = ctx.alloc("volume")
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        st = lib.wfbp_run_static(ctx.handle, C.c_void_p(raw.data_ptr()), C.c_void_p(got.data_ptr()), stream)
        assert st == 0, lib.wfbp_last_error(ctx.handle)
        torch.cuda.synchronize()
        a, b = got.cpu().numpy(), ref.cpu().numpy()
        rms, mx, n = orc.hu_error(a, b)
        assert n == a.size
        assert rms <= 1e-3 and mx <= 1e-2, (rms, mx)  # same kernels on the same layout
        # second call in a row on the same array
        got2 = ctx.alloc("volume")
        st = lib.wfbp_run_static(ctx.handle, C.c_void_p(raw.data_ptr()), C.c_void_p(got2.data_ptr()), stream)
        assert st == 0
        torch.cuda.synchronize()
        assert np.array_equal(got2.cpu().numpy(), a)
        ctx.close()


def test_run_static_rejects_oversized_geometry(orc):
    spec = scans.small()  # 37 M samples: intermediates far above the static array
    lib = wfbp.load()
    ctx = _ctx(spec, T.PRECISION_FP32)
    raw = ctx.alloc("raw")
    vol = ctx.alloc("volume")
    st = lib.wfbp_run_static(ctx.handle, C.c_void_p(raw.data_ptr()), C.c_void_p(vol.data_ptr()), None)
    assert st == 1
    msg = lib.wfbp_last_error(ctx.handle).decode()
    assert "static scratch" in msg and str(32 << 20) in msg
    ctx.close()
