"""wfbp_run_static: the reconstruction with no device allocation.

Some callers cannot let the library call cudaMalloc -- their device memory
belongs to their own pool, or they run inside a fixed memory budget, or they
cannot afford cudaMalloc's synchronisation in their loop. wfbp_run_static
keeps the intermediates in a static device array instead. These tests call it
through the C ABI and check it against wfbp_run on the same context, bit for
bit, twice in a row (the array keeps the previous call's contents); that the
device's free memory does not change across its calls (nothing is allocated);
and that oversized geometries are rejected. This file is collected last so
that a failure here does not stop a run before the other tests.
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


def _static(lib, ctx, raw, vol):
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.wfbp_run_static(ctx.handle, C.c_void_p(raw.data_ptr()), C.c_void_p(vol.data_ptr()), stream)


@pytest.mark.parametrize("precision", [T.PRECISION_FP32, T.PRECISION_MIXED])
def test_run_static_matches_run_twice(orc, precision):
    lib = wfbp.load()
    dev = torch.device("cuda", 0)
    # the first call on a device loads the library's device code that holds the
    # static array and looks up its address: done once, outside the check
    warm = scans.tiny(seed=2)
    wctx = _ctx(warm, precision)
    wraw = torch.from_numpy(orc.synth_project(warm.synth(), warm.ellipsoids())).to(dev)
    wvol = wctx.alloc("volume")
    assert _static(lib, wctx, wraw, wvol) == 0, lib.wfbp_last_error(wctx.handle)
    torch.cuda.synchronize()
    wctx.close()
    for seed in (3, 4):  # two different scans, back to back, each on a fresh context
        spec = scans.tiny(seed=seed)
        raw = torch.from_numpy(orc.synth_project(spec.synth(), spec.ellipsoids())).to(dev)
        ctx = _ctx(spec, precision)
        got, got2 = ctx.alloc("volume"), ctx.alloc("volume")
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(dev)
        st = _static(lib, ctx, raw, got)
        assert st == 0, lib.wfbp_last_error(ctx.handle)
        st = _static(lib, ctx, raw, got2)  # second call in a row on the same array
        assert st == 0, lib.wfbp_last_error(ctx.handle)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(dev)
        assert free1 == free0, "wfbp_run_static changed the device's free memory by %d bytes" % (free0 - free1)
        # the existing entry point (which allocates its own scratch) on the same context
        ref = ctx.alloc("volume")
        ctx.run(raw, ref)
        torch.cuda.synchronize()
        a = got.cpu().numpy()
        assert np.isfinite(a).any()
        assert np.array_equal(a, ref.cpu().numpy(), equal_nan=True)
        assert np.array_equal(got2.cpu().numpy(), a, equal_nan=True)
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
