"""Failure detection without a GPU fault: a kernel waits on an mbarrier that
nothing ever arrives at, the wait gives up after its wall-clock limit, the
kernel records WFBP_ERR_TIMEOUT in the context's error word and returns; the
host reads the status, and the context keeps working."""
import time

import numpy as np
import pytest

from freect_b200 import scans, wfbp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda", 0)


def test_bounded_wait_reports_timeout_and_context_survives(orc):
    spec = scans.tiny()
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    ctx = wfbp.Context(cg, spec.recon_config(), wfbp.make_ext(filter_window=spec.window), device=0)
    ctx.set_views(tube, table)
    raw = torch.from_numpy(orc.synth_project(spec.synth(), spec.ellipsoids())).to(DEV)
    before = ctx.alloc("volume")
    ctx.run(raw, before)
    torch.cuda.synchronize()
    ctx.check_device_status()
    t0 = time.perf_counter()
    ctx.selftest_bounded_wait(limit_ms=50)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    assert 0.04 < dt < 5.0
    with pytest.raises(wfbp.WfbpError) as e:
        ctx.check_device_status()
    assert e.value.status == 4  # WFBP_ERR_TIMEOUT
    ctx.check_device_status()  # read-and-clear: the word is clean again
    after = ctx.alloc("volume")
    ctx.run(raw, after)
    torch.cuda.synchronize()
    ctx.check_device_status()
    assert np.array_equal(after.cpu().numpy(), before.cpu().numpy(), equal_nan=True)
    with pytest.raises(wfbp.WfbpError):
        ctx.selftest_bounded_wait(limit_ms=0)
