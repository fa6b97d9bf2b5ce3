"""HU error of a GPU reconstruction against the FP64 oracle on one slab.

TEST INFRASTRUCTURE (the checker): used by tests/, smoke() and bench.py's HU
check, never by the product path.

The FP64 oracle reconstructs the slab of one requested slice from its own
window of readings, with the whole scan's slice positions, index angles and
z_rot (the construction of freect_b200.shard, which equals the whole-scan
result on that slab), so a full-size scan is checked in seconds instead of
reconstructing the whole volume in FP64 on the host.
"""
import os
import time

import numpy as np

from . import oracle as O


def hu_vs_fp64_slab(spec, cg, rp, tube, table, raw_window, vol, which=None):
    """RMS and max HU error of `vol` (numpy [nzr][ny][nx], or a callable
    (r0, r1) -> numpy slab) against the FP64 oracle on the slab of requested
    slice `which` (default: the middle one). raw_window(a0, a1) returns the
    raw readings [a0, a1) as a float32 numpy array."""
    from freect_b200 import shard
    O.set_threads(os.cpu_count() or 1)
    ce = O.ffs_effective(cg) if (cg.ffs_phi or cg.ffs_z) else cg
    nat, req = O.slice_locations(ce, rp)
    plans = shard.plan(cg, rp, table, req.size)
    p = plans[req.size // 2 if which is None else which]
    a0, a1 = p.readings
    t0 = time.perf_counter()
    ref = O.reconstruct_window_f64(shard.sub_geometry(cg, p), rp, spec.window, tube[a0:a1], table[a0:a1],
                                   raw_window(a0, a1), a0, nat[p.native[0]:p.native[1]],
                                   req[p.requested[0]:p.requested[1]])
    got = vol(*p.requested) if callable(vol) else np.asarray(vol)[p.requested[0]:p.requested[1]]
    rms, mx, n = O.hu_error(got, ref)
    return {"rms": rms, "max": mx, "voxels": n, "requested_slices": list(p.requested),
            "oracle_seconds": time.perf_counter() - t0,
            "note": "FP64 oracle on the slab of requested slice %d, full-coverage voxels" % p.requested[0]}
