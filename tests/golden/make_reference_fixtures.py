"""Golden fixtures from the reference's own kernels.

Runs applications/fct_wfbp/include/cuda_kernels.cuh -- compiled unmodified
from the reference tree into oracle/_ref/libref_wfbp_shim.so by
oracle/ref_shim/Makefile -- on a CUDA device, with the stage logic of
ReconstructionMachine.cu restated in oracle/ref_shim/ref_kernels_shim.cu,
and stores inputs and outputs as .npz files:

  ref_<case>.npz   raw frames, tube angles, table positions, the reference's
                   filtered projections, native volume and final volume
  tex_probe.npz    hardware bilinear texture samples at random coordinates
  tex_ramp.npz     samples of ramp textures on a fine grid of coordinates:
                   the texture unit's effective fractional weights
  full_ref_small.npz  the small scanner at its full size (672 ch x 16 rows x
                   3480 readings -> 256^2 x 16 slices, Ram-Lak): the seed, the
                   SHA-256 of the synthesised raw frames (150 MB, regenerated
                   from the seed by the test instead of being stored) and the
                   reference's final volume

Usage (needs a GPU):
  python tests/golden/make_reference_fixtures.py [outdir]               small cases
  python tests/golden/make_reference_fixtures.py --small-full [outdir]  full-size small scanner
"""
import ctypes as C
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from freect_b200 import abi_types as T  # noqa: E402
from freect_b200 import scans  # noqa: E402
from oracle import oracle as O  # noqa: E402

SHIM = os.path.join(ROOT, "oracle", "_ref", "libref_wfbp_shim.so")


def cases():
    """(name, spec) pairs small enough to commit."""
    out = [("tiny", scans.tiny(seed=11))]
    s = scans.tiny(seed=12, nch=160, nr=12, P=200, rotations=3, nx=64, n_slices=6)
    out.append(("medium", s))
    s = scans.tiny(seed=13, nch=64, nr=4, P=64, rotations=2.5, nx=32, n_slices=3)
    s.rotations = (64 * 2 + 69) / 64.0  # V = 197: views past the rebin grid
    out.append(("oddviews", s))
    s = scans.tiny(seed=14, nch=96, nr=8, P=96, rotations=3, nx=32, n_slices=4, window=T.FILTER_SHEPP_LOGAN)
    out.append(("shepplogan", s))
    return out


def load_shim():
    lib = C.CDLL(SHIM)
    F = C.POINTER(C.c_float)
    lib.ref_shim_run.restype = C.c_int
    lib.ref_shim_run.argtypes = [C.POINTER(T.CTGeometry), C.POINTER(T.ReconConfig), C.POINTER(T.GPUPrecompute),
                                 F, F, F, F, F, C.c_int, F, C.c_int, F, F, F]
    lib.ref_shim_tex_probe.restype = C.c_int
    lib.ref_shim_tex_probe.argtypes = [F, C.c_int, C.c_int, F, C.c_int, F]
    return lib


def taps_for(spec, cg):
    if spec.window == T.FILTER_REFERENCE:
        return O.taps_ref_fft(cg)
    return O.taps_fft_from_half(cg, O.taps_f64(cg, spec.window).astype(np.float32))


def run_reference(lib, spec, raw):
    tube, table = spec.views()
    cg, gp = O.configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    zn, zr = O.slice_locations(cg, rp)
    gp.n_slices_native, gp.n_slices_requested = zn.size, zr.size
    taps = taps_for(spec, cg)
    V, nr, nch = spec.V, spec.nr, spec.nch
    filt = np.zeros((V, nr, nch), np.float32)
    native = np.zeros((zn.size, spec.ny, spec.nx), np.float32)
    vol = np.zeros((zr.size, spec.ny, spec.nx), np.float32)
    raw = np.ascontiguousarray(raw, np.float32)
    st = lib.ref_shim_run(C.byref(cg), C.byref(rp), C.byref(gp), O.fp(raw), O.fp(taps), O.fp(tube), O.fp(table),
                          O.fp(zn), zn.size, O.fp(zr), zr.size, O.fp(filt), O.fp(native), O.fp(vol))
    if st != 0:
        raise RuntimeError("ref_shim_run failed with %d" % st)
    return dict(raw=raw, tube=tube, table=table, taps_fft=taps, filtered=filt, native=native, volume=vol,
                z_native=zn, z_req=zr)


def tex_probe(lib, seed=5, w=37, h=23, n=20000):
    rng = np.random.default_rng(seed)
    img = rng.standard_normal((h, w)).astype(np.float32)
    xy = np.stack([rng.uniform(-2, w + 2, n), rng.uniform(-2, h + 2, n)], 1).astype(np.float32)
    out = np.zeros(n, np.float32)
    st = lib.ref_shim_tex_probe(O.fp(img), w, h, O.fp(np.ascontiguousarray(xy)), n, O.fp(out))
    if st != 0:
        raise RuntimeError("ref_shim_tex_probe failed with %d" % st)
    return dict(img=img, xy=xy, out=out)


def tex_ramp_probe(lib, w=16, h=16, steps=4096):
    """Ramp textures T = i (along x) and T = j (along y), sampled on a fine
    grid of fractional coordinates: the outputs are the texture unit's
    effective interpolation weights."""
    ramp_x = np.tile(np.arange(w, dtype=np.float32), (h, 1))
    ramp_y = np.tile(np.arange(h, dtype=np.float32)[:, None], (1, w))
    f = (np.arange(steps, dtype=np.float64) / steps).astype(np.float32)
    xs = (np.float32(5.5) + f).astype(np.float32)
    xy_x = np.stack([xs, np.full(steps, 7.75, np.float32)], 1)
    xy_y = np.stack([np.full(steps, 7.75, np.float32), xs], 1)
    ox = np.zeros(steps, np.float32)
    oy = np.zeros(steps, np.float32)
    if lib.ref_shim_tex_probe(O.fp(ramp_x), w, h, O.fp(np.ascontiguousarray(xy_x)), steps, O.fp(ox)) != 0:
        raise RuntimeError("tex ramp probe x failed")
    if lib.ref_shim_tex_probe(O.fp(ramp_y), w, h, O.fp(np.ascontiguousarray(xy_y)), steps, O.fp(oy)) != 0:
        raise RuntimeError("tex ramp probe y failed")
    return dict(coord=xs, out_x=ox, out_y=oy)


SMALL_FULL_SEED = 3


def raw_digest(raw):
    """SHA-256 of the raw frames' bytes (float32, C order)."""
    return hashlib.sha256(np.ascontiguousarray(raw, np.float32).tobytes()).hexdigest()


def small_full(outdir):
    spec = scans.small(seed=SMALL_FULL_SEED)
    raw = O.synth_project(spec.synth(), spec.ellipsoids())
    res = run_reference(load_shim(), spec, raw)
    np.savez_compressed(os.path.join(outdir, "full_ref_small.npz"), seed=np.int64(SMALL_FULL_SEED),
                        raw_sha256=np.array(raw_digest(raw)), volume=res["volume"], z_native=res["z_native"],
                        z_req=res["z_req"])
    print("small_full", spec.V, spec.nr, spec.nch, res["volume"].shape, raw_digest(raw))


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    lib = load_shim()
    for name, spec in cases():
        raw = O.synth_project(spec.synth(), spec.ellipsoids())
        res = run_reference(lib, spec, raw)
        np.savez_compressed(os.path.join(outdir, "ref_%s.npz" % name), **res)
        print(name, spec.V, spec.nr, spec.nch, res["volume"].shape, float(np.nanmean(res["volume"])))
    np.savez_compressed(os.path.join(outdir, "tex_probe.npz"), **tex_probe(lib))
    np.savez_compressed(os.path.join(outdir, "tex_ramp.npz"), **tex_ramp_probe(lib))
    print("wrote", outdir)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    out = args[0] if args else os.path.dirname(os.path.abspath(__file__))
    if "--small-full" in sys.argv:
        small_full(out)
    else:
        main(out)
