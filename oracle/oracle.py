"""ctypes wrapper of the CPU oracle (oracle/wfbp_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker. The product (freect_b200) never
imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from freect_b200 import abi_types as T

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_wfbp.so")
_lib = None

_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)


def build():
    r = subprocess.run(["make", "-s", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        G, R, GP = C.POINTER(T.CTGeometry), C.POINTER(T.ReconConfig), C.POINTER(T.GPUPrecompute)
        protos = {
            "orc_set_threads": (None, [C.c_int]),
            "orc_get_threads": (C.c_int, []),
            "orc_configure_geometry": (C.c_int, [C.POINTER(T.ScanMeta), _F, G, GP]),
            "orc_slice_locations": (C.c_int, [G, R, _F, C.c_int, C.POINTER(C.c_int), _F, C.c_int,
                                              C.POINTER(C.c_int)]),
            "orc_filter_taps_ref_fft": (None, [G, C.c_float, C.c_float, _F]),
            "orc_filter_taps_f64": (None, [G, C.c_int, C.c_double, C.c_double, _D, C.c_int]),
            "orc_rebin_ref32": (None, [G, _F, C.c_int, _F]),
            "orc_rebin_f64": (None, [G, _F, _D]),
            "orc_rebin_f64_off": (None, [G, _F, C.c_long, _D]),
            "orc_filter_f64": (None, [C.c_int, C.c_long, _D, _D, _D]),
            "orc_filter_f32": (None, [C.c_int, C.c_long, _D, _F, _F]),
            "orc_rebin_filter_ref32": (C.c_int, [G, _F, _F, C.c_int, _F]),
            "orc_backproject_ref32": (None, [G, R, GP, _F, _F, _F, _F, C.c_int, _F]),
            "orc_backproject_f64": (C.c_ulonglong, [G, R, _D, _D, _D, _D, C.c_int, _D]),
            "orc_thicken_ref32": (None, [R, _F, _F, C.c_int, _F, C.c_int, _F]),
            "orc_thicken_f64": (None, [R, _D, _D, C.c_int, _D, C.c_int, _D]),
            "orc_synth_project": (C.c_int, [C.POINTER(T.SynthScan), C.POINTER(T.Ellipsoid), C.c_int, _F]),
            "orc_voxelize": (None, [C.POINTER(T.Ellipsoid), C.c_int, R, _D, C.c_int, C.c_double, C.c_int, _D]),
            "orc_ffs_effective": (C.c_int, [G, G]),
            "orc_rebin_ffs_f64": (C.c_int, [G, _F, _D]),
            "orc_rebin_ffs_f64_off": (C.c_int, [G, _F, C.c_long, _D]),
            "orc_thicken_adjoint_f64": (None, [R, _D, _D, C.c_int, _D, C.c_int, _D]),
            "orc_backproject_adjoint_f64": (None, [G, R, _D, _D, _D, _D, C.c_int, _D]),
            "orc_taps_gradient_f64": (None, [C.c_int, C.c_long, _D, _D, C.c_int, _D]),
            "orc_rebin_adjoint_f64": (None, [G, _D, _D]),
            "orc_adaptive_filter_f64": (None, [_F, C.c_long, C.c_int, C.c_int, C.c_double, _D]),
        }
        for name, (res, args) in protos.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def fp(a):
    return a.ctypes.data_as(_F)


def dp(a):
    return a.ctypes.data_as(_D)


def set_threads(n):
    load().orc_set_threads(int(n))


def threads():
    return load().orc_get_threads()


def configure_geometry(meta, table):
    cg, gp = T.CTGeometry(), T.GPUPrecompute()
    t = _f(table)
    st = load().orc_configure_geometry(C.byref(meta), fp(t), C.byref(cg), C.byref(gp))
    if st:
        raise ValueError("orc_configure_geometry: status %d" % st)
    return cg, gp


def slice_locations(cg, rp):
    lib = load()
    nn, nr = C.c_int(), C.c_int()
    lib.orc_slice_locations(C.byref(cg), C.byref(rp), None, 0, C.byref(nn), None, 0, C.byref(nr))
    nat = np.zeros(nn.value, np.float32)
    req = np.zeros(nr.value, np.float32)
    lib.orc_slice_locations(C.byref(cg), C.byref(rp), fp(nat), nn.value, C.byref(nn), fp(req), nr.value,
                            C.byref(nr))
    return nat, req


def taps_ref_fft(cg, c=1.0, a=1.0):
    out = np.zeros(int(cg.num_detector_cols_padded_fft), np.float32)
    load().orc_filter_taps_ref_fft(C.byref(cg), c, a, fp(out))
    return out


def taps_f64(cg, window=T.FILTER_REFERENCE, c=1.0, a=1.0, n=None):
    n = int(cg.num_detector_cols) if n is None else n
    out = np.zeros(n, np.float64)
    load().orc_filter_taps_f64(C.byref(cg), window, c, a, dp(out), n)
    return out


def taps_fft_from_half(cg, half):
    """fftshifted N_fft float taps (generate_filter's layout) from symmetric half taps"""
    N = int(cg.num_detector_cols_padded_fft)
    out = np.zeros(N, np.float32)
    half = np.asarray(half)
    for j in range(N):
        i = j if j < N // 2 else j - N
        a = abs(i)
        if a < half.size:
            out[j] = half[a]
    return out


def rebin_ref32(cg, raw, q8=False):
    V, nr, nch = int(cg.total_number_of_projections), int(cg.num_detector_rows), int(cg.num_detector_cols)
    out = np.zeros((V, nr, nch), np.float32)
    r = _f(raw)
    load().orc_rebin_ref32(C.byref(cg), fp(r), int(bool(q8)), fp(out))
    return out


def adaptive_filter_f64(raw, s):
    """Adaptive filtration of raw readings [n][rows][channels] with strength
    s (ReconConfig.adaptive_filtration_s), FP64 (wfbp_oracle.c)."""
    r = _f(raw)
    out = np.zeros(r.shape, np.float64)
    load().orc_adaptive_filter_f64(fp(r), r.shape[0], r.shape[1], r.shape[2], float(s), dp(out))
    return out


def rebin_f64(cg, raw, offset=0):
    """offset: index of raw's first reading within the whole scan (a window
    is rebinned with the whole scan's index angles)."""
    V, nr, nch = int(cg.total_number_of_projections), int(cg.num_detector_rows), int(cg.num_detector_cols)
    out = np.zeros((V, nr, nch), np.float64)
    r = _f(raw)
    load().orc_rebin_f64_off(C.byref(cg), fp(r), int(offset), dp(out))
    return out


def filter_f64(rows, half):
    rows = _d(rows)
    nch = rows.shape[-1]
    out = np.zeros_like(rows)
    h = _d(half)
    load().orc_filter_f64(nch, rows.size // nch, dp(h), dp(rows), dp(out))
    return out


def filter_f32(rows, half):
    rows = _f(rows)
    nch = rows.shape[-1]
    out = np.zeros_like(rows)
    h = _d(half)
    load().orc_filter_f32(nch, rows.size // nch, dp(h), fp(rows), fp(out))
    return out


def rebin_filter_ref32(cg, raw, taps_fft, q8=False):
    V, nr, nch = int(cg.total_number_of_projections), int(cg.num_detector_rows), int(cg.num_detector_cols)
    out = np.zeros((V, nr, nch), np.float32)
    r, t = _f(raw), _f(taps_fft)
    st = load().orc_rebin_filter_ref32(C.byref(cg), fp(r), fp(t), int(bool(q8)), fp(out))
    if st:
        raise MemoryError("orc_rebin_filter_ref32")
    return out


def backproject_ref32(cg, rp, gp, filtered, tube, table, slices):
    slices = _f(slices)
    vol = np.zeros((slices.size, int(rp.ny), int(rp.nx)), np.float32)
    f, t, z = _f(filtered), _f(tube), _f(table)
    load().orc_backproject_ref32(C.byref(cg), C.byref(rp), C.byref(gp), fp(f), fp(t), fp(z), fp(slices),
                                 slices.size, fp(vol))
    return vol


def backproject_f64(cg, rp, filtered, tube, table, slices):
    slices = _d(slices)
    vol = np.zeros((slices.size, int(rp.ny), int(rp.nx)), np.float64)
    f, t, z = _d(filtered), _d(tube), _d(table)
    n = load().orc_backproject_f64(C.byref(cg), C.byref(rp), dp(f), dp(t), dp(z), dp(slices), slices.size, dp(vol))
    return vol, int(n)


def thicken_ref32(rp, vol_native, z_native, z_req):
    vn, zn, zr = _f(vol_native), _f(z_native), _f(z_req)
    out = np.zeros((zr.size,) + vn.shape[1:], np.float32)
    load().orc_thicken_ref32(C.byref(rp), fp(vn), fp(zn), zn.size, fp(zr), zr.size, fp(out))
    return out


def thicken_f64(rp, vol_native, z_native, z_req):
    vn, zn, zr = _d(vol_native), _d(z_native), _d(z_req)
    out = np.zeros((zr.size,) + vn.shape[1:], np.float64)
    load().orc_thicken_f64(C.byref(rp), dp(vn), dp(zn), zn.size, dp(zr), zr.size, dp(out))
    return out


def synth_project(scan, ellipsoids):
    out = np.zeros((scan.n_readings, scan.rows, scan.channels), np.float32)
    arr = (T.Ellipsoid * max(len(ellipsoids), 1))()
    for i, e in enumerate(ellipsoids):
        arr[i] = e
    st = load().orc_synth_project(C.byref(scan), arr, len(ellipsoids), fp(out))
    if st:
        raise ValueError("orc_synth_project: status %d" % st)
    return out


def voxelize(ellipsoids, rp, z, dz, ss=3):
    z = _d(z)
    out = np.zeros((z.size, int(rp.ny), int(rp.nx)), np.float64)
    arr = (T.Ellipsoid * max(len(ellipsoids), 1))()
    for i, e in enumerate(ellipsoids):
        arr[i] = e
    load().orc_voxelize(arr, len(ellipsoids), C.byref(rp), dp(z), z.size, dz, ss, dp(out))
    return out


# --------------------------------------------------------------------------
# whole-path helpers
# --------------------------------------------------------------------------

def reconstruct_ref32(spec, raw, taps_half=None, q8=False):
    """The reference's FP32 path on raw frames: (native volume, final volume, slices)."""
    tube, table = spec.views()
    cg, gp = configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    if taps_half is None:
        if spec.window == T.FILTER_REFERENCE:
            taps_fft = taps_ref_fft(cg)
        else:
            taps_fft = taps_fft_from_half(cg, taps_f64(cg, spec.window).astype(np.float32))
    else:
        taps_fft = taps_fft_from_half(cg, taps_half)
    filt = rebin_filter_ref32(cg, raw, taps_fft, q8=q8)
    zn, zr = slice_locations(cg, rp)
    gp.n_slices_native, gp.n_slices_requested = zn.size, zr.size
    vn = backproject_ref32(cg, rp, gp, filt, tube, table, zn)
    vol = thicken_ref32(rp, vn, zn, zr)
    return dict(cg=cg, gp=gp, rp=rp, filtered=filt, native=vn, volume=vol, z_native=zn, z_req=zr)


def ffs_effective(cg):
    """effective geometry of a flying-focal-spot scan (one view per state cycle)"""
    ce = T.CTGeometry()
    st = load().orc_ffs_effective(C.byref(cg), C.byref(ce))
    if st:
        raise ValueError("orc_ffs_effective: readings not a multiple of the focal states")
    return ce


def rebin_ffs_f64(cg, raw, offset_views=0):
    """offset_views: index of raw's first view (focal-state cycle) within the whole scan."""
    ce = ffs_effective(cg)
    out = np.zeros((int(ce.total_number_of_projections), int(ce.num_detector_rows), int(ce.num_detector_cols)),
                   np.float64)
    r = _f(raw)
    st = load().orc_rebin_ffs_f64_off(C.byref(cg), fp(r), int(offset_views), dp(out))
    if st:
        raise ValueError("orc_rebin_ffs_f64: status %d" % st)
    return out


def reconstruct_f64(spec, raw, taps_half=None):
    """FP64 oracle of the same algorithm (effective geometry with FFS)."""
    tube, table = spec.views()
    cg, gp = configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    if cg.ffs_phi or cg.ffs_z:
        G = (2 if cg.ffs_phi else 1) * (2 if cg.ffs_z else 1)
        reb = rebin_ffs_f64(cg, raw)
        cg = ffs_effective(cg)
        tube, table = tube[::G].copy(), table[::G].copy()
        half = taps_f64(cg, spec.window) if taps_half is None else np.asarray(taps_half, np.float64)
    else:
        half = taps_f64(cg, spec.window) if taps_half is None else np.asarray(taps_half, np.float64)
        reb = rebin_f64(cg, raw)
    filt = filter_f64(reb, half)
    zn, zr = slice_locations(cg, rp)
    vn, n_updates = backproject_f64(cg, rp, filt, tube.astype(np.float64), table.astype(np.float64), zn)
    vol = thicken_f64(rp, vn, zn, zr)
    return dict(cg=cg, gp=gp, rp=rp, rebinned=reb, filtered=filt, native=vn, volume=vol, z_native=zn, z_req=zr,
                updates=n_updates)


def reconstruct_window_f64(cg, rp, window, tube_w, table_w, raw_w, offset_readings, z_native, z_req):
    """FP64 oracle of a slab reconstructed from a window of a scan's readings:
    cg is the whole scan's geometry with total_number_of_projections set to
    the window's readings (z_rot kept), offset_readings the window's first
    reading; the rebin uses the whole scan's index angles, the slices are the
    given lists. With FFS the window starts on a focal-state cycle."""
    G = (2 if cg.ffs_phi else 1) * (2 if cg.ffs_z else 1)
    if G > 1:
        x = rebin_ffs_f64(cg, raw_w, offset_views=offset_readings // G)
        ce = ffs_effective(cg)
    else:
        x = rebin_f64(cg, raw_w, offset=offset_readings)
        ce = cg
    y = filter_f64(x, taps_f64(ce, window))
    tw = np.asarray(tube_w, np.float64)[::G]
    zw = np.asarray(table_w, np.float64)[::G]
    vn, _ = backproject_f64(ce, rp, y, tw, zw, z_native)
    return thicken_f64(rp, vn, z_native, z_req)


def hu_error(a, b, mu_water=0.019):
    """RMS and max |a-b| in HU over voxels finite in both (and nonzero mask)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = np.isfinite(a) & np.isfinite(b)
    d = (a[m] - b[m]) * 1000.0 / mu_water
    if d.size == 0:
        return float("nan"), float("nan"), 0
    return float(np.sqrt(np.mean(d * d))), float(np.max(np.abs(d))), int(m.sum())


# --------------------------------------------------------------------------
# adjoints and the FP64 gradient of an image loss
# --------------------------------------------------------------------------

def thicken_adjoint_f64(rp, g_vol, z_native, z_req):
    gv, zn, zr = _d(g_vol), _d(z_native), _d(z_req)
    out = np.zeros((zn.size,) + gv.shape[1:], np.float64)
    load().orc_thicken_adjoint_f64(C.byref(rp), dp(gv), dp(zn), zn.size, dp(zr), zr.size, dp(out))
    return out


def backproject_adjoint_f64(cg, rp, g_native, tube, table, slices):
    gn, t, z, sl = _d(g_native), _d(tube), _d(table), _d(slices)
    out = np.zeros((int(cg.total_number_of_projections), int(cg.num_detector_rows), int(cg.num_detector_cols)),
                   np.float64)
    load().orc_backproject_adjoint_f64(C.byref(cg), C.byref(rp), dp(gn), dp(t), dp(z), dp(sl), sl.size, dp(out))
    return out


def taps_gradient_f64(g_filtered, rebinned, ntaps):
    g, x = _d(g_filtered), _d(rebinned)
    nch = g.shape[-1]
    out = np.zeros(ntaps, np.float64)
    load().orc_taps_gradient_f64(nch, g.size // nch, dp(g), dp(x), ntaps, dp(out))
    return out


def rebin_adjoint_f64(cg, g_rebinned):
    g = _d(g_rebinned)
    out = np.zeros((int(cg.total_number_of_projections), int(cg.num_detector_rows), int(cg.num_detector_cols)),
                   np.float64)
    load().orc_rebin_adjoint_f64(C.byref(cg), dp(g), dp(out))
    return out


def _forward_f64(spec, raw, taps_half):
    tube, table = spec.views()
    cg, gp = configure_geometry(spec.meta(), table)
    rp = spec.recon_config()
    x = rebin_f64(cg, raw)
    y = filter_f64(x, np.asarray(taps_half, np.float64))
    zn, zr = slice_locations(cg, rp)
    t64, z64 = tube.astype(np.float64), table.astype(np.float64)
    vn, _ = backproject_f64(cg, rp, y, t64, z64, zn)
    vol = thicken_f64(rp, vn, zn, zr)
    return cg, rp, x, y, zn, zr, t64, z64, vn, vol


def loss_f64(spec, raw, taps_half, target):
    """L = mean over finite voxels of (vol - target)^2, FP64 path with the
    filter taps `taps_half` (exact texel weights)."""
    vol = _forward_f64(spec, raw, taps_half)[-1]
    m = np.isfinite(vol)
    return float(((vol[m] - target[m]) ** 2).sum() / m.sum())


def loss_and_grad_f64(spec, raw, taps_half, target, ntaps):
    """L of loss_f64 and its gradient by the FP64 adjoints: returns
    (L, dL/draw, dL/dtaps[:ntaps], vol)."""
    cg, rp, x, y, zn, zr, t64, z64, vn, vol = _forward_f64(spec, raw, taps_half)
    taps = np.asarray(taps_half, np.float64)
    m = np.isfinite(vol)
    n = m.sum()
    diff = np.where(m, vol - target, 0.0)
    L = float((diff[m] ** 2).sum() / n)
    g_vol = 2.0 * diff / n
    g_vn = thicken_adjoint_f64(rp, g_vol, zn, zr)
    g_vn[~np.isfinite(vn)] = 0.0
    g_y = backproject_adjoint_f64(cg, rp, g_vn, t64, z64, zn)
    g_x = filter_f64(g_y, taps)
    g_raw = rebin_adjoint_f64(cg, g_x)
    g_taps = taps_gradient_f64(g_y, x, ntaps)
    return L, g_raw, g_taps, vol
