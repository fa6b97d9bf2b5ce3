"""ctypes binding of the C ABI in include/freect_wfbp.h.

The library is the compiled sm_100a code in freect_b200/lib/libfreect_wfbp.so;
there is no fallback: if the library is missing or a call fails, an exception
is raised. Device buffers are torch tensors (their data pointers are passed
through the ABI) and every stage runs on torch's current CUDA stream unless a
stream is given.
"""
import ctypes as C
import os

import numpy as np

from . import abi_types as T

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libfreect_wfbp.so")
_lib = None

# name -> (restype, argtypes); the exported symbols of include/freect_wfbp.h
_VP = C.c_void_p
_PROTOS = {
    "wfbp_configure_geometry": (C.c_int, [C.POINTER(T.ScanMeta), C.POINTER(C.c_float), C.POINTER(T.CTGeometry),
                                          C.POINTER(T.GPUPrecompute)]),
    "wfbp_effective_geometry": (C.c_int, [C.POINTER(T.CTGeometry), C.POINTER(T.CTGeometry)]),
    "wfbp_slice_locations": (C.c_int, [C.POINTER(T.CTGeometry), C.POINTER(T.ReconConfig), C.POINTER(C.c_float),
                                       C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_int,
                                       C.POINTER(C.c_int)]),
    "wfbp_filter_taps": (C.c_int, [C.POINTER(T.CTGeometry), C.c_int, C.c_float, C.c_float, C.POINTER(C.c_float),
                                   C.c_int]),
    "wfbp_dicom_read_meta": (C.c_int, [C.c_char_p, C.POINTER(T.ScanMeta)]),
    "wfbp_dicom_read_frames": (C.c_int, [C.c_char_p, C.POINTER(T.ScanMeta), C.c_int, C.c_int, C.POINTER(C.c_float),
                                         C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "wfbp_recon_kernel_filter": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float),
                                           C.POINTER(C.c_float)]),
    "wfbp_ctx_create": (C.c_int, [C.POINTER(T.CTGeometry), C.POINTER(T.ReconConfig), C.POINTER(T.Ext), C.c_int,
                                  C.POINTER(_VP)]),
    "wfbp_ctx_destroy": (C.c_int, [_VP]),
    "wfbp_query": (C.c_int, [_VP, C.POINTER(T.Dims)]),
    "wfbp_set_views": (C.c_int, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "wfbp_get_slices": (C.c_int, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "wfbp_set_reading_offset": (C.c_int, [_VP, C.c_int]),
    "wfbp_set_slices": (C.c_int, [_VP, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float), C.c_int]),
    "wfbp_get_geometry": (C.c_int, [_VP, C.POINTER(T.CTGeometry), C.POINTER(T.GPUPrecompute)]),
    "wfbp_bp_configs": (C.c_int, [_VP, C.POINTER(T.BpConfig), C.c_int, C.POINTER(C.c_int)]),
    "wfbp_get_bp_config": (C.c_int, [_VP, C.POINTER(T.BpConfig)]),
    "wfbp_set_bp_config": (C.c_int, [_VP, C.POINTER(T.BpConfig)]),
    "wfbp_last_error": (C.c_char_p, [_VP]),
    "wfbp_check_device_status": (C.c_int, [_VP]),
    "wfbp_selftest_bounded_wait": (C.c_int, [_VP, C.c_int, _VP]),
    "wfbp_status_string": (C.c_char_p, [C.c_int]),
    "wfbp_rebin": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wfbp_filter": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "wfbp_backproject": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "wfbp_thicken": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wfbp_run": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wfbp_run_host": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wfbp_run_timed": (C.c_int, [_VP, _VP, _VP, _VP, C.POINTER(C.c_float)]),
    "wfbp_run_static": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wfbp_set_taps": (C.c_int, [_VP, _VP, C.c_int, _VP]),
    "wfbp_get_taps": (C.c_int, [_VP, _VP, _VP]),
    "wfbp_thicken_adjoint": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wfbp_backproject_adjoint": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wfbp_filter_adjoint": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wfbp_rebin_adjoint": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wfbp_taps_gradient": (C.c_int, [_VP, _VP, _VP, _VP, C.c_int, _VP]),
    "wfbp_batch_create": (C.c_int, [C.POINTER(_VP), C.c_int, C.POINTER(_VP)]),
    "wfbp_batch_destroy": (C.c_int, [_VP]),
    "wfbp_batch_run": (C.c_int, [_VP, C.POINTER(_VP), C.POINTER(_VP), _VP]),
    "wfbp_batch_run_host": (C.c_int, [_VP, C.POINTER(_VP), C.POINTER(_VP), _VP]),
    "wfbp_batch_size": (C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "wfbp_batch_bp_configs": (C.c_int, [_VP, C.POINTER(T.BpConfig), C.c_int, C.POINTER(C.c_int)]),
    "wfbp_batch_get_bp_config": (C.c_int, [_VP, C.POINTER(T.BpConfig)]),
    "wfbp_batch_set_bp_config": (C.c_int, [_VP, C.POINTER(T.BpConfig)]),
    "wfbp_batch_check_device_status": (C.c_int, [_VP]),
    "wfbp_batch_last_error": (C.c_char_p, [_VP]),
    "wfbp_parse_recon_config": (C.c_int, [C.c_char_p, C.POINTER(T.ReconConfig)]),
    "wfbp_read_meta": (C.c_int, [C.c_char_p, C.POINTER(T.ScanMeta)]),
    "wfbp_read_frames": (C.c_int, [C.c_char_p, C.POINTER(T.ScanMeta), C.c_int, C.c_int, _VP, _VP, _VP]),
    "wfbp_write_scan": (C.c_int, [C.c_char_p, C.POINTER(T.ScanMeta), _VP, _VP, _VP]),
    "wfbp_synth_project": (C.c_int, [C.POINTER(T.SynthScan), C.POINTER(T.Ellipsoid), C.c_int, _VP, _VP]),
}


class WfbpError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (T.STATUS_NAMES.get(status, status), msg))
        self.status = status


def lib_path():
    return _LIB_PATH


def load():
    """Loads the compiled library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError("freect_b200: %s is missing; build it with `python -m freect_b200.build_lib`"
                              % _LIB_PATH)
        lib = C.CDLL(_LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def exported_symbols():
    return sorted(_PROTOS)


def _check(status, what, ctx=None):
    if status != 0:
        msg = what
        if ctx is not None:
            m = load().wfbp_last_error(ctx)
            if m:
                msg += ": " + m.decode()
        raise WfbpError(status, msg)


def _fptr(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def _dptr(t):
    """device pointer of a torch tensor (or None)"""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def configure_geometry(meta, table_positions):
    """ReconstructionMachine::ConfigureCTGeometry + GPUPrecompute::InitFromCTGeometry."""
    cg, gp = T.CTGeometry(), T.GPUPrecompute()
    tbl, ptr = _fptr(table_positions)
    if tbl.size < meta.total_num_projections:
        raise ValueError("table_positions shorter than total_num_projections")
    _check(load().wfbp_configure_geometry(C.byref(meta), ptr, C.byref(cg), C.byref(gp)), "wfbp_configure_geometry")
    return cg, gp


def effective_geometry(cg):
    """The geometry a context's stages work on (effective one with a flying focal spot)."""
    eff = T.CTGeometry()
    _check(load().wfbp_effective_geometry(C.byref(cg), C.byref(eff)), "wfbp_effective_geometry")
    return eff


def slice_locations(cg, rp):
    """Native and requested slice z lists (float32), ReconstructionMachine.cu:107-137."""
    lib = load()
    nn, nr = C.c_int(), C.c_int()
    _check(lib.wfbp_slice_locations(C.byref(cg), C.byref(rp), None, 0, C.byref(nn), None, 0, C.byref(nr)),
           "wfbp_slice_locations")
    nat = np.zeros(nn.value, np.float32)
    req = np.zeros(nr.value, np.float32)
    _check(lib.wfbp_slice_locations(C.byref(cg), C.byref(rp), nat.ctypes.data_as(C.POINTER(C.c_float)), nn.value,
                                    C.byref(nn), req.ctypes.data_as(C.POINTER(C.c_float)), nr.value, C.byref(nr)),
           "wfbp_slice_locations")
    return nat, req


def filter_taps(cg, window=T.FILTER_REFERENCE, c=1.0, a=1.0, n=None):
    n = int(cg.num_detector_cols) if n is None else n
    out = np.zeros(n, np.float32)
    _check(load().wfbp_filter_taps(C.byref(cg), window, c, a, out.ctypes.data_as(C.POINTER(C.c_float)), n),
           "wfbp_filter_taps")
    return out


def recon_kernel_filter(recon_kernel):
    """(window, c, a) that ReconConfig.recon_kernel selects (wfbp_recon_kernel)."""
    w, c, a = C.c_int(), C.c_float(), C.c_float()
    _check(load().wfbp_recon_kernel_filter(recon_kernel, C.byref(w), C.byref(c), C.byref(a)),
           "wfbp_recon_kernel_filter")
    return w.value, c.value, a.value


def make_ext(precision=T.PRECISION_FP32, filter_window=T.FILTER_REFERENCE, filter_c=1.0, filter_a=1.0,
             user_taps=None, tex_weights=0, bp_slab=0, filtered_layout=T.LAYOUT_REFERENCE, adjoint_scale_table=0):
    e = T.Ext()
    e.version = T.EXT_VERSION
    e.precision = precision
    e.filter_window = filter_window
    e.filter_c = filter_c
    e.filter_a = filter_a
    e.tex_weights = tex_weights
    e.bp_slab = bp_slab
    e.filtered_layout = filtered_layout
    e.adjoint_scale_table = adjoint_scale_table
    if user_taps is not None:
        arr = np.ascontiguousarray(user_taps, dtype=np.float32)
        e._taps_keepalive = arr
        e.user_taps = arr.ctypes.data_as(C.POINTER(C.c_float))
        e.n_user_taps = arr.size
    return e


class Context:
    """One scan geometry + recon config on one device (wfbp_ctx)."""

    def __init__(self, cg, rp, ext=None, device=0):
        self._lib = load()
        self._h = C.c_void_p()
        self.cg, self.rp = cg, rp
        self.ext = ext if ext is not None else make_ext()
        _check(self._lib.wfbp_ctx_create(C.byref(cg), C.byref(rp), C.byref(self.ext), device, C.byref(self._h)),
               "wfbp_ctx_create")
        self.device = device
        d = T.Dims()
        _check(self._lib.wfbp_query(self._h, C.byref(d)), "wfbp_query", self._h)
        self.dims = d

    def close(self):
        if self._h:
            self._lib.wfbp_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def geometry(self):
        """(CTGeometry, GPUPrecompute) the stages work on (effective ones with FFS)."""
        cg, gp = T.CTGeometry(), T.GPUPrecompute()
        _check(self._lib.wfbp_get_geometry(self._h, C.byref(cg), C.byref(gp)), "wfbp_get_geometry", self._h)
        return cg, gp

    def check_device_status(self):
        _check(self._lib.wfbp_check_device_status(self._h), "wfbp_check_device_status", self._h)

    def selftest_bounded_wait(self, limit_ms=50, stream=None):
        """Runs a wait that can never complete, bounded to limit_ms."""
        _check(self._lib.wfbp_selftest_bounded_wait(self._h, int(limit_ms), _stream(stream)),
               "wfbp_selftest_bounded_wait", self._h)

    @property
    def handle(self):
        return self._h

    def slices(self):
        nat = np.zeros(self.dims.n_slices_native, np.float32)
        req = np.zeros(self.dims.n_slices_requested, np.float32)
        _check(self._lib.wfbp_get_slices(self._h, nat.ctypes.data_as(C.POINTER(C.c_float)),
                                         req.ctypes.data_as(C.POINTER(C.c_float))), "wfbp_get_slices", self._h)
        return nat, req

    def set_reading_offset(self, offset):
        """Index of this context's first reading within the whole scan."""
        _check(self._lib.wfbp_set_reading_offset(self._h, int(offset)), "wfbp_set_reading_offset", self._h)

    def set_slices(self, native_z, requested_z):
        """Explicit native / requested slice lists (e.g. a z-slab of a larger scan)."""
        n, npp = _fptr(native_z)
        r, rpp = _fptr(requested_z)
        _check(self._lib.wfbp_set_slices(self._h, npp, n.size, rpp, r.size), "wfbp_set_slices", self._h)
        d = T.Dims()
        _check(self._lib.wfbp_query(self._h, C.byref(d)), "wfbp_query", self._h)
        self.dims = d

    def set_views(self, tube_angles, table_positions):
        t, tp = _fptr(tube_angles)
        z, zp = _fptr(table_positions)
        if t.size < self.dims.n_readings or z.size < self.dims.n_readings:
            raise ValueError("need %d tube angles and table positions" % self.dims.n_readings)
        _check(self._lib.wfbp_set_views(self._h, tp, zp), "wfbp_set_views", self._h)

    # ---- backprojection launch configuration ----
    def bp_configs(self):
        """Backprojection configurations that fit this geometry (after set_views)."""
        n = C.c_int()
        _check(self._lib.wfbp_bp_configs(self._h, None, 0, C.byref(n)), "wfbp_bp_configs", self._h)
        arr = (T.BpConfig * max(n.value, 1))()
        _check(self._lib.wfbp_bp_configs(self._h, arr, n.value, C.byref(n)), "wfbp_bp_configs", self._h)
        return [arr[i] for i in range(n.value)]

    def bp_config(self):
        c = T.BpConfig()
        _check(self._lib.wfbp_get_bp_config(self._h, C.byref(c)), "wfbp_get_bp_config", self._h)
        return c

    def set_bp_config(self, config):
        if isinstance(config, (tuple, list)):
            c = T.BpConfig()
            c.tile_x, c.tile_y, c.cols_per_step = config[:3]
            c.consumer_warps = config[3] if len(config) > 3 else 0
            c.slab = config[4] if len(config) > 4 else 0
            config = c
        _check(self._lib.wfbp_set_bp_config(self._h, C.byref(config)), "wfbp_set_bp_config", self._h)

    # ---- stages (torch CUDA tensors) ----
    def rebin(self, raw, rebinned, stream=None):
        _check(self._lib.wfbp_rebin(self._h, _dptr(raw), _dptr(rebinned), _stream(stream)), "wfbp_rebin", self._h)

    def filter(self, rebinned, filtered, row_scales=None, stream=None):
        _check(self._lib.wfbp_filter(self._h, _dptr(rebinned), _dptr(filtered), _dptr(row_scales), _stream(stream)),
               "wfbp_filter", self._h)

    def backproject(self, filtered, volume_native, row_scales=None, update_count=None, stream=None):
        _check(self._lib.wfbp_backproject(self._h, _dptr(filtered), _dptr(row_scales), _dptr(volume_native),
                                          _dptr(update_count), _stream(stream)), "wfbp_backproject", self._h)

    def thicken(self, volume_native, volume, stream=None):
        _check(self._lib.wfbp_thicken(self._h, _dptr(volume_native), _dptr(volume), _stream(stream)),
               "wfbp_thicken", self._h)

    def run(self, raw, volume, stream=None):
        _check(self._lib.wfbp_run(self._h, _dptr(raw), _dptr(volume), _stream(stream)), "wfbp_run", self._h)

    def run_timed(self, raw, volume, stream=None):
        """wfbp_run with per-stage device times: {rebin, filter, backproject, thicken} in ms."""
        ms = (C.c_float * 4)()
        _check(self._lib.wfbp_run_timed(self._h, _dptr(raw), _dptr(volume), _stream(stream), ms), "wfbp_run_timed",
               self._h)
        return dict(zip(("rebin", "filter", "backproject", "thicken"), list(ms)))

    def run_static(self, raw, volume, stream=None):
        """wfbp_run with the intermediates in the library's static device
        array (no allocation; small geometries only)."""
        _check(self._lib.wfbp_run_static(self._h, _dptr(raw), _dptr(volume), _stream(stream)), "wfbp_run_static",
               self._h)

    def run_host(self, raw_host, volume_host=None, stream=None):
        """raw_host: float32 array (numpy or pinned torch CPU tensor); returns the volume."""
        import torch
        d = self.dims
        shape = (d.n_slices_requested, d.ny, d.nx)
        if volume_host is None:
            volume_host = np.zeros(shape, np.float32)
        rp = raw_host.data_ptr() if isinstance(raw_host, torch.Tensor) else raw_host.ctypes.data
        vp = volume_host.data_ptr() if isinstance(volume_host, torch.Tensor) else volume_host.ctypes.data
        _check(self._lib.wfbp_run_host(self._h, C.c_void_p(rp), C.c_void_p(vp), _stream(stream)), "wfbp_run_host",
               self._h)
        return volume_host

    # ---- adjoints (FP32 form; reference-layout FP32 buffers) ----
    def set_taps(self, taps, stream=None):
        """Overwrites h[0..n-1] of the filter's half taps (CUDA float32 tensor)."""
        _check(self._lib.wfbp_set_taps(self._h, _dptr(taps), int(taps.numel()), _stream(stream)), "wfbp_set_taps",
               self._h)

    def get_taps(self, stream=None):
        import torch
        out = torch.empty(self.dims.n_channels, dtype=torch.float32, device=torch.device("cuda", self.device))
        _check(self._lib.wfbp_get_taps(self._h, _dptr(out), _stream(stream)), "wfbp_get_taps", self._h)
        return out

    def thicken_adjoint(self, g_volume, g_native, stream=None):
        _check(self._lib.wfbp_thicken_adjoint(self._h, _dptr(g_volume), _dptr(g_native), _stream(stream)),
               "wfbp_thicken_adjoint", self._h)

    def backproject_adjoint(self, g_native, g_filtered, stream=None):
        _check(self._lib.wfbp_backproject_adjoint(self._h, _dptr(g_native), _dptr(g_filtered), _stream(stream)),
               "wfbp_backproject_adjoint", self._h)

    def filter_adjoint(self, g_filtered, g_rebinned, stream=None):
        _check(self._lib.wfbp_filter_adjoint(self._h, _dptr(g_filtered), _dptr(g_rebinned), _stream(stream)),
               "wfbp_filter_adjoint", self._h)

    def rebin_adjoint(self, g_rebinned, g_raw, stream=None):
        _check(self._lib.wfbp_rebin_adjoint(self._h, _dptr(g_rebinned), _dptr(g_raw), _stream(stream)),
               "wfbp_rebin_adjoint", self._h)

    def taps_gradient(self, raw, g_filtered, g_taps, stream=None):
        _check(self._lib.wfbp_taps_gradient(self._h, _dptr(raw), _dptr(g_filtered), _dptr(g_taps),
                                            int(g_taps.numel()), _stream(stream)), "wfbp_taps_gradient", self._h)

    # ---- allocation helpers ----
    def alloc(self, what, device=None):
        import torch
        dev = torch.device("cuda", self.device if device is None else device)
        d = self.dims
        if what == "raw":
            return torch.empty((d.n_readings, d.raw_rows, d.raw_channels), dtype=torch.float32, device=dev)
        if what == "rebinned":
            return torch.empty((d.rebinned_bytes + 3) // 4, dtype=torch.float32, device=dev)
        if what == "filtered":
            if self.ext.filtered_layout == T.LAYOUT_BACKPROJECTION:
                return torch.empty(d.filtered_bytes // 4, dtype=torch.float32, device=dev)
            if d.precision == 1:
                return torch.empty((d.n_views, d.n_rows, d.n_channels), dtype=torch.float16, device=dev)
            return torch.empty((d.n_views, d.n_rows, d.n_channels), dtype=torch.float32, device=dev)
        if what == "row_scales":
            return torch.empty(max(d.row_scale_bytes // 4, 1), dtype=torch.float32, device=dev)
        if what == "native":
            return torch.empty((d.n_slices_native, d.ny, d.nx), dtype=torch.float32, device=dev)
        if what == "volume":
            return torch.empty((d.n_slices_requested, d.ny, d.nx), dtype=torch.float32, device=dev)
        raise ValueError(what)


def parse_recon_config(path):
    """fct_wfbp's recon-parameter YAML file -> ReconConfig."""
    rp = T.ReconConfig()
    _check(load().wfbp_parse_recon_config(os.fsencode(path), C.byref(rp)), "wfbp_parse_recon_config " + str(path))
    return rp


def read_meta(directory):
    """meta.yaml of a FreeCT scan directory -> wfbp_scan_meta."""
    m = T.ScanMeta()
    _check(load().wfbp_read_meta(os.fsencode(directory), C.byref(m)), "wfbp_read_meta " + str(directory))
    return m


def read_frames(directory, meta, first=0, count=None, out=None):
    """Readings [first, first+count) of projections.dat: (tube angles, table
    positions, raw [count][rows][channels]) as float32 arrays. `out` may be a
    (pinned) float32 torch CPU tensor or numpy array for the raw frames."""
    count = meta.total_num_projections - first if count is None else count
    tube = np.zeros(count, np.float32)
    table = np.zeros(count, np.float32)
    shape = (count, meta.detector_rows, meta.detector_channels)
    if out is None:
        out = np.zeros(shape, np.float32)
    ptr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
    _check(load().wfbp_read_frames(os.fsencode(directory), C.byref(meta), int(first), int(count),
                                   tube.ctypes.data_as(_VP), table.ctypes.data_as(_VP), C.c_void_p(ptr)),
           "wfbp_read_frames " + str(directory))
    return tube, table, out


def dicom_read_meta(directory):
    """Scan metadata of a DICOM-CT-PD directory (wfbp_dicom_read_meta)."""
    m = T.ScanMeta()
    _check(load().wfbp_dicom_read_meta(directory.encode(), C.byref(m)), "wfbp_dicom_read_meta")
    return m


def dicom_read_frames(directory, meta, first=0, count=None):
    """Readings [first, first + count) of a DICOM-CT-PD directory:
    (tube angles, table positions, raw [count][rows][channels])."""
    count = meta.total_num_projections - first if count is None else count
    raw = np.zeros((count, meta.detector_rows, meta.detector_channels), np.float32)
    ang = np.zeros(count, np.float32)
    z = np.zeros(count, np.float32)
    _check(load().wfbp_dicom_read_frames(directory.encode(), C.byref(meta), first, count, _fptr(ang)[1], _fptr(z)[1],
                                         _fptr(raw)[1]), "wfbp_dicom_read_frames")
    return ang, z, raw


def write_scan(directory, meta, tube_angles, table_positions, raw):
    t, _ = _fptr(tube_angles)
    z, _ = _fptr(table_positions)
    r = np.ascontiguousarray(raw, dtype=np.float32)
    _check(load().wfbp_write_scan(os.fsencode(directory), C.byref(meta), t.ctypes.data_as(_VP),
                                  z.ctypes.data_as(_VP), r.ctypes.data_as(_VP)), "wfbp_write_scan " + str(directory))


class Batch:
    """Several scans reconstructed together (wfbp_batch): per-scan rebin and
    filter, one persistent backprojection launch over all scans, per-scan
    thickening, captured into a CUDA graph and replayed."""

    def __init__(self, contexts):
        self._lib = load()
        self.contexts = list(contexts)  # the contexts must outlive the batch
        arr = (_VP * len(self.contexts))(*[c.handle.value for c in self.contexts])
        self._h = C.c_void_p()
        st = self._lib.wfbp_batch_create(arr, len(self.contexts), C.byref(self._h))
        if st != 0:
            raise WfbpError(st, "wfbp_batch_create")

    def _check(self, st, what):
        if st != 0:
            m = self._lib.wfbp_batch_last_error(self._h)
            raise WfbpError(st, what + (": " + m.decode() if m else ""))

    def close(self):
        if self._h:
            self._lib.wfbp_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def size(self):
        a, b = C.c_int(), C.c_int()
        self._check(self._lib.wfbp_batch_size(self._h, C.byref(a), C.byref(b)), "wfbp_batch_size")
        return a.value, b.value

    def run(self, raws, volumes, stream=None):
        n = len(self.contexts)
        if len(raws) != n or len(volumes) != n:
            raise ValueError("need one raw and one volume tensor per scan")
        ra = (_VP * n)(*[_dptr(r).value for r in raws])
        va = (_VP * n)(*[_dptr(v).value for v in volumes])
        self._check(self._lib.wfbp_batch_run(self._h, ra, va, _stream(stream)), "wfbp_batch_run")

    def run_host(self, raws_host, volumes_host, stream=None):
        """wfbp_batch_run_host: raws_host / volumes_host are float32 host tensors
        or arrays (pinned torch tensors overlap the copies with the work)."""
        import torch
        n = len(self.contexts)
        if len(raws_host) != n or len(volumes_host) != n:
            raise ValueError("need one raw and one volume buffer per scan")

        def ptr(a):
            return a.data_ptr() if isinstance(a, torch.Tensor) else a.ctypes.data
        ra = (_VP * n)(*[ptr(r) for r in raws_host])
        va = (_VP * n)(*[ptr(v) for v in volumes_host])
        self._check(self._lib.wfbp_batch_run_host(self._h, ra, va, _stream(stream)), "wfbp_batch_run_host")

    def bp_configs(self):
        n = C.c_int()
        self._check(self._lib.wfbp_batch_bp_configs(self._h, None, 0, C.byref(n)), "wfbp_batch_bp_configs")
        arr = (T.BpConfig * max(n.value, 1))()
        self._check(self._lib.wfbp_batch_bp_configs(self._h, arr, n.value, C.byref(n)), "wfbp_batch_bp_configs")
        return [arr[i] for i in range(n.value)]

    def bp_config(self):
        c = T.BpConfig()
        self._check(self._lib.wfbp_batch_get_bp_config(self._h, C.byref(c)), "wfbp_batch_get_bp_config")
        return c

    def set_bp_config(self, config):
        if isinstance(config, (tuple, list)):
            c = T.BpConfig()
            c.tile_x, c.tile_y, c.cols_per_step = config[:3]
            c.consumer_warps = config[3] if len(config) > 3 else 0
            c.slab = config[4] if len(config) > 4 else 0
            config = c
        self._check(self._lib.wfbp_batch_set_bp_config(self._h, C.byref(config)), "wfbp_batch_set_bp_config")

    def check_device_status(self):
        self._check(self._lib.wfbp_batch_check_device_status(self._h), "wfbp_batch_check_device_status")


def synth_project(scan, ellipsoids, out, stream=None):
    """Line integrals (+ noise) of an ellipsoid phantom into out (CUDA float32)."""
    arr = (T.Ellipsoid * max(len(ellipsoids), 1))()
    for i, e in enumerate(ellipsoids):
        arr[i] = e
    _check(load().wfbp_synth_project(C.byref(scan), arr, len(ellipsoids), _dptr(out), _stream(stream)),
           "wfbp_synth_project")
