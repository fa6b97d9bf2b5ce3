"""Differentiable WFBP: a torch.autograd.Function over the C ABI.

The forward pass is the FP32 form's four stages (wfbp_rebin, wfbp_filter,
wfbp_backproject, wfbp_thicken, exact texel weights; the TMA-staged
backprojection in the backprojection layout where the geometry allows it);
the backward pass runs their hand-written adjoint kernels in reverse
(wfbp_thicken_adjoint, wfbp_backproject_adjoint, wfbp_filter_adjoint,
wfbp_rebin_adjoint) and, for the learnable filter taps,
wfbp_taps_gradient, which recomputes the rebinned rows from the saved raw
readings inside its kernel: only the raw readings and the taps are saved
between the passes, not the rebinned or filtered data.

The reference (fct_wfbp) has no backward pass; the forward it
differentiates is ReconstructionMachine::RunReconstruction
(ReconstructionMachine.cu:141-434).

    rec = Reconstructor(cg, rp, tube_angles, table_positions, n_taps=64)
    taps = torch.nn.Parameter(rec.initial_taps())
    vol = rec(raw, taps)            # raw: [B][readings][rows][channels] or one scan
    loss = ((vol - target)[torch.isfinite(vol)] ** 2).mean()
    loss.backward()                 # raw.grad (if it requires grad), taps.grad
"""
import torch

from . import abi_types as T
from . import wfbp


class Reconstructor:
    """One scan geometry on one device, FP32 form, with `n_taps` learnable
    taps h[0..n_taps-1] of the symmetric filter (the rest stay fixed)."""

    def __init__(self, cg, rp, tube_angles, table_positions, n_taps=64, filter_window=T.FILTER_REFERENCE,
                 device=0):
        ext = wfbp.make_ext(precision=T.PRECISION_FP32, filter_window=filter_window, tex_weights=0,
                            filtered_layout=T.LAYOUT_BACKPROJECTION)
        self.ctx = wfbp.Context(cg, rp, ext, device=device)
        self.ctx.set_views(tube_angles, table_positions)
        try:
            self.ctx.bp_config()
        except wfbp.WfbpError:  # no TMA launch fits: the reference layout and the generic kernel
            ext = wfbp.make_ext(precision=T.PRECISION_FP32, filter_window=filter_window, tex_weights=0,
                                filtered_layout=T.LAYOUT_REFERENCE)
            self.ctx = wfbp.Context(cg, rp, ext, device=device)
            self.ctx.set_views(tube_angles, table_positions)
        self.device = torch.device("cuda", device)
        self.n_taps = int(n_taps)
        if not 1 <= self.n_taps <= self.ctx.dims.n_channels:
            raise ValueError("n_taps must be in [1, channels]")
        self.base_taps = self.ctx.get_taps()
        torch.cuda.synchronize(self.device)
        d = self.ctx.dims
        self.raw_shape = (d.n_readings, d.raw_rows, d.raw_channels)
        self._buf = {}

    def initial_taps(self):
        """The context's filter taps h[0..n_taps-1] (the ramp of its window)."""
        return self.base_taps[: self.n_taps].clone()

    def buf(self, name):
        """Per-reconstructor scratch: rebinned / gradient rows [V][nr][nch], the
        forward's filtered rows (context layout), native volume."""
        if name not in self._buf:
            d = self.ctx.dims
            if name == "filtered":
                self._buf[name] = self.ctx.alloc("filtered")
                return self._buf[name]
            if name in ("rebinned", "rows"):
                shape = (d.n_views, d.n_rows, d.n_channels)
            elif name == "native":
                shape = (d.n_slices_native, d.ny, d.nx)
            else:
                raise ValueError(name)
            self._buf[name] = torch.empty(shape, dtype=torch.float32, device=self.device)
        return self._buf[name]

    def __call__(self, raw, taps, ready=None):
        """ready: optional list of CUDA events, one per scan of a batched raw;
        the forward waits for event b before it reads scan b (so the caller can
        copy the scans in on another stream while earlier ones reconstruct)."""
        return WFBPFunction.apply(raw, taps, self, ready)


class WFBPFunction(torch.autograd.Function):
    """vol = WFBP(raw; taps). raw: float32 CUDA [B][readings][rows][channels]
    or [readings][rows][channels]; taps: float32 CUDA [n_taps]."""

    @staticmethod
    def forward(fctx, raw, taps, rec, ready=None):
        if raw.dtype != torch.float32 or taps.dtype != torch.float32:
            raise TypeError("raw and taps must be float32")
        batched = raw.dim() == 4
        rb = raw if batched else raw.unsqueeze(0)
        if tuple(rb.shape[1:]) != rec.raw_shape:
            raise ValueError("raw shape %s does not match the geometry %s" % (tuple(rb.shape[1:]), rec.raw_shape))
        if taps.numel() != rec.n_taps:
            raise ValueError("expected %d taps" % rec.n_taps)
        rb = rb.contiguous()
        ctx = rec.ctx
        ctx.set_taps(taps.detach().contiguous())
        d = ctx.dims
        out = torch.empty((rb.shape[0], d.n_slices_requested, d.ny, d.nx), dtype=torch.float32, device=raw.device)
        reb, filt, vn = rec.buf("rebinned"), rec.buf("filtered"), rec.buf("native")
        if ready is not None and len(ready) != rb.shape[0]:
            raise ValueError("need one ready event per scan")
        for b in range(rb.shape[0]):
            if ready is not None:
                torch.cuda.current_stream(raw.device).wait_event(ready[b])
            ctx.rebin(rb[b], reb)
            ctx.filter(reb, filt)
            ctx.backproject(filt, vn)
            ctx.thicken(vn, out[b])
        fctx.rec = rec
        fctx.batched = batched
        fctx.save_for_backward(rb, taps)
        return out if batched else out[0]

    @staticmethod
    def backward(fctx, g):
        rb, taps = fctx.saved_tensors
        rec = fctx.rec
        ctx = rec.ctx
        need_raw, need_taps = fctx.needs_input_grad[0], fctx.needs_input_grad[1]
        gb = (g if fctx.batched else g.unsqueeze(0)).contiguous()
        ctx.set_taps(taps.detach().contiguous())
        g_raw = torch.empty_like(rb) if need_raw else None
        g_taps = torch.zeros_like(taps) if need_taps else None
        t_b = torch.empty_like(taps) if need_taps else None
        gvn, gf, gr = rec.buf("native"), rec.buf("rows"), rec.buf("rebinned")
        for b in range(rb.shape[0]):
            ctx.thicken_adjoint(gb[b], gvn)
            ctx.backproject_adjoint(gvn, gf)
            if need_raw:
                ctx.filter_adjoint(gf, gr)
                ctx.rebin_adjoint(gr, g_raw[b])
            if need_taps:
                ctx.taps_gradient(rb[b], gf, t_b)
                g_taps += t_b
        if need_raw and not fctx.batched:
            g_raw = g_raw[0]
        return g_raw, g_taps, None, None
