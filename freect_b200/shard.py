"""Z-slab sharding of one scan across ranks (one process per GPU).

The reconstruction partitions along z with no exchange on the data path:
a slab of requested slices needs only the native slices its thickening
reads (weights 1 - |dz| / slice_thickness > 0, cuda_kernels.cuh:303-317),
those need only the views whose table position lies within z_rot of them
(the backprojection's z cull, cuda_kernels.cuh:232), and those views need
only the readings the rebin reaches (the fan half-angle, in views, either
side: rebin_kernel, cuda_kernels.cuh:17-36). Each rank therefore
reconstructs its slab from its own window of readings, rebinning and
filtering the window itself (overlapping windows are recomputed, not
exchanged). The window starts on a half-turn boundary and keeps the whole
scan's slice positions (wfbp_set_slices) and z_rot, so every voxel sums the
same views in the same order as a reconstruction of the whole scan: the
stitched slabs equal it bit for bit. The only collective is the optional
gather of the slabs to one rank at the end.

A batch of scans shards by whole scans instead (assign_scans): each rank
reconstructs its scans independently (one persistent batch launch per rank)
and the volumes may be gathered to one rank at the end (gather_volumes).

The reference has no multi-GPU path (ReconstructionMachine runs on one
device, ReconstructionMachine.cu:141-434).
"""
import dataclasses
import math

import numpy as np

from . import abi_types as T
from . import wfbp


@dataclasses.dataclass
class SlabPlan:
    rank: int
    world: int
    requested: tuple  # [r0, r1) requested slice indices
    native: tuple     # [n0, n1) native slice indices
    views: tuple      # [v0, v1) views of the window (effective views with a flying focal spot)
    readings: tuple   # [a0, a1) raw readings of the window

    @property
    def n_requested(self):
        return self.requested[1] - self.requested[0]


def _readings_per_view(cg):
    return (2 if cg.ffs_phi else 1) * (2 if cg.ffs_z else 1)


def rebin_reach(cg):
    """Views the rebin reads either side of a view: the largest |fan angle|
    of a channel over the angular step, rounded up, plus the interpolation."""
    nch = int(cg.num_detector_cols)
    dcol, sdd, c0 = cg.detector_pixel_size_col, cg.distance_source_to_detector, cg.detector_central_col
    beta = max(abs(math.asin(max(-1.0, min(1.0, (c - c0) * dcol / sdd)))) for c in (0, nch - 1))
    return int(math.ceil(beta * cg.projections_per_rotation / (2 * math.pi))) + 2


def plan(cg, rp, table_positions, world):
    """Slab plans for `world` ranks. cg: the scan's CTGeometry
    (wfbp_configure_geometry), rp: its ReconConfig, table_positions: one per
    reading. Requested slices are split into contiguous runs of near-equal
    length."""
    G = _readings_per_view(cg)
    table = np.asarray(table_positions, np.float32)
    # slice lists follow the geometry the stages work on (effective with FFS)
    nat, req = wfbp.slice_locations(wfbp.effective_geometry(cg), rp)
    V = int(cg.total_number_of_projections) // G
    P = int(cg.projections_per_rotation) // G
    P2 = P // 2
    K = V // P2
    zv = table[::G][:V]
    used = K * P2  # views the backprojection of the whole scan reads (cuda_kernels.cuh:230)
    reach = rebin_reach(cg) // G + 2
    if world < 1 or world > req.size:
        raise ValueError("world must be in [1, requested slices]")
    edges = np.linspace(0, req.size, world + 1).round().astype(int)
    out = []
    for r in range(world):
        r0, r1 = int(edges[r]), int(edges[r + 1])
        zr = req[r0:r1]
        w = np.abs(nat[:, None] - zr[None, :]) < rp.slice_thickness
        idx = np.nonzero(w.any(axis=1))[0]
        if idx.size == 0:
            raise ValueError("slab %d has no native slice" % r)
        n0, n1 = int(idx[0]), int(idx[-1]) + 1
        zlo, zhi = float(nat[n0:n1].min()), float(nat[n0:n1].max())
        need = np.nonzero((zv[:used] >= zlo - cg.z_rot) & (zv[:used] <= zhi + cg.z_rot))[0]
        if need.size == 0:
            raise ValueError("slab %d sees no view" % r)
        v0 = max(0, int(need[0]) - reach)
        v0 -= v0 % P2  # the window starts on a half-turn boundary: theta~ = j mod P/2 is kept
        # whole half turns, so that the window's backprojection reads every
        # view up to the last one needed (it reads floor(views / (P/2)) half turns)
        span = max(int(need[-1]) + 1 + reach - v0, P + 1)
        v1 = min(V, v0 + -(-span // P2) * P2)
        out.append(SlabPlan(r, world, (r0, r1), (n0, n1), (v0, v1), (v0 * G, v1 * G)))
    return out


def sub_geometry(cg, p):
    """CTGeometry of a slab's window: the scan's, with the window's reading
    count and the whole scan's z_rot."""
    sub = T.CTGeometry.from_buffer_copy(bytes(cg))
    sub.total_number_of_projections = p.readings[1] - p.readings[0]
    return sub


def slab_context(cg, rp, ext, tube_angles, table_positions, p, device=0):
    """A context that reconstructs slab `p` from the readings of its window."""
    a0, a1 = p.readings
    nat, req = wfbp.slice_locations(wfbp.effective_geometry(cg), rp)
    ctx = wfbp.Context(sub_geometry(cg, p), rp, ext, device=device)
    ctx.set_reading_offset(a0)
    ctx.set_views(np.asarray(tube_angles, np.float32)[a0:a1], np.asarray(table_positions, np.float32)[a0:a1])
    ctx.set_slices(nat[p.native[0]:p.native[1]], req[p.requested[0]:p.requested[1]])
    return ctx


def reconstruct_distributed(cg, rp, ext, tube_angles, table_positions, raw_window, device, gather=True):
    """Reconstructs this rank's slab of one scan (torch.distributed must be
    initialised; one process per GPU). raw_window(a0, a1) returns the device
    tensor of readings [a0, a1). Returns the slab, and on rank 0 with
    gather=True the whole volume (other ranks: None)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(), dist.get_world_size()
    plans = plan(cg, rp, table_positions, world)
    p = plans[rank]
    ctx = slab_context(cg, rp, ext, tube_angles, table_positions, p, device=device)
    slab = ctx.alloc("volume")
    ctx.run(raw_window(*p.readings), slab)
    ctx.close()
    if not gather:
        return slab, None
    return slab, gather_slabs(slab, plans, rank)


def gather_slabs(slab, plans, rank, dst=0):
    """Collects the slabs on rank `dst` (point-to-point, the only exchange):
    returns the whole [nz][ny][nx] volume there, None elsewhere."""
    import torch
    import torch.distributed as dist
    if rank != dst:
        dist.send(slab.contiguous(), dst)
        return None
    parts = []
    for p in plans:
        if p.rank == dst:
            parts.append(slab)
            continue
        buf = torch.empty((p.n_requested,) + tuple(slab.shape[1:]), dtype=slab.dtype, device=slab.device)
        dist.recv(buf, p.rank)
        parts.append(buf)
    return torch.cat(parts, dim=0)


def scan_cost(cg, rp):
    """Relative cost of reconstructing one scan: voxel columns x native slices x
    views per rotation (a voxel of a slice collects about one rotation of
    contributing views), the estimate the batch planner also sorts by."""
    nat, _ = wfbp.slice_locations(wfbp.effective_geometry(cg), rp)
    P = int(cg.projections_per_rotation) // _readings_per_view(cg)
    return float(rp.nx) * float(rp.ny) * float(nat.size) * float(P)


def assign_scans(costs, world):
    """Whole scans to `world` ranks: largest estimated cost first, each onto the
    rank with the least total so far (ties to the lower rank). Deterministic, so
    every rank computes the same assignment. Returns one ascending list of scan
    indices per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(costs[i])
    return [sorted(a) for a in out]


def gather_volumes(volumes, assignment, rank, shapes, dst=0, dtype=None, device=None):
    """Collects the volumes of a batch on rank `dst` (point-to-point). volumes:
    this rank's volumes in the order of assignment[rank]; shapes: the shape of
    every scan's volume; dtype / device of the receive buffers (default: those
    of this rank's first volume, else float32 on the CPU). Returns the list of
    all volumes in scan order on dst, None elsewhere."""
    import torch
    import torch.distributed as dist
    if dtype is None:
        dtype = volumes[0].dtype if volumes else torch.float32
    if device is None:
        device = volumes[0].device if volumes else "cpu"
    if rank != dst:
        for v in volumes:
            dist.send(v.contiguous(), dst)
        return None
    mine = dict(zip(assignment[dst], volumes))
    out = [None] * len(shapes)
    for r, scans_r in enumerate(assignment):
        for i in scans_r:
            if r == dst:
                out[i] = mine[i]
                continue
            buf = torch.empty(tuple(shapes[i]), dtype=dtype, device=device)
            dist.recv(buf, r)
            out[i] = buf
    return out
