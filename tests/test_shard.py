"""Z-slab sharding (freect_b200.shard): the plans, and the sharded path run
as two gloo ranks on CPU with the FP64 oracle as the per-rank engine, its
slabs gathered to rank 0 and compared with the whole-scan reconstruction
(bit-identical: each voxel sums the same views in the same order)."""
import os
import socket

import numpy as np
import pytest

from freect_b200 import abi_types as T
from freect_b200 import scans, shard, wfbp

torch = pytest.importorskip("torch")


def _geometry(spec):
    tube, table = spec.views()
    cg, gp = wfbp.configure_geometry(spec.meta(), table)
    return cg, spec.recon_config(), tube, table


def test_effective_geometry_matches_oracle(orc):
    for mode in (T.FFS_NONE, T.FFS_PHI, T.FFS_Z, T.FFS_PHIZ):
        spec = scans.tiny_ffs(mode=mode)
        tube, table = spec.views()
        cg, _ = wfbp.configure_geometry(spec.meta(), table)
        eff = wfbp.effective_geometry(cg)
        assert bytes(eff) == (bytes(cg) if mode == T.FFS_NONE else bytes(orc.ffs_effective(cg)))


@pytest.mark.parametrize("name", ["tiny", "small", "rows64", "ffs"])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_plan_covers_and_aligns(name, world):
    spec = scans.WORKLOADS[name]()
    cg, rp, tube, table = _geometry(spec)
    nat, req = wfbp.slice_locations(wfbp.effective_geometry(cg), rp)
    if world > req.size:
        pytest.skip("fewer slices than ranks")
    plans = shard.plan(cg, rp, table, world)
    G = shard._readings_per_view(cg)
    V, P = int(cg.total_number_of_projections) // G, int(cg.projections_per_rotation) // G
    P2 = P // 2
    K = V // P2
    zv = np.asarray(table, np.float32)[::G][:V]
    assert [p.requested for p in plans][0][0] == 0 and plans[-1].requested[1] == req.size
    for a, b in zip(plans, plans[1:]):
        assert a.requested[1] == b.requested[0]
    reach = shard.rebin_reach(cg) // G
    for p in plans:
        r0, r1 = p.requested
        n0, n1 = p.native
        v0, v1 = p.views
        assert p.readings == (v0 * G, v1 * G)
        # every native slice the slab's thickening weights reach is inside
        w = np.abs(nat[:, None] - req[None, r0:r1]) < rp.slice_thickness
        assert not w[:n0].any() and not w[n1:].any()
        # half-turn aligned window, more than one rotation, inside the whole scan's used views
        assert v0 % P2 == 0 and v1 - v0 > P and v1 <= V
        Ks = (v1 - v0) // P2
        assert v0 + Ks * P2 <= K * P2
        # every view within z_rot of the slab is read by the window's backprojection,
        # with the rebin's reach inside the window too
        zlo, zhi = nat[n0:n1].min(), nat[n0:n1].max()
        need = np.nonzero((zv[:K * P2] >= zlo - cg.z_rot) & (zv[:K * P2] <= zhi + cg.z_rot))[0]
        assert need[0] - v0 >= min(reach, need[0]) and need[-1] < v0 + Ks * P2
        assert v1 - 1 - need[-1] >= min(reach, V - 1 - need[-1])


def _oracle_slab(orc, cg, rp, tube, table, raw, p, window=T.FILTER_REFERENCE):
    """The slab of plan p through the FP64 oracle, from the window's readings only."""
    a0, a1 = p.readings
    ce = orc.ffs_effective(cg) if (cg.ffs_phi or cg.ffs_z) else cg
    nat, req = orc.slice_locations(ce, rp)
    return orc.reconstruct_window_f64(shard.sub_geometry(cg, p), rp, window, tube[a0:a1], table[a0:a1], raw[a0:a1],
                                      a0, nat[p.native[0]:p.native[1]], req[p.requested[0]:p.requested[1]])


def _rank_main(rank, world, port, result_path):
    import torch.distributed as dist
    from oracle import oracle as orc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        spec = scans.tiny(nch=64, nr=6, P=96, rotations=5, nx=24, n_slices=9)
        cg, rp, tube, table = _geometry(spec)
        raw = orc.synth_project(spec.synth(), spec.ellipsoids())
        plans = shard.plan(cg, rp, table, world)
        slab = torch.from_numpy(_oracle_slab(orc, cg, rp, tube, table, raw, plans[rank]).copy())
        whole = shard.gather_slabs(slab, plans, rank)
        if rank == 0:
            np.save(result_path, whole.numpy())
    finally:
        dist.destroy_process_group()


def test_sharded_oracle_two_ranks_matches_whole(orc, tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "whole.npy")
    mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
    got = np.load(out)
    spec = scans.tiny(nch=64, nr=6, P=96, rotations=5, nx=24, n_slices=9)
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    ref = orc.reconstruct_f64(spec, raw)["volume"]
    assert got.shape == ref.shape
    assert np.array_equal(got, ref, equal_nan=True)
    assert np.isfinite(ref).mean() > 0.5
    # and the plans of 3 ranks, run in one process, stitch to the same volume
    cg, rp, tube, table = _geometry(spec)
    parts = [_oracle_slab(orc, cg, rp, tube, table, raw, p) for p in shard.plan(cg, rp, table, 3)]
    assert np.array_equal(np.concatenate(parts), ref, equal_nan=True)


def test_sharded_oracle_ffs_matches_whole(orc):
    spec = scans.tiny_ffs(mode=T.FFS_PHIZ, nch=64, nr=4, P=128, rotations=6, nx=32, n_slices=12)
    cg, rp, tube, table = _geometry(spec)
    raw = orc.synth_project(spec.synth(), spec.ellipsoids())
    ref = orc.reconstruct_f64(spec, raw)["volume"]
    for world in (2, 3):
        parts = [_oracle_slab(orc, cg, rp, tube, table, raw, p) for p in shard.plan(cg, rp, table, world)]
        assert np.array_equal(np.concatenate(parts), ref, equal_nan=True), world


def test_assign_scans_whole_and_balanced():
    costs = [5.0, 1.0, 4.0, 2.0, 3.0]
    a = shard.assign_scans(costs, 2)
    assert a == [[0, 1, 3], [2, 4]]  # largest first onto the least-loaded rank
    for world in (1, 3, 4, 7):
        got = shard.assign_scans(costs, world)
        assert sorted(i for r in got for i in r) == list(range(len(costs)))
        loads = [sum(costs[i] for i in r) for r in got]
        assert max(loads) - min(loads) <= max(costs)
    with pytest.raises(ValueError):
        shard.assign_scans(costs, 0)
    # the cost estimate grows with the matrix and the slices
    a = scans.tiny(nch=64, nr=6, P=96, rotations=3, nx=24, n_slices=4)
    b = scans.tiny(nch=64, nr=6, P=96, rotations=3, nx=48, n_slices=8)
    ca = shard.scan_cost(_geometry(a)[0], a.recon_config())
    cb = shard.scan_cost(_geometry(b)[0], b.recon_config())
    assert cb > 4 * ca


def _batch_rank_main(rank, world, port, result_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        costs = [5.0, 1.0, 4.0, 2.0, 3.0]
        shapes = [(2, 3, 4), (1, 2, 2), (3, 3, 3), (2, 2, 5), (1, 4, 4)]
        a = shard.assign_scans(costs, world)
        # this rank's "reconstructions": scan i's volume filled with i
        mine = [torch.full(shapes[i], float(i)) for i in a[rank]]
        got = shard.gather_volumes(mine, a, rank, shapes)
        if rank == 0:
            np.save(result_path, np.concatenate([g.numpy().ravel() for g in got]))
            assert [tuple(g.shape) for g in got] == shapes
    finally:
        dist.destroy_process_group()


def test_batch_sharded_by_scan_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "vols.npy")
    mp.spawn(_batch_rank_main, args=(2, port, out), nprocs=2, join=True)
    got = np.load(out)
    shapes = [(2, 3, 4), (1, 2, 2), (3, 3, 3), (2, 2, 5), (1, 4, 4)]
    ref = np.concatenate([np.full(int(np.prod(s)), float(i), np.float32) for i, s in enumerate(shapes)])
    assert np.array_equal(got, ref)
