"""Frame sharding across ranks (world_size 2, gloo on CPU).

Each rank filters only its shard of a clip -- with the CPU oracle standing in for the GPU, which
this host does not have -- and the assembled result must equal the unsharded run: Basic frames
need no neighbours; VBasic -> VAggregate shards recompute a halo of stacked frames.  The ranks
exchange only the timing reduction (max over ranks), as bench.py does.
"""
import os
import socket

import numpy as np
import pytest

from bm3d_b200 import shard, synth

R = 1            # V-BM3D radius of the test
NF = 5           # frames in the clip (odd: the shards differ in size)
H, W = 24, 32


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _clip():
    nz, _ = synth.gray_frames(41, NF, H, W, 15.0)
    return nz


def _worker(rank, world, port, outdir):
    import datetime
    import torch
    import torch.distributed as dist
    import oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        clip = _clip()
        # Basic: frames are independent
        first, count = shard.frame_range(NF, rank, world)
        pb = oracle.default_params(0, False, "fast", 15.0, width=W, height=H)
        basic = oracle.bm3d(pb, clip[first:first + count])
        # VBasic -> VAggregate with a halo
        rg = shard.vbm3d_ranges(NF, rank, world, R)
        r0, rn = rg["read"]
        s0, sn = rg["stack"]
        pv = oracle.default_params(0, True, "fast", 15.0, width=W, height=H, radius=R)
        stacks = oracle.vbm3d(pv, clip[r0:r0 + rn], n0=s0 - r0, count=sn)
        agg = oracle.vaggregate(R, stacks)[first - s0:first - s0 + count]
        np.save(os.path.join(outdir, f"basic{rank}.npy"), basic)
        np.save(os.path.join(outdir, f"vagg{rank}.npy"), agg)
        # the only collective: max over ranks of a per-rank time
        t = torch.tensor([float(rank + 1)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        np.save(os.path.join(outdir, f"tmax{rank}.npy"), t.numpy())
    finally:
        dist.destroy_process_group()


def test_frame_range_partitions_the_clip():
    for n in range(0, 23):
        for world in range(1, 9):
            got = [shard.frame_range(n, r, world) for r in range(world)]
            assert sum(c for _, c in got) == n
            pos = 0
            for f, c in got:
                assert f == pos
                pos += c
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        shard.frame_range(4, 2, 2)


def test_vbm3d_ranges_cover_the_windows():
    for n in range(1, 15):
        for world in range(1, 5):
            for r in range(1, 4):
                for rank in range(world):
                    g = shard.vbm3d_ranges(n, rank, world, r)
                    f, c = g["out"]
                    s0, sn = g["stack"]
                    r0, rn = g["read"]
                    for k in range(f, f + c):      # VAggregate reads stacks k-r..k+r
                        assert s0 <= max(0, k - r) and min(n, k + r + 1) <= s0 + sn
                    for k in range(s0, s0 + sn):   # a stack reads inputs k-r..k+r
                        assert r0 <= max(0, k - r) and min(n, k + r + 1) <= r0 + rn


def test_two_rank_gloo_sharding_matches_unsharded(tmp_path):
    import torch.multiprocessing as mp
    import oracle
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    clip = _clip()
    pb = oracle.default_params(0, False, "fast", 15.0, width=W, height=H)
    pv = oracle.default_params(0, True, "fast", 15.0, width=W, height=H, radius=R)
    basic = oracle.bm3d(pb, clip)
    vagg = oracle.vaggregate(R, oracle.vbm3d(pv, clip))
    got_b = np.concatenate([np.load(tmp_path / f"basic{r}.npy") for r in range(world)])
    got_v = np.concatenate([np.load(tmp_path / f"vagg{r}.npy") for r in range(world)])
    assert got_b.shape == basic.shape and np.array_equal(got_b, basic)
    assert got_v.shape == vagg.shape and np.array_equal(got_v, vagg)
    for r in range(world):
        assert float(np.load(tmp_path / f"tmax{r}.npy")[0]) == float(world)
