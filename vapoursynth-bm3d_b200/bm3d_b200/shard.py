"""Frame sharding of a clip across processes, one process per GPU.

BM3D Basic/Final frames are independent (the reference registers them rpStrictSpatial,
source/VSPlugin.cpp:175-177), so a clip splits into contiguous frame ranges with no exchange
between ranks.  V-BM3D reads +-radius neighbour frames (source/VBM3D_Base.cpp:540-659) and
VAggregate reads the +-radius stacked outputs around each frame (source/VAggregate.cpp:93-160), so
a V-BM3D shard also computes a halo: stacks for `radius` frames on each side of its range, which
need input frames `2 * radius` beyond it.  Halo frames are recomputed locally -- replicas only, no
collective on the data path.
"""


def frame_range(num_frames, rank, world):
    """Contiguous [first, first + count) of frames for `rank`; the first num_frames % world ranks
    take one extra frame."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(num_frames, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def vbm3d_ranges(num_frames, rank, world, radius):
    """Ranges a V-BM3D -> VAggregate shard touches, as (first, count) pairs:
    out:   frames whose VAggregate output this rank produces;
    stack: frames whose VBasic/VFinal stacked output it computes (out +- radius, clipped);
    read:  input frames it reads (stack +- radius, clipped)."""
    first, count = frame_range(num_frames, rank, world)
    s0 = max(0, first - radius)
    s1 = min(num_frames, first + count + radius)
    r0 = max(0, s0 - radius)
    r1 = min(num_frames, s1 + radius)
    return {"out": (first, count), "stack": (s0, s1 - s0), "read": (r0, r1 - r0)}
