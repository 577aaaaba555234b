"""Frame sharding over ranks (one process per GPU).

Decoding is independent per frame: a batch splits into contiguous frame ranges, one
per rank, with no exchange on the data path.  These helpers give each rank its range
of a global batch and combine per-rank timings as the slowest rank's (the job is done
when the last rank is).  Collectives appear only for that timing reduction and for
optional gathers a caller asks for; the decode itself never waits on another rank.
"""
from __future__ import annotations

LANE_FRAMES = 32  # frames one warp of the lane-batched LDPC kernel carries


def frame_range(nframes: int, rank: int, world: int, align: int = LANE_FRAMES) -> tuple[int, int]:
    """[lo, hi) of the frames rank `rank` of `world` decodes.

    Ranges are contiguous, cover [0, nframes) exactly once, and start on multiples
    of `align` (so every rank but the last fills whole lane batches); sizes differ
    by at most `align` frames.
    """
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank %d outside world of %d" % (rank, world))
    if nframes < 0 or align <= 0:
        raise ValueError("nframes must be >= 0 and align > 0")
    units = -(-nframes // align)
    base, extra = divmod(units, world)
    # the last `extra` ranks take one unit more; the last rank also holds the ragged
    # final unit, so no two ranks differ by more than `align` frames
    first_big = world - extra
    lo_u = rank * base + max(0, rank - first_big)
    hi_u = lo_u + base + (1 if rank >= first_big else 0)
    return min(lo_u * align, nframes), min(hi_u * align, nframes)


def shard(array, nframes: int, rank: int, world: int, align: int = LANE_FRAMES):
    """The rows of `array` (frame-major, flattened or [nframes][...]) this rank owns."""
    lo, hi = frame_range(nframes, rank, world, align)
    per = array.shape[0] // nframes if array.ndim == 1 and nframes else None
    if per is not None:
        return array[lo * per:hi * per]
    return array[lo:hi]


def decode_shard(codec, llr, nframes: int, rank: int, world: int, out=None):
    """Decode this rank's frames of a global batch `llr` ([nframes * paritySize]).

    Returns the decoded bits of frames frame_range(nframes, rank, world); no
    collective is involved.
    """
    part = shard(llr, nframes, rank, world)
    return codec.decode(part, out=out) if out is not None else codec.decode(part)


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (a time: the job's time is its slowest rank's)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
