"""Frame sharding over ranks (one process per GPU).

Decoding is independent per frame: a batch splits into contiguous frame ranges, one
per rank, with no exchange on the data path.  These helpers give each rank its range
of a global batch, share a mix of decode jobs among ranks by estimated cost
(`partition_jobs`, `frame_cost`), and combine per-rank timings as the slowest
rank's (the job is done when the last rank is).  Collectives appear only for that timing reduction and for
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


# Device time per unit of decode work on one B200, from the bench workloads: an LDPC
# edge-iteration (each check-to-bit message read and written once by the check pass
# and read by the bit pass) with FP32, FP16 (packed) and int8 messages -- DVB-S2
# normal frames, 3 rates x 512, 67.7 / 44.3 / 58.7 ms for 9.98 G edge-iterations --
# and a trellis step of the windowed LTE turbo decoder (1024 frames of K = 6144,
# 6 iterations: 1.64 ms for 75.5 M steps).
PS_PER_EDGE_ITERATION = {0: 6.8, 1: 4.4, 2: 5.9}
PS_PER_TRELLIS_STEP = 21.7


def frame_cost(codec) -> float:
    """Estimated device seconds to decode one frame of `codec` running all its
    iterations: E x I for LDPC (E = stateSize, the edge count) and, for turbo codes,
    the trellis steps of one iteration over all constituents (stateSize, 2 (K + 3)
    for LTE) x I, each times its measured per-unit time.  Convolutional codes take
    one pass over their message.  Early stops make real decodes cheaper; the
    estimate is for balancing work between ranks, not for timing."""
    from . import Convolutional, Ldpc, Turbo
    if isinstance(codec, Ldpc):
        d = codec.getDecoderOptions()
        return codec.stateSize() * d.iterations() * PS_PER_EDGE_ITERATION.get(d.precision(), 6.8) * 1e-12
    if isinstance(codec, Turbo):
        return codec.stateSize() * codec.getDecoderOptions().iterations() * PS_PER_TRELLIS_STEP * 1e-12
    if isinstance(codec, Convolutional):
        return codec.msgSize() * PS_PER_TRELLIS_STEP * 1e-12
    raise TypeError("frame_cost: not a codec")


def partition_jobs(jobs, world: int, align: int = LANE_FRAMES):
    """Share the frames of several decode jobs among `world` ranks by estimated cost.

    jobs: a sequence of (cost per frame, frame count).  Each job is cut into chunks of
    `align` frames (one lane batch of the LDPC kernels; a job's last chunk may be
    short), and chunks go, costliest first, to the rank with the least work so far
    (the longest-processing-time rule; ties go to the lower rank, then to the earlier
    job).  The full chunks of a job cost the same, so each rank's count of them is
    then laid out as one contiguous range, the owner of the short chunk last.  The
    result is deterministic, so every rank can compute it alone.

    Returns, per rank, a list of (job index, lo, hi): at most one frame range [lo, hi)
    per job.  Every frame of every job is in exactly one range, and the busiest
    rank's estimated cost is at most the average per rank plus one chunk.
    """
    if world <= 0 or align <= 0:
        raise ValueError("world and align must be > 0")
    chunks = []
    for j, (cost, n) in enumerate(jobs):
        if n < 0 or cost < 0:
            raise ValueError("job %d: frame count and cost must be >= 0" % j)
        for lo in range(0, int(n), align):
            hi = min(int(n), lo + align)
            chunks.append((-(cost * (hi - lo)), j, lo, hi))
    chunks.sort()
    load = [0.0] * world
    full = [[0] * len(jobs) for _ in range(world)]
    short_owner = {}
    for neg_cost, j, lo, hi in chunks:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] -= neg_cost
        if hi - lo < align:
            short_owner[j] = r
        else:
            full[r][j] += 1
    parts = [[] for _ in range(world)]
    for j, (_, n) in enumerate(jobs):
        s_r = short_owner.get(j)
        order = [r for r in range(world) if r != s_r] + ([s_r] if s_r is not None else [])
        lo = 0
        for r in order:
            k = full[r][j] + (1 if r == s_r else 0)
            hi = min(int(n), lo + k * align)
            if hi > lo:
                parts[r].append((j, lo, hi))
            lo = hi
    return parts
