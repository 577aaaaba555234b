"""Frame sharding over ranks: ranges cover a batch exactly once, and a 2-rank gloo job
that encodes its shards and gathers them reproduces the whole-batch result; the
timing reduction takes the slowest rank.  CPU only (gloo); the GPU decode path of
each rank is the single-GPU decode the other tests cover."""
import os
import socket

import numpy as np
import pytest

from fecl_b200.shard import frame_range


@pytest.mark.parametrize("nframes", [0, 1, 31, 32, 33, 100, 1024, 4097])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_frame_ranges_partition_the_batch(nframes, world):
    seen = np.zeros(nframes, np.int32)
    sizes = []
    prev_hi = 0
    for r in range(world):
        lo, hi = frame_range(nframes, r, world)
        assert lo == prev_hi and lo <= hi
        assert lo % 32 == 0 or lo == nframes
        seen[lo:hi] += 1
        sizes.append(hi - lo)
        prev_hi = hi
    assert prev_hi == nframes and np.all(seen == 1)
    assert max(sizes) - min(sizes) <= 32


def test_frame_range_rejects_bad_rank():
    with pytest.raises(ValueError):
        frame_range(10, 2, 2)
    with pytest.raises(ValueError):
        frame_range(10, 0, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nframes, result_path):
    import datetime

    import torch.distributed as dist

    import fecl_b200 as F
    from fecl_b200.shard import frame_range, max_over_ranks, shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        code = F.Turbo.lte(256)
        rng = np.random.default_rng(5)
        msg = rng.integers(0, 2, nframes * code.msgSize(), dtype=np.uint8)
        parity = code.encode(shard(msg, nframes, rank, world))
        parts = [None] * world
        dist.all_gather_object(parts, (frame_range(nframes, rank, world), np.asarray(parity)))
        slowest = max_over_ranks(1.0 + rank)
        if rank == 0:
            whole = np.asarray(code.encode(msg))
            joined = np.concatenate([p for _, p in sorted(parts, key=lambda x: x[0][0])])
            ok = bool(np.array_equal(joined, whole)) and slowest == float(world)
            with open(result_path, "w") as f:
                f.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_reassemble_the_batch(tmp_path):
    import torch.multiprocessing as mp
    result = str(tmp_path / "result")
    mp.spawn(_rank_main, args=(2, _free_port(), 77, result), nprocs=2, join=True)
    assert open(result).read() == "ok"


def _random_jobs(rng, count):
    return [(float(rng.uniform(0.1, 50.0)), int(rng.integers(0, 600))) for _ in range(count)]


@pytest.mark.parametrize("world", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_partition_jobs_covers_each_frame_once_and_balances(world, seed):
    """Every frame of every job is in exactly one range, a rank holds at most one range
    per job, ranges start on chunk boundaries, and the busiest rank's cost is within
    the list-scheduling bound (average per rank + one chunk)."""
    from fecl_b200.shard import partition_jobs
    rng = np.random.default_rng(seed)
    jobs = _random_jobs(rng, int(rng.integers(1, 12)))
    parts = partition_jobs(jobs, world)
    assert len(parts) == world
    seen = [np.zeros(n, np.int32) for _, n in jobs]
    loads = []
    for p in parts:
        js = [j for j, _, _ in p]
        assert len(js) == len(set(js))
        load = 0.0
        for j, lo, hi in p:
            assert 0 <= lo < hi <= jobs[j][1] and lo % 32 == 0
            seen[j][lo:hi] += 1
            load += jobs[j][0] * (hi - lo)
        loads.append(load)
    assert all(np.all(s == 1) for s in seen)
    total = sum(c * n for c, n in jobs)
    biggest = max((c * min(n, 32) for c, n in jobs), default=0.0)
    assert max(loads) <= total / world + biggest + 1e-9
    assert partition_jobs(jobs, world) == parts


def test_partition_jobs_one_rank_and_errors():
    from fecl_b200.shard import partition_jobs
    assert partition_jobs([(1.0, 100), (2.0, 0), (0.5, 33)], 1) == [[(0, 0, 100), (2, 0, 33)]]
    with pytest.raises(ValueError):
        partition_jobs([(1.0, 10)], 0)
    with pytest.raises(ValueError):
        partition_jobs([(-1.0, 10)], 2)


def test_frame_cost_orders_the_codes():
    """The cost model: an LDPC frame costs E x I edge-iterations, a turbo frame its
    trellis steps per iteration x I, each at the measured per-unit time."""
    from fractions import Fraction

    import fecl_b200 as F
    from fecl_b200.shard import PS_PER_EDGE_ITERATION, PS_PER_TRELLIS_STEP, frame_cost
    H = F.Ldpc.DvbS2.matrix(64800, Fraction(1, 2))
    ldpc = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(50).precision(1))
    turbo = F.Turbo.lte(6144, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6))
    assert frame_cost(ldpc) == pytest.approx(ldpc.stateSize() * 50 * PS_PER_EDGE_ITERATION[1] * 1e-12)
    assert frame_cost(turbo) == pytest.approx(2 * (6144 + 3) * 6 * PS_PER_TRELLIS_STEP * 1e-12)
    assert frame_cost(ldpc) > 10 * frame_cost(turbo)
    with pytest.raises(TypeError):
        frame_cost(object())


def _partition_rank_main(rank, world, port, result_path):
    import datetime

    import torch.distributed as dist

    from fecl_b200.shard import partition_jobs

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        jobs = _random_jobs(np.random.default_rng(9), 7)
        mine = partition_jobs(jobs, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        if rank == 0:
            ok = got == partition_jobs(jobs, world)
            counts = [np.zeros(n, np.int32) for _, n in jobs]
            for p in got:
                for j, lo, hi in p:
                    counts[j][lo:hi] += 1
            ok = ok and all(np.all(c == 1) for c in counts)
            with open(result_path, "w") as f:
                f.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


def test_two_ranks_compute_the_same_partition(tmp_path):
    """Each rank computes its own share of a mixed job list with no exchange; gathered,
    the shares are rank 0's partition and cover every frame once."""
    import torch.multiprocessing as mp
    result = str(tmp_path / "result")
    mp.spawn(_partition_rank_main, args=(2, _free_port(), result), nprocs=2, join=True)
    assert open(result).read() == "ok"
