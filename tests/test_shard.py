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
