"""The decode server (fecl_server_*): continuous batching of requests of mixed codes.
Each request's decisions must equal the codec's own decode of the same L-values --
the same alone and in the mix -- whatever the batches it landed in, under a memory
budget that forces many small batches, from several submitting threads, and under
a Poisson replay."""
import threading
from fractions import Fraction

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _codes():
    import fecl_b200 as F
    codes = []
    tdec = F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6).scheduling(F.Serial)
    for K in (40, 512, 1504, 6144):
        codes.append(F.Turbo.lte(K, tdec))
    ms = F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(50).scalingFactor(0.75).precision(1)
    for n, r in ((16200, (1, 2)), (16200, (5, 6)), (64800, (3, 4))):
        codes.append(F.Ldpc(F.Ldpc.EncoderOptions(F.Ldpc.DvbS2.matrix(n, Fraction(*r))), ms))
    return codes


def _alone(reqs):
    """Each request decoded by its codec alone; LTE turbo codecs with the window shape
    of the server's mixed-K kernel (64 segments), which a decode of a few frames would
    otherwise replace by 128 (a difference of FP32 rounding in frames that fail)."""
    import fecl_b200 as F
    out = []
    for c, llr in reqs:
        if isinstance(c, F.Turbo):
            c.setWindowSegments(64)
        out.append(c.decode(llr))
        if isinstance(c, F.Turbo):
            c.setWindowSegments(0)
    return out


def _requests(codes, count, seed):
    from fecl_b200 import channel as ch
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        c = codes[int(rng.integers(len(codes)))]
        nf = int(rng.integers(1, 4))
        K, N = c.msgSize(), c.paritySize()
        msg = ch.random_bits(nf * K, seed * 1000 + i)
        llr = ch.awgn_llr(c.encode(msg), float(rng.uniform(0.5, 3.0)), K / N, seed * 1000 + i, np.float16)
        reqs.append((c, llr))
    return reqs


def test_results_same_alone_and_in_the_mix():
    import fecl_b200 as F
    codes = _codes()
    reqs = _requests(codes, 60, 1)
    alone = _alone(reqs)
    srv = F.Server(device_budget=4 << 30, max_batch_frames=512, slots=3)
    got = [None] * len(reqs)

    def submitter(idx):
        tickets = [(i, srv.submit(reqs[i][0], reqs[i][1])) for i in idx]
        for i, t in tickets:
            got[i] = srv.wait(t)

    threads = [threading.Thread(target=submitter, args=(list(range(k, len(reqs), 3)),)) for k in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for i, (a, g) in enumerate(zip(alone, got)):
        msg, lat = g
        assert lat > 0
        assert np.array_equal(a, msg), i
    rep = srv.report()
    assert rep["requests"] == len(reqs) and rep["batches"] >= 1
    assert rep["p99_s"] >= rep["p50_s"] > 0
    srv.close()


def test_small_budget_forces_many_batches_and_rejects_oversize():
    import fecl_b200 as F
    codes = _codes()
    reqs = [r for r in _requests(codes, 40, 2) if r[0].paritySize() <= 16200 * 1 or r[0].msgSize() <= 6144]
    alone = _alone(reqs)
    # about 96 MiB per slot: a few short LDPC frames or turbo frames per batch
    srv = F.Server(device_budget=3 * (96 << 20), max_batch_frames=64, slots=3)
    tickets = [srv.submit(c, llr) for c, llr in reqs]
    for a, t in zip(alone, tickets):
        msg, _ = srv.wait(t)
        assert np.array_equal(a, msg)
    assert srv.report()["batches"] > 3
    # a request larger than a slot's memory cannot be admitted
    big = codes[-1]
    from fecl_b200 import channel as ch
    llr = ch.awgn_llr(big.encode(ch.random_bits(200 * big.msgSize(), 3)), 3.0, 0.75, 3, np.float32)
    t = srv.submit(big, llr)
    with pytest.raises(F.FeclError):
        srv.wait(t)
    srv.close()


def test_poisson_replay():
    import fecl_b200 as F
    codes = _codes()
    reqs = _requests(codes, 200, 4)
    alone = _alone(reqs)
    rng = np.random.default_rng(5)
    arrivals = np.cumsum(rng.exponential(1.0 / 5000.0, size=len(reqs)))
    srv = F.Server(slots=3)
    outs, lat = srv.replay(arrivals, reqs)
    for a, m in zip(alone, outs):
        assert np.array_equal(a, m)
    assert np.all(lat > 0)
    srv.close()


def test_batches_larger_than_the_initial_staging():
    """Batches whose L-values (FP32 DVB-S2 normal frames, 259 KB each) and decisions
    outgrow a slot's initial pinned staging (64 MiB in, 16 MiB out): the buffers grow
    while other slots' batches are in flight, and every request still gets the
    decisions of its codec decoding alone."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    ms = F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(20).scalingFactor(0.75).precision(1)
    code = F.Ldpc(F.Ldpc.EncoderOptions(F.Ldpc.DvbS2.matrix(64800, Fraction(3, 4))), ms)
    K, N = code.msgSize(), code.paritySize()
    reqs = []
    for i in range(6):
        n = 100 + 20 * i
        msg = ch.random_bits(n * K, 600 + i)
        reqs.append((code, ch.awgn_llr(code.encode(msg), 2.8, K / N, 600 + i, np.float32)))
    alone = _alone(reqs)
    srv = F.Server(device_budget=12 << 30, max_batch_frames=400, slots=2)
    tickets = [srv.submit(c, llr) for c, llr in reqs]
    for a, t in zip(alone, tickets):
        msg, _ = srv.wait(t)
        assert np.array_equal(a, msg)
    rep = srv.report()
    assert rep["requests"] == len(reqs) and rep["frames"] == sum(100 + 20 * i for i in range(6))
    srv.close()
