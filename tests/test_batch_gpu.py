"""Mixed batches (fecl_batch_*): frames of several codecs in one CUDA graph launch --
LTE turbo frames of many K in one persistent launch, LDPC codes of several sizes,
rates, algorithms and message precisions, a non-LTE turbo code.  Each job's
decisions and iteration counts must equal those of the codec's own decode, bit for
bit, with and without autotuning."""
from fractions import Fraction

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _jobs(seed=0, dtype=np.float32):
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    rng = np.random.default_rng(seed)
    specs = []
    tdec = F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6).scheduling(F.Serial)
    for K, n in ((6144, 6), (40, 9), (1024, 5), (3200, 4), (512, 7)):
        specs.append((F.Turbo.lte(K, tdec), n, rng.uniform(0.3, 1.5)))
    specs.append((F.Turbo.lte(2048, F.Turbo.DecoderOptions().algorithm(F.Exact).iterations(4)), 3, 0.8))
    ms = F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(30).scalingFactor(0.75)
    H = F.Ldpc.DvbS2.matrix(16200, Fraction(1, 2))
    specs.append((F.Ldpc(F.Ldpc.EncoderOptions(H), ms.precision(1)), 40, 1.6))
    H = F.Ldpc.DvbS2.matrix(16200, Fraction(3, 4))
    specs.append((F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(30)
                         .scalingFactor(0.75).precision(2)), 33, 2.8))
    H = F.Ldpc.Gallager.matrix(2048, 3, 5, 0)
    specs.append((F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(F.Exact).iterations(20)), 12, 2.0))
    # a turbo code the windowed kernel does not cover: three constituents
    tr = F.Trellis([4], [[0o15]], [0o13])
    K = 256
    perms = [np.arange(K), rng.permutation(K), rng.permutation(K)]
    specs.append((F.Turbo(F.Turbo.EncoderOptions([tr], perms), F.Turbo.DecoderOptions().algorithm(F.Linear)
                          .iterations(4)), 5, 1.0))
    jobs = []
    for i, (code, n, ebn0) in enumerate(specs):
        K, N = code.msgSize(), code.paritySize()
        msg = ch.random_bits(n * K, 100 + i)
        llr = ch.awgn_llr(code.encode(msg), ebn0, K / N, 100 + i, dtype)
        d_llr = torch.from_numpy(llr).cuda()
        jobs.append((code, d_llr, torch.zeros(n * K, dtype=torch.uint8, device="cuda"),
                     torch.zeros(n, dtype=torch.int32, device="cuda")))
    return jobs


def _alone(jobs):
    """Each job decoded by its codec alone; LTE turbo codecs with the window shape of
    the batch's mixed-K kernel (64 segments), which a decode of a few frames would
    otherwise replace by 128 (a difference of FP32 rounding in frames that fail)."""
    import fecl_b200 as F
    out = []
    for code, llr, _, _ in jobs:
        if isinstance(code, F.Turbo):
            code.setWindowSegments(64)
        bits, its = code.decode(llr, iterations=True)
        if isinstance(code, F.Turbo):
            code.setWindowSegments(0)
        out.append((bits.cpu().numpy(), its.cpu().numpy()))
    return out


@pytest.mark.parametrize("autotune", [False, True])
@pytest.mark.parametrize("dtype", [np.float32, np.float16])
def test_batch_equals_each_codec_alone(autotune, dtype):
    import torch
    import fecl_b200 as F
    jobs = _jobs(1, dtype)
    ref = _alone(jobs)
    b = F.Batch(jobs, autotune=autotune)
    plan = b.describe()
    assert "turbo LTE mixed-K" in plan and "ldpc" in plan
    for rep in range(2):
        for _, _, m, it in jobs:
            m.zero_()
            it.zero_()
        b.run()
        torch.cuda.synchronize()
        for (code, _, m, it), (rb, ri) in zip(jobs, ref):
            assert np.array_equal(m.cpu().numpy(), rb), (rep, code.msgSize())
            assert np.array_equal(it.cpu().numpy(), ri), (rep, code.msgSize())


def test_batch_rerun_with_new_inputs_and_option_change():
    import torch
    import fecl_b200 as F
    jobs = _jobs(2)
    b = F.Batch(jobs)
    fresh = _jobs(3)
    for (_, llr, _, _), (_, llr2, _, _) in zip(jobs, fresh):
        llr.copy_(llr2)
    b.run()
    torch.cuda.synchronize()
    # the same codecs on the new L-values (the random interleavers of _jobs depend on its seed)
    for (code, llr, m, _), (rb, _) in zip(jobs, _alone(jobs)):
        assert np.array_equal(m.cpu().numpy(), rb)
    code = jobs[-3][0]
    code.setDecoderOptions(F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(10))
    with pytest.raises(ValueError):
        b.run()


@pytest.mark.parametrize("shared", [None, "passes", "persistent"])
def test_batch_shared_ldpc_launch_equals_each_codec_alone(shared):
    """FP16-message LDPC jobs of several codes and check-degree classes, several
    frame groups each and more than one wave, beside turbo frames: with the shared
    persistent LDPC launch (and without it) every job's decisions and iteration
    counts equal its codec's own decode bit for bit, on two runs in a row."""
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    dec = F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(50).scalingFactor(0.75).precision(1)
    specs = []
    for (n, r, frames, ebn0) in ((16200, (1, 2), 70, 1.3), (16200, (3, 4), 130, 2.6), (16200, (5, 6), 20, 3.4),
                                 (64800, (1, 2), 65, 1.5), (64800, (9, 10), 10, 3.9), (16200, (2, 3), 3, 2.0)):
        H = F.Ldpc.DvbS2.matrix(n, Fraction(*r))
        specs.append((F.Ldpc(F.Ldpc.EncoderOptions(H), dec), frames, ebn0))
    specs.append((F.Turbo.lte(1024, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6)), 5, 0.8))
    jobs = []
    for i, (code, nf, ebn0) in enumerate(specs):
        K, N = code.msgSize(), code.paritySize()
        msg = ch.random_bits(nf * K, 300 + i)
        llr = ch.awgn_llr(code.encode(msg), ebn0, K / N, 300 + i, np.float16)
        jobs.append((code, torch.from_numpy(llr).cuda(), torch.zeros(nf * K, dtype=torch.uint8, device="cuda"),
                     torch.zeros(nf, dtype=torch.int32, device="cuda")))
    ref = _alone(jobs)
    b = F.Batch(jobs, shared_ldpc=shared)
    assert ("ldpc shared" in b.describe()) == (shared is not None)
    for rep in range(2):
        for _, _, m, it in jobs:
            m.fill_(7)
            it.fill_(-7)
        b.run()
        torch.cuda.synchronize()
        for (code, _, m, it), (rb, ri) in zip(jobs, ref):
            assert np.array_equal(it.cpu().numpy(), ri), (rep, code.msgSize())
            assert np.array_equal(m.cpu().numpy(), rb), (rep, code.msgSize())
