"""Edge cases on the GPU as callers of the reference meet them: calls with no frames,
batch sizes that leave the host pipeline's chunks ragged, erased (zero) and
saturated L-values.  Decisions are compared with the compiled reference (through
the oracle) under the parity rules of tests/parity.py, or with the same frames
decoded from device memory, which must agree bit for bit."""
from fractions import Fraction

import numpy as np
import pytest

from parity import assert_hard_parity

pytestmark = pytest.mark.gpu


def _ldpc(alg, iterations=30, scaling=1.0, n=16200, rate=(1, 2)):
    import fecl_b200 as F
    H = F.Ldpc.DvbS2.matrix(n, Fraction(*rate))
    d = F.Ldpc.DecoderOptions().algorithm(alg).iterations(iterations).scalingFactor(scaling)
    return H, F.Ldpc(F.Ldpc.EncoderOptions(H), d)


def _lte(K, alg=2, iterations=6):
    import fecl_b200 as F
    return F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(alg).iterations(iterations).scheduling(F.Serial))


def _codes():
    import fecl_b200 as F
    codes = [_ldpc(F.Approximate)[1], _lte(1024)]
    rsc = F.Trellis([4], [[0o15]], [0o13])
    codes.append(F.Turbo(F.Turbo.EncoderOptions([rsc], [np.arange(512), np.random.default_rng(3).permutation(512),
                                                       np.random.default_rng(4).permutation(512)]),
                         F.Turbo.DecoderOptions().algorithm(F.Linear).iterations(4)))
    codes.append(F.Convolutional(F.Convolutional.EncoderOptions(F.Trellis([7], [[0o171, 0o133]]), 500).termination(0),
                                 F.Convolutional.DecoderOptions()))
    return codes


def test_calls_with_no_frames_return_empty_outputs():
    """Codec::decode and soDecode of an empty buffer return empty buffers (the
    reference's size checks accept 0 frames), from host and from device memory."""
    import torch
    import fecl_b200 as F
    for code in _codes():
        empty = np.zeros(0, np.float32)
        assert code.decode(empty).size == 0
        out = code.soDecode(F.Codec.Input().parity(empty), F.Codec.Output(np.float32).msg().parity())
        assert out.msg().size == 0 and out.parity().size == 0
        d = torch.zeros(0, dtype=torch.float32, device="cuda")
        assert code.decode(d).numel() == 0


@pytest.mark.parametrize("n", [1, 63, 65, 129, 515])
def test_ragged_batches_through_the_host_pipeline(n):
    """Host-memory decodes cut the batch into chunks of at least 64 frames (the last
    one shorter); whatever the cut, the bits and iteration counts equal a
    device-memory decode of the whole batch."""
    import torch
    from fecl_b200 import channel as ch
    import fecl_b200 as F
    for code, ebn0 in ((_lte(1024), 0.8), (_ldpc(F.Approximate, 20, 0.75)[1], 2.0)):
        K, N = code.msgSize(), code.paritySize()
        msg = ch.random_bits(n * K, 70 + n)
        llr = ch.awgn_llr(code.encode(msg), ebn0, K / N, 70 + n, np.float32)
        bits, its = code.decode(llr, iterations=True)
        dbits, dits = code.decode(torch.from_numpy(llr).cuda(), iterations=True)
        assert np.array_equal(bits, dbits.cpu().numpy()) and np.array_equal(its, dits.cpu().numpy()), (n, K)


def _erase(llr, fraction, seed):
    """Zero a fraction of the L-values (erasures: punctured or lost bits)."""
    out = llr.copy()
    out[np.random.default_rng(seed).random(out.size) < fraction] = 0.0
    return out


@pytest.mark.parametrize("alg", [0, 2])
def test_ldpc_erasures_match_reference(alg):
    """DVB-S2 short frames with 15 % of their L-values erased: the GPU's decisions
    equal the reference's in every frame it decodes (ties excepted), and frames it
    fails fail on the GPU too."""
    from fecl_b200 import channel as ch
    from oracle import checker
    H, code = _ldpc(alg, 30, 0.75 if alg == 2 else 1.0)
    K, N = code.msgSize(), code.paritySize()
    n = 24
    msg = ch.random_bits(n * K, 81)
    llr = _erase(ch.awgn_llr(code.encode(msg), 2.6, K / N, 81, np.float32), 0.15, 82)
    bits = code.decode(llr)
    ref_bits, ref_app = checker.ldpc_decode(H, alg, 30, 0.75 if alg == 2 else 1.0, llr)
    assert_hard_parity(bits, ref_bits, msg, K, ref_app=ref_app)


def test_turbo_erasures_match_reference():
    """LTE K=1024 with 10 % of the L-values erased, max-log-MAP, 6 iterations."""
    from fecl_b200 import channel as ch
    from oracle import checker
    import fecl_b200 as F
    code = _lte(1024)
    K, N = code.msgSize(), code.paritySize()
    n = 32
    msg = ch.random_bits(n * K, 83)
    llr = _erase(ch.awgn_llr(code.encode(msg), 1.2, K / N, 83, np.float32), 0.10, 84)
    bits = code.decode(llr)
    ref_bits, ref_app = checker.turbo_lte_decode(K, F.Approximate, 6, F.Serial, llr)
    assert_hard_parity(bits, ref_bits, msg, K, ref_app=ref_app)


@pytest.mark.parametrize("which", ["ldpc", "turbo"])
def test_saturated_llrs_match_reference(which):
    """L-values a thousand times larger than the channel's (a receiver with a wrong
    noise estimate, or hard decisions fed as +-L), with 2 % of them of the wrong sign:
    no overflow on the GPU, and the same decisions as the reference."""
    from fecl_b200 import channel as ch
    from oracle import checker
    import fecl_b200 as F
    if which == "ldpc":
        H, code = _ldpc(F.Approximate, 20, 0.75)
    else:
        code = _lte(1024)
    K, N = code.msgSize(), code.paritySize()
    n = 16
    msg = ch.random_bits(n * K, 85)
    cw = code.encode(msg).astype(np.float32)
    rng = np.random.default_rng(86)
    llr = (2.0 * cw - 1.0) * rng.uniform(500.0, 5000.0, cw.size).astype(np.float32)
    llr[rng.random(llr.size) < 0.02] *= -1.0
    bits = code.decode(llr)
    assert bits.shape == msg.shape
    if which == "ldpc":
        ref_bits, ref_app = checker.ldpc_decode(H, F.Approximate, 20, 0.75, llr)
    else:
        ref_bits, ref_app = checker.turbo_lte_decode(K, F.Approximate, 6, F.Serial, llr)
    assert_hard_parity(bits, ref_bits, msg, K, ref_app=ref_app)
