"""Device encoders (fecl_encode with device memory) and the device BPSK/AWGN channel
(fecl_awgn_llr).  The encoders must reproduce the host encoders -- which are pinned
to the reference's -- bit for bit on every code family; the channel must have the
model's statistics, be deterministic per seed, and feed the decoders end to end."""
from fractions import Fraction

import numpy as np
import pytest

from goldens import ARRAYS, SUITE3, T17

pytestmark = pytest.mark.gpu


def _ldpc(n, rate):
    import fecl_b200 as F
    return F.Ldpc(F.Ldpc.EncoderOptions(F.Ldpc.DvbS2.matrix(n, Fraction(*rate))), F.Ldpc.DecoderOptions().iterations(30))


def _codes():
    import fecl_b200 as F
    codes = [_ldpc(16200, r) for r in ((1, 4), (1, 2), (3, 4), (8, 9))]
    codes += [_ldpc(64800, r) for r in ((1, 2), (9, 10))]
    codes.append(F.Ldpc(F.Ldpc.EncoderOptions(F.Ldpc.Gallager.matrix(2048, 3, 5, 0)), F.Ldpc.DecoderOptions()))
    codes += [F.Turbo.lte(K) for K in (40, 1504, 6144)]
    perms = [ARRAYS["perm_1024"], ARRAYS["perm_512"], ARRAYS["perm_even_512"]]
    for term in (0, 1):
        codes.append(F.Turbo(F.Turbo.EncoderOptions([F.Trellis(*s) for s in SUITE3], perms).termination(term),
                             F.Turbo.DecoderOptions()))
    codes.append(F.Turbo(F.Turbo.EncoderOptions([F.Trellis(*T17)], [np.arange(1024), ARRAYS["perm_1024"]]),
                         F.Turbo.DecoderOptions()))
    return codes


def test_device_encoders_equal_host_encoders():
    import torch
    from fecl_b200 import channel as ch
    for i, code in enumerate(_codes()):
        n = 5 if code.paritySize() > 20000 else 37
        msg = ch.random_bits(n * code.msgSize(), 60 + i)
        host = code.encode(msg)
        dev = code.encode(torch.from_numpy(msg).cuda()).cpu().numpy()
        assert np.array_equal(host, dev), (i, code.msgSize(), code.paritySize())
        assert code.check(dev)


def test_awgn_statistics_and_determinism():
    import torch
    from fecl_b200 import channel as ch
    n = 1 << 22
    bits = torch.from_numpy(ch.random_bits(n, 61)).cuda()
    ebn0, rate = 1.0, 0.5
    esn0 = 10 ** (ebn0 / 10) * rate
    s2 = 1.0 / (2.0 * esn0)
    a = ch.awgn_llr_device(bits, ebn0, rate, 1234)
    b = ch.awgn_llr_device(bits, ebn0, rate, 1234)
    c = ch.awgn_llr_device(bits, ebn0, rate, 1235)
    assert torch.equal(a, b) and not torch.equal(a, c)
    x = bits.double() * 2 - 1
    noise = (a.double() * s2 / 2 - x).cpu().numpy()
    assert abs(noise.mean()) < 5 * np.sqrt(s2 / n)
    assert abs(noise.var() / s2 - 1.0) < 0.01
    # fourth moment of a normal: 3 sigma^4
    assert abs(np.mean(noise ** 4) / (3 * s2 * s2) - 1.0) < 0.03
    # other output types carry the same values
    h = ch.awgn_llr_device(bits, ebn0, rate, 1234, torch.float16)
    d = ch.awgn_llr_device(bits, ebn0, rate, 1234, torch.float64)
    assert torch.equal(h, a.half()) and torch.allclose(d.float(), a, rtol=1e-6, atol=1e-6)


def test_device_inputs_decode_end_to_end():
    """Message bits, codeword and L-values all made on the GPU, then decoded there:
    no frame errors well above threshold, and the same decisions as decoding the
    same L-values from host memory."""
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    nms = F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(30).scalingFactor(0.75)
    ldpc = F.Ldpc(F.Ldpc.EncoderOptions(F.Ldpc.DvbS2.matrix(16200, Fraction(1, 2))), nms)
    lte = F.Turbo.lte(6144, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6))
    for code, ebn0 in ((ldpc, 3.5), (lte, 2.0)):
        n = 16
        K = code.msgSize()
        msg = torch.randint(0, 2, (n * K,), dtype=torch.uint8, device="cuda")
        llr = ch.awgn_llr_device(code.encode(msg), ebn0, K / code.paritySize(), 99)
        bits = code.decode(llr)
        assert np.array_equal(bits.cpu().numpy(), code.decode(llr.cpu().numpy()))
        errors = (bits != msg).view(n, K).any(dim=1).sum().item()
        assert errors == 0, (K, errors)
