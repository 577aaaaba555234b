"""The convolutional codec on the GPU against the compiled reference: Viterbi
decisions bit for bit (both use FP64 path metrics in the same comparison order),
MAP soft outputs within the parity rules, device encoding equal to the host's."""
import numpy as np
import pytest

from parity import assert_soft_parity, frame_ok

from test_conv import TRELLISES, _pair

pytestmark = pytest.mark.gpu


def _llr(bits, snrdb, seed):
    snr = 10.0 ** (snrdb / 10.0)
    rng = np.random.default_rng(seed)
    return np.where(np.asarray(bits) > 0, 1.0, -1.0) * rng.normal(snr * 4.0, 4.0 * np.sqrt(snr / 2.0), size=len(bits))


@pytest.mark.parametrize("term", [0, 1])
@pytest.mark.parametrize("spec", TRELLISES)
def test_viterbi_matches_reference(spec, term):
    mine, rc = _pair(spec, 500, term)
    n = 40
    msg = np.random.default_rng(81).integers(0, 2, n * mine.msgSize()).astype(np.uint8)
    p = mine.encode(msg)
    for snr in (-3.0, 0.0, 3.0):
        llr = _llr(p, snr, 82).astype(np.float32)
        got = mine.decode(llr)
        want = rc.decode(llr.astype(np.float64))
        assert np.array_equal(got, want), snr


@pytest.mark.parametrize("alg", [0, 1, 2])
@pytest.mark.parametrize("spec", TRELLISES[:3])
def test_map_soDecode_matches_reference(spec, alg):
    import fecl_b200 as F
    for term in (0, 1):
        mine, rc = _pair(spec, 300, term, alg, 0.8)
        n = 12
        msg = np.random.default_rng(83).integers(0, 2, n * mine.msgSize()).astype(np.uint8)
        llr = _llr(mine.encode(msg), -1.0, 84).astype(np.float32).astype(np.float64)
        syst = (0.3 * _llr(np.zeros(n * mine.systSize(), np.uint8), -6.0, 85)).astype(np.float32).astype(np.float64)
        for s in (None, syst):
            want = rc.so_decode(llr, syst=s, outputs=("msg", "syst", "parity"))
            inp = F.Codec.Input().parity(llr)
            if s is not None:
                inp.syst(s)
            out = mine.soDecode(inp, F.Codec.Output().msg().syst().parity())
            ok = frame_ok((want["msg"] > 0).astype(np.uint8), msg, mine.msgSize())
            assert_soft_parity(out.msg(), want["msg"], ok, mine.msgSize(), what="msg", exact=alg == F.Exact)
            assert_soft_parity(out.syst(), want["syst"], ok, mine.systSize(), what="syst", exact=alg == F.Exact)
            assert_soft_parity(out.parity(), want["parity"], ok, mine.paritySize(), what="parity", exact=alg == F.Exact)


def test_device_encode_equals_host():
    import torch
    for spec in TRELLISES:
        for term in (0, 1):
            mine, _ = _pair(spec, 333, term)
            msg = np.random.default_rng(86).integers(0, 2, 7 * mine.msgSize()).astype(np.uint8)
            assert np.array_equal(mine.encode(msg), mine.encode(torch.from_numpy(msg).cuda()).cpu().numpy())
