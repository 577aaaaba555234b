"""The convolutional codec's host side against the compiled reference, on CPU:
sizes, encode (greedy tail), check and puncturing, for non-recursive, recursive
and 2-input trellises under both terminations."""
import numpy as np
import pytest

ref = pytest.importorskip("oracle.ref")
pytestmark = pytest.mark.skipif(not ref.available(), reason="reference library not built")

TRELLISES = [([7], [[0o171, 0o133]], None), ([3], [[0o7, 0o5]], None), ([4], [[0o15]], [0o13]),
             ([3, 3], [[0o5, 0o3, 0], [0, 0o3, 0o7]], [0o7, 0o5])]


def _pair(spec, length, term, alg=2, sf=1.0):
    import fecl_b200 as F
    mine = F.Convolutional(F.Convolutional.EncoderOptions(F.Trellis(*spec), length).termination(term),
                           F.Convolutional.DecoderOptions().algorithm(alg).scalingFactor(sf))
    return mine, ref.RefCodec.conv(spec, length, term, alg, sf)


@pytest.mark.parametrize("term", [0, 1])
@pytest.mark.parametrize("spec", TRELLISES)
def test_sizes_encode_check(spec, term):
    mine, rc = _pair(spec, 257, term)
    assert (mine.msgSize(), mine.systSize(), mine.paritySize(), mine.stateSize()) == (rc.msg, rc.syst, rc.parity, rc.state)
    msg = np.random.default_rng(80).integers(0, 2, 9 * mine.msgSize()).astype(np.uint8)
    p = mine.encode(msg)
    assert np.array_equal(p, rc.encode(msg))
    assert mine.check(p) and rc.check(p)
    bad = p.copy()
    bad[5] ^= 1
    assert mine.check(bad) == rc.check(bad)


@pytest.mark.parametrize("masks", [((), ()), ((1, 1, 0),), ((0, 1, 1, 1),), ((1, 0), (1,)), ((), (0, 1, 1))])
@pytest.mark.parametrize("term", [0, 1])
def test_puncturing_matches_reference(masks, term):
    import fecl_b200 as F
    mask = masks[0]
    tail = masks[1] if len(masks) > 1 else ()
    mine, rc = _pair(TRELLISES[0], 100, term)
    seq, ins = rc.conv_puncturing(mask, tail)
    p = mine.puncturing(F.Convolutional.PunctureOptions().mask(mask).tailMask(tail))
    assert p.inputSize() == ins and np.array_equal(p.sequence(), seq)
