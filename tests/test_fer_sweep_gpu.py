"""FER of the DVB-S2 normal-frame decoders against the FP64 reference decoder.

The sweep (fecl_b200/fer.py): rates 1/2, 3/4, 9/10, 512 seeded frames per Eb/N0
point, normalised min-sum 0.75, at most 50 iterations with the syndrome stop.  The
reference's frame failures on the same L-values are the committed fixture
tests/golden/fer_sweep_oracle.json (made by tests/golden/make_fer_sweep.py from the
compiled reference).  The tests decode the points of each rate's waterfall (oracle
FER strictly between 0 and 1, with one point on each side):

* FP32 messages: the failing frames are the reference's, frame by frame, up to
  FP32_FRAME_SLACK frames per point (a frame that converges in the last iterations
  can go either way between FP32 and FP64 rounding).
* FP16 messages lose at most 0.1 dB: on the same noise draws 0.1 dB better, the FP16
  decoder fails no more frames than the reference at the point itself, up to
  LOSS_SLACK frames.
* Saturated int8 (Q5.2) messages also lose at most 0.1 dB, by the same comparison.

Measured on a B200 (bench.py --workload fer-sweep, same frames): the FP32 failures
equal the reference's in all 19,968 frames, the FP16 FER equals the reference's at
every point, and int8 at +0.1 dB never fails more frames than the reference.
"""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FP32_FRAME_SLACK = 2
LOSS_SLACK = 2


def _oracle():
    with open(os.path.join(HERE, "golden", "fer_sweep_oracle.json")) as f:
        return json.load(f)


def waterfall_points(fer_curve):
    """Indices of the points with 0 < FER < 1, widened by one point on each side."""
    inside = [i for i, f in enumerate(fer_curve) if 0.0 < f < 1.0]
    if not inside:
        return []
    lo, hi = max(0, inside[0] - 1), min(len(fer_curve) - 1, inside[-1] + 1)
    return list(range(lo, hi + 1))


@pytest.mark.gpu
@pytest.mark.parametrize("rate_index", [0, 1, 2])
def test_fer_sweep_against_reference(rate_index):
    import torch

    from fecl_b200 import fer
    oracle = _oracle()
    num, den = fer.RATES[rate_index]
    ref = oracle["rates"]["%d/%d" % (num, den)]
    assert oracle["frames"] == fer.FRAMES and oracle["ebn0_db"] == list(fer.EBN0_DB)
    codes = {q: fer.code(rate_index, q) for q in (0, 1, 2)}
    K = codes[0].msgSize()
    assert K == ref["K"]
    points = waterfall_points(ref["fer"])
    assert points, "the sweep must cross this rate's waterfall"
    out = torch.empty(fer.FRAMES * K, dtype=torch.uint8, device="cuda")

    def fails(q, llr, msg):
        codes[q].decode(torch.from_numpy(llr).cuda(), out=out)
        return fer.frame_fails(out.cpu().numpy(), msg, fer.FRAMES)

    for p in points:
        msg = fer.sweep_msg(K, rate_index, p)
        cw = codes[0].encode(msg)
        ofails = fer.unpack_fails(ref["fails"][p], fer.FRAMES)
        f32 = fails(0, fer.sweep_llr(cw, K, rate_index, p), msg)
        assert int(np.sum(f32 != ofails)) <= FP32_FRAME_SLACK, (p, int(f32.sum()), int(ofails.sum()))
        f16 = fails(1, fer.sweep_llr(cw, K, rate_index, p, shift_db=0.1), msg)
        assert int(f16.sum()) <= int(ofails.sum()) + LOSS_SLACK, ("f16 +0.1 dB", p, int(f16.sum()), int(ofails.sum()))
        i8 = fails(2, fer.sweep_llr(cw, K, rate_index, p, shift_db=0.1), msg)
        assert int(i8.sum()) <= int(ofails.sum()) + LOSS_SLACK, ("i8 +0.1 dB", p, int(i8.sum()), int(ofails.sum()))
