"""CPU checks of the FER sweep: its host helpers and its oracle fixture.

tests/golden/fer_sweep_oracle.json holds the frame failures of the compiled
reference decoder on the sweep of fecl_b200/fer.py.  Here it is pinned to the C
restatement of the reference decoder (oracle/fecl_oracle.c, FP64): on 32 frames of
each rate's mid-waterfall point, the frames the restatement fails are the ones the
fixture lists.
"""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _oracle():
    with open(os.path.join(HERE, "golden", "fer_sweep_oracle.json")) as f:
        return json.load(f)


def test_threshold_interpolation():
    from fecl_b200 import fer
    e = [1.0, 1.25, 1.5, 1.75]
    # log10 FER falls from -0.5 to -1.5 between 1.25 and 1.5 dB: it crosses -1 half way
    assert fer.threshold_db(e, [1.0, 10 ** -0.5, 10 ** -1.5, 0.0], 0.1) == pytest.approx(1.375)
    assert fer.threshold_db(e, [0.05, 0.0, 0.0, 0.0], 0.1) == 1.0
    assert fer.threshold_db(e, [1.0, 1.0, 1.0, 0.5], 0.1) is None
    # zero errors count as half a frame (FER 0.5 / 512)
    x = fer.threshold_db([1.0, 1.25], [1.0, 0.0], 0.01, frames=512)
    assert 1.0 < x < 1.25


def test_fail_flags_round_trip_and_loss_check():
    from fecl_b200 import fer
    rng = np.random.default_rng(3)
    f = rng.random(512) < 0.3
    assert np.array_equal(fer.unpack_fails(fer.pack_fails(f), 512), f)
    assert fer.loss_check([0.5, 0.01], [0.5, 0.0], frames=512, slack=2) == [(1, 5, 0)]
    assert fer.loss_check([0.5, 2 / 512], [0.5, 0.0], frames=512, slack=2) == []


def test_fixture_shape():
    from fecl_b200 import fer
    o = _oracle()
    assert o["frames"] == fer.FRAMES and o["ebn0_db"] == list(fer.EBN0_DB)
    assert o["iterations"] == fer.ITERATIONS and o["scaling"] == fer.SCALING
    for (num, den) in fer.RATES:
        r = o["rates"]["%d/%d" % (num, den)]
        assert r["K"] == fer.N * num // den
        curve = [float(fer.unpack_fails(h, fer.FRAMES).mean()) for h in r["fails"]]
        assert curve == pytest.approx(r["fer"])
        # each rate's curve runs from all frames failing to none within the grid
        assert r["fer"][0] > 0.9 and r["fer"][-1] == 0.0


@pytest.mark.parametrize("rate_index", [0, 1, 2])
def test_fixture_matches_restated_decoder(rate_index):
    import fecl_b200 as F
    from fecl_b200 import fer
    from oracle import restated
    o = _oracle()
    num, den = fer.RATES[rate_index]
    ref = o["rates"]["%d/%d" % (num, den)]
    p = min(range(len(ref["fer"])), key=lambda i: abs(ref["fer"][i] - 0.5))
    H = F.Ldpc.DvbS2.matrix(fer.N, Fraction(num, den))
    code = fer.code(rate_index)
    K = code.msgSize()
    msg = fer.sweep_msg(K, rate_index, p)
    llr = fer.sweep_llr(code.encode(msg), K, rate_index, p)
    n = 32
    oracle = restated.Ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx)
    bits, _ = oracle.decode(llr[:n * fer.N].astype(np.float64), F.Approximate, fer.ITERATIONS, fer.SCALING, None)
    got = fer.frame_fails(bits, msg[:n * K], n)
    want = fer.unpack_fails(ref["fails"][p], fer.FRAMES)[:n]
    assert np.array_equal(got, want), (p, np.nonzero(got != want)[0].tolist())
    assert 0 < want.sum() < n
