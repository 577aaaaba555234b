"""Puncturing patterns (Codec::puncturing) against the compiled reference, on CPU:
LDPC masks and systematic masks, turbo masks, tail masks and both bit orderings, on
the LTE code and the reference suite's three-constituent code with a 2-input
trellis.  The sequences and input sizes must be identical."""
from fractions import Fraction

import numpy as np
import pytest

from goldens import ARRAYS, SUITE3

ref = pytest.importorskip("oracle.ref")
pytestmark = pytest.mark.skipif(not ref.available(), reason="reference library not built")

LDPC_OPTIONS = [((), ()), ((1, 1, 0),), ((0, 1),), ((1, 0, 1, 1),), ((), (1, 0)), ((1, 1, 0), (1, 1, 1, 0)),
                ((0,), (1,)), ((1, 0), (0, 1, 1))]


@pytest.mark.parametrize("opts", LDPC_OPTIONS)
def test_ldpc_puncturing_matches_reference(opts):
    import fecl_b200 as F
    mask = opts[0]
    syst = opts[1] if len(opts) > 1 else ()
    for H in (F.Ldpc.DvbS2.matrix(16200, Fraction(1, 2)), F.Ldpc.Gallager.matrix(512, 3, 4, 1)):
        code = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions())
        rc = ref.RefCodec.ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx, 2, 10)
        seq, ins = rc.ldpc_puncturing(mask, syst)
        p = code.puncturing(F.Ldpc.PunctureOptions().mask(mask).systMask(syst))
        assert p.inputSize() == ins and np.array_equal(p.sequence(), seq)


TURBO_OPTIONS = [
    ([], [], 0), ([], [], 1),
    ([[1], [1, 0], [0, 1]], [], 0), ([[1], [1, 0], [0, 1]], [], 1),
    ([[1, 1, 0], [], [1, 0, 0]], [], 0),
    ([[1], [1, 0], [0, 1]], [[1, 0], [0], [1], [1, 1, 0]], 0),
    ([[1], [1, 0], [0, 1]], [[1, 0], [0], [1], [1, 1, 0]], 1),
    ([], [[0], [], [], [1, 0]], 1),
]


@pytest.mark.parametrize("masks,tails,ordering", TURBO_OPTIONS)
def test_lte_turbo_puncturing_matches_reference(masks, tails, ordering):
    import fecl_b200 as F
    K = 1024
    code = F.Turbo.lte(K)
    rc = ref.RefCodec.turbo([([4], [[0o15]], [0o13])], [np.arange(K), F.Turbo.Lte3Gpp.interleaver(K)], 0, 2, 0, 4)
    seq, ins = rc.turbo_puncturing(masks, tails, ordering)
    p = code.puncturing(F.Turbo.PunctureOptions().mask(masks).tailMask(tails).bitOrdering(ordering))
    assert p.inputSize() == ins and np.array_equal(p.sequence(), seq)


@pytest.mark.parametrize("ordering", [0, 1])
@pytest.mark.parametrize("term", [0, 1])
def test_three_constituent_puncturing_matches_reference(ordering, term):
    import fecl_b200 as F
    perms = [ARRAYS["perm_1024"], ARRAYS["perm_512"], ARRAYS["perm_even_512"]]
    code = F.Turbo(F.Turbo.EncoderOptions([F.Trellis(*s) for s in SUITE3], perms).termination(term), F.Turbo.DecoderOptions())
    rc = ref.RefCodec.turbo(SUITE3, perms, term, 2, 0, 4)
    masks = [[1, 0], [1, 1, 0], [0, 1], [1, 0, 0, 1]]
    tails = [[1], [0, 1], [1, 0], [], [0], [1, 1, 0]]
    for m, t in (([], []), (masks, []), (masks, tails)):
        seq, ins = rc.turbo_puncturing(m, t, ordering)
        p = code.puncturing(F.Turbo.PunctureOptions().mask(m).tailMask(t).bitOrdering(ordering))
        assert p.inputSize() == ins and np.array_equal(p.sequence(), seq), (m, t)


def test_invalid_mask_counts_raise_like_the_reference():
    import fecl_b200 as F
    code = F.Turbo.lte(40)
    with pytest.raises(ValueError):
        code.puncturing(F.Turbo.PunctureOptions().mask([[1], [1]]))
    with pytest.raises(ValueError):
        code.puncturing(F.Turbo.PunctureOptions().tailMask([[1]]))
