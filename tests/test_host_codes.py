"""Host-side code construction against the reference (no GPU): DVB-S2 and Gallager
matrices, the encoder transform (row order = soft-state layout), encoders, trellis
tables and the LTE interleaver, checked against the golden fixtures made with the
compiled reference and, where that library is built here, against it directly."""
from fractions import Fraction

import numpy as np
import pytest

from goldens import ARRAYS, GOLDEN, SUITE3, T17, LTE, sha

DVBS2 = [(k.split("_")) for k in GOLDEN["dvbs2"] if k[0].isdigit()]


@pytest.mark.parametrize("n,num,den", [(int(a), int(b), int(c)) for a, b, c in DVBS2])
def test_dvbs2_transform_and_encoder_match_reference(n, num, den):
    import fecl_b200 as F
    g = GOLDEN["dvbs2"]["%d_%d_%d" % (n, num, den)]
    H = F.Ldpc.DvbS2.matrix(n, Fraction(num, den))
    assert sha(np.concatenate([H.row_ptr, H.col_idx])) == g["H_sha"]
    code = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().iterations(10))
    assert code.msgSize() == g["msg_size"] and code.stateSize() == g["edges"]
    ck = code.checks()
    assert sha(np.concatenate([ck.row_ptr, ck.col_idx])) == g["checks_sha"]
    from fecl_b200 import channel as ch
    cw = code.encode(ch.random_bits(code.msgSize(), 104))
    assert sha(cw) == g["encode_sha"]
    assert code.check(cw)
    # msg = first K bits, rate K/n, standard codeword layout | info | parity |
    assert code.msgSize() * den == n * num or n == 16200


def test_dvbs2_64800_half_equals_the_reference_builder():
    import fecl_b200 as F
    H = F.Ldpc.DvbS2.matrix(64800, Fraction(1, 2))
    assert sha(np.concatenate([H.row_ptr, H.col_idx])) == GOLDEN["dvbs2"]["reference_builder_64800_1_2_sha"]


def test_gallager_matches_reference():
    import fecl_b200 as F
    G = F.Ldpc.Gallager.matrix(2048, 3, 5, 0)
    assert sha(np.concatenate([G.row_ptr, G.col_idx])) == GOLDEN["dvbs2"]["gallager_2048_3_5_0_sha"]
    code = F.Ldpc(F.Ldpc.EncoderOptions(G), F.Ldpc.DecoderOptions().iterations(30))
    assert code.msgSize() == GOLDEN["cases"]["gallager_exact_2db"]["msg_size"]


@pytest.mark.parametrize("n,wc,wr", [(60, 3, 6), (120, 3, 5), (256, 3, 4), (480, 2, 4), (512, 5, 10), (1000, 3, 6)])
def test_gallager_transform_matches_live_reference(has_ref, n, wc, wr):
    """The encoder transform (src/detail/Ldpc.cpp:216-331) on Gallager matrices, whose
    columns of equal weight and dependent rows exercise the column retirement, the
    row moves and the gap elimination: the transformed matrix (the soft-state edge
    order), the message size and the codewords equal the compiled reference's."""
    if not has_ref:
        pytest.skip("compiled reference not built here")
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    from oracle import ref as R
    for seed in range(4):
        H = F.Ldpc.Gallager.matrix(n, wc, wr, seed)
        code = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().iterations(10))
        rc = R.RefCodec.ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx, 2, 10)
        rows, cols, ptr, idx = rc.checks()
        ck = code.checks()
        assert (ck.rows(), ck.cols()) == (rows, cols)
        assert np.array_equal(ck.row_ptr, ptr) and np.array_equal(ck.col_idx, idx), (n, wc, wr, seed)
        assert code.msgSize() == rc.msg
        m = ch.random_bits(3 * code.msgSize(), seed)
        assert np.array_equal(code.encode(m), rc.encode(m))


def test_encode_block_all_zero_all_one():
    """test/Cpp/operations.h:61-71 and :86-92: all-0 / all-1 messages encode to codewords."""
    import fecl_b200 as F
    for code in (F.Ldpc(F.Ldpc.EncoderOptions(F.Ldpc.Gallager.matrix(2048, 3, 5, 0)), F.Ldpc.DecoderOptions().iterations(30)),
                 F.Turbo.lte(1024)):
        for v in (0, 1):
            for n in (1, 5):
                p = code.encode(np.full(code.msgSize() * n, v, np.uint8))
                assert code.check(p)
        p = code.encode(np.ones(code.msgSize(), np.uint8))
        p[3] ^= 1
        assert not code.check(p)


@pytest.mark.parametrize("key", list(GOLDEN["trellis"]))
def test_trellis_tables_match_reference(key):
    import fecl_b200 as F
    g = GOLDEN["trellis"][key]
    t = F.Trellis(*g["spec"])
    assert (t.stateCount(), t.inputCount(), t.outputSize()) == (g["state_count"], g["input_count"], g["output_size"])
    assert t.next_state.tolist() == g["next_state"] and t.output.tolist() == g["output"]


def test_lte_interleaver_matches_reference():
    import fecl_b200 as F
    for k, h in GOLDEN["lte_interleaver_sha"].items():
        assert sha(F.Turbo.Lte3Gpp.interleaver(int(k))) == h


@pytest.mark.parametrize("name", [n for n, c in GOLDEN["cases"].items()])
def test_codewords_match_reference(name):
    """Every golden case's codeword (the encoders of src/detail/Ldpc.cpp:180-209 and
    src/detail/Turbo.cpp:155-170 with the greedy tail of src/detail/Convolutional.cpp:189-211)."""
    import fecl_b200 as F
    from goldens import case_inputs, check_matrix, turbo_layout
    c = GOLDEN["cases"][name]
    if c["kind"] == "ldpc":
        code = F.Ldpc(F.Ldpc.EncoderOptions(check_matrix(c["code"])), F.Ldpc.DecoderOptions().iterations(c["iterations"]))
    else:
        specs, perms = turbo_layout(c["code"])
        code = F.Turbo(F.Turbo.EncoderOptions([F.Trellis(*s) for s in specs], perms).termination(c["termination"]))
    msg, cw, llr = case_inputs(name, code.encode)
    assert sha(cw) == c["sha"]["codeword"]


def test_live_reference_agrees(has_ref):
    if not has_ref:
        pytest.skip("compiled reference not built here")
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    from oracle import ref as R
    specs = SUITE3
    perms = [ARRAYS["perm_1024"], ARRAYS["perm_512"], ARRAYS["perm_even_512"]]
    for term in (0, 1):
        code = F.Turbo(F.Turbo.EncoderOptions([F.Trellis(*s) for s in specs], perms).termination(term))
        rc = R.RefCodec.turbo(specs, perms, term, 0, 0, 4)
        m = ch.random_bits(3 * code.msgSize(), 9)
        assert np.array_equal(code.encode(m), rc.encode(m))
        assert (code.msgSize(), code.systSize(), code.paritySize(), code.stateSize()) == (rc.msg, rc.syst, rc.parity, rc.state)
