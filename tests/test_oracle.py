"""The CPU restatement (oracle/fecl_oracle.c) is pinned against the reference: its
outputs on every golden case must equal the compiled reference's bit for bit
(SHA-256 of the float64 outputs recorded by tests/golden/make_golden.py)."""
import numpy as np
import pytest

from goldens import GOLDEN, case_inputs, check_matrix, sha, turbo_layout


@pytest.fixture(scope="module")
def restated():
    from oracle import restated as O
    if not O.available():
        pytest.skip("oracle/_build/libfecl_oracle.so not built")
    return O


LDPC_CASES = [n for n, c in GOLDEN["cases"].items() if c["kind"] == "ldpc"]
TURBO_CASES = [n for n, c in GOLDEN["cases"].items() if c["kind"] == "turbo"]


@pytest.mark.parametrize("name", LDPC_CASES)
def test_ldpc_restatement_is_bit_exact(restated, name):
    c = GOLDEN["cases"][name]
    H = check_matrix(c["code"])
    code = restated.Ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx)
    msg, cw, llr = case_inputs(name, code.encode)
    assert sha(cw) == c["sha"]["codeword"]
    bits, its = code.decode(llr, c["algorithm"], c["iterations"], c["scaling"], threads=4)
    assert sha(bits) == c["sha"]["hard"]
    out = code.so_decode(llr, c["algorithm"], c["iterations"], c["scaling"], threads=4)
    for k in ("msg", "syst", "parity", "state"):
        assert sha(out[k]) == c["sha"][k], k


@pytest.mark.parametrize("name", TURBO_CASES)
def test_turbo_restatement_is_bit_exact(restated, name):
    c = GOLDEN["cases"][name]
    specs, perms = turbo_layout(c["code"])
    code = restated.Turbo([restated.trellis(*s) for s in specs], perms, c["termination"])
    msg, cw, llr = case_inputs(name, code.encode)
    assert sha(cw) == c["sha"]["codeword"]
    scaling = None if c["scaling"] is None else np.asarray(c["scaling"])
    bits = code.decode(llr, c["algorithm"], c["iterations"], c["scheduling"], scaling=scaling, threads=4)
    assert sha(bits) == c["sha"]["hard"]
    out = code.so_decode(llr, c["algorithm"], c["iterations"], c["scheduling"], threads=4)
    for k in ("msg", "syst", "parity", "state"):
        assert sha(out[k]) == c["sha"][k], k


def test_restated_dvbs2_matrix_equals_product_builder(restated):
    from fractions import Fraction
    import fecl_b200 as F
    for n, r in ((16200, Fraction(1, 2)), (64800, Fraction(3, 4)), (64800, Fraction(9, 10))):
        H = F.Ldpc.DvbS2.matrix(n, r)
        _, _, p, i = restated.dvbs2_matrix(n, r.numerator, r.denominator)
        assert np.array_equal(p, H.row_ptr) and np.array_equal(i, H.col_idx)


def test_restatement_against_live_reference(restated, has_ref):
    """Where the reference is compiled here, compare on fresh inputs too (soft
    decode with a-priori and state inputs, both schedulings)."""
    if not has_ref:
        pytest.skip("compiled reference not built here")
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    from oracle import ref as R
    K = 512
    perm = F.Turbo.Lte3Gpp.interleaver(K)
    t = restated.lte_turbo(K)
    msg = ch.random_bits(3 * K, 77)
    cw = t.encode(msg)
    for alg in (0, 1, 2):
        for sched in (0, 1):
            rc = R.RefCodec.turbo([([4], [[0o15]], [0o13])], [np.arange(K), perm], 0, alg, sched, 5)
            llr = ch.awgn_llr(cw, 0.3, 1 / 3, 78, np.float32).astype(np.float64)
            state = rc.so_decode(llr, outputs=("state",))["state"]
            syst = ch.awgn_llr(np.zeros(3 * t.syst, np.uint8), 0.0, 1.0, 79)
            a = t.so_decode(llr, alg, 5, sched, syst=syst, state=state)
            b = rc.so_decode(llr, syst=syst, state=state, outputs=("msg", "syst", "parity", "state"))
            for k in b:
                assert np.array_equal(a[k], b[k]), (alg, sched, k)
