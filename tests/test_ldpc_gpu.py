"""LDPC belief propagation on the GPU, against the FP64 oracle and the reference's
own property tests (test/Cpp/operations.h, test/Cpp/Ldpc.cpp), called through the
C-ABI (fecl_b200's ctypes binding)."""
from fractions import Fraction

import numpy as np
import pytest

from goldens import ARRAYS, GOLDEN, case_inputs, check_matrix, hard
from parity import assert_hard_parity, assert_soft_parity, frame_ok, soft_error

pytestmark = pytest.mark.gpu

LDPC_CASES = [n for n, c in GOLDEN["cases"].items() if c["kind"] == "ldpc"]


def make_code(H, alg, iterations, scaling=1.0):
    import fecl_b200 as F
    return F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(alg).iterations(iterations).scalingFactor(scaling))


def distort(bits, snrdb, seed):
    """The reference's test channel (test/Cpp/operations.h:42-59): L = (+-1) * N(4 snr, 4 sqrt(snr/2))."""
    snr = 10.0 ** (snrdb / 10.0)
    rng = np.random.default_rng(seed)
    return np.where(np.asarray(bits) > 0, 1.0, -1.0) * rng.normal(snr * 4.0, 4.0 * np.sqrt(snr / 2.0), size=len(bits))


@pytest.mark.parametrize("name", LDPC_CASES)
def test_golden_parity(name):
    """Hard and soft outputs against the reference's on the golden cases."""
    import fecl_b200 as F
    c = GOLDEN["cases"][name]
    code = make_code(check_matrix(c["code"]), c["algorithm"], c["iterations"], c["scaling"])
    msg, cw, llr = case_inputs(name, code.encode)
    K = c["msg_size"]
    ref_hard = hard(name)
    ref_msg = ARRAYS[name + "__msg"]
    bits = code.decode(llr.astype(np.float32))
    assert_hard_parity(bits, ref_hard, msg, K, ref_app=ref_msg)
    out = code.soDecode(F.Codec.Input().parity(llr.astype(np.float32)), F.Codec.Output().msg().parity().state())
    ok = frame_ok(ref_hard, msg, K)
    ex = c["algorithm"] == F.Exact
    assert_soft_parity(out.msg(), ref_msg, ok, K, what="msg", exact=ex)
    assert_soft_parity(out.parity(), ARRAYS[name + "__parity"], ok, c["parity_size"], what="parity", exact=ex)
    if name + "__state" in ARRAYS.files:
        assert_soft_parity(out.state(), ARRAYS[name + "__state"], ok, c["state_size"], what="state", exact=ex)


@pytest.mark.parametrize("alg", [0, 1, 2])
def test_config1_scale_parity(alg):
    """DVB-S2 short frame rate 1/2, 64 frames at Eb/N0 1.5 dB, 20 iterations,
    against the oracle on the same FP32 L-values."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    from oracle import checker
    H = F.Ldpc.DvbS2.matrix(16200, Fraction(1, 2))
    code = make_code(H, alg, 20)
    K, N = code.msgSize(), code.paritySize()
    msg = ch.random_bits(64 * K, 11)
    llr = ch.awgn_llr(code.encode(msg), 1.5, K / N, 11, np.float32)
    bits, its = code.decode(llr, iterations=True)
    ref_bits, ref_app = checker.ldpc_decode(H, alg, 20, 1.0, llr)
    assert_hard_parity(bits, ref_bits, msg, K, ref_app=ref_app)
    assert its.min() >= 1 and its.max() <= 20
    out = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg())
    assert_soft_parity(out.msg(), ref_app, frame_ok(ref_bits, msg, K), K, what="APP", exact=alg == F.Exact)


@pytest.fixture(scope="module", params=[0, 1, 2], ids=["exact", "linear", "approximate"])
def suite_code(request):
    """The reference suite's code: Gallager(2048, 3, 5, seed 0), 30 iterations."""
    import fecl_b200 as F
    return make_code(F.Ldpc.Gallager.matrix(2048, 3, 5, 0), request.param, 30), request.param


def test_decode(suite_code):
    """test_decode (operations.h:113-127) at the suite SNR, n = 1 and 5."""
    code, _ = suite_code
    for n in (1, 5):
        msg = np.ones(code.msgSize() * n, np.uint8)
        p = code.encode(msg)
        assert np.array_equal(code.decode(distort(p, 2.0, n)), msg)


def test_soDecode_agrees_with_decode(suite_code):
    """test_soDecode (operations.h:159-180) at -5 dB."""
    import fecl_b200 as F
    code, _ = suite_code
    p = code.encode(np.ones(code.msgSize(), np.uint8))
    llr = distort(p, -5.0, 3)
    out = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg())
    dec = code.decode(llr)
    assert np.array_equal(dec, (out.msg() >= 0).astype(np.uint8))


def test_soDecode_parityOut(suite_code):
    """test_soDecode_parityOut (operations.h:210-235)."""
    import fecl_b200 as F
    code, _ = suite_code
    msg = np.ones(code.msgSize(), np.uint8)
    p = code.encode(msg)
    llr = distort(p, 2.0, 4)
    out = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg().parity())
    assert np.array_equal(msg, (out.msg() > 0).astype(np.uint8))
    assert np.array_equal(p, ((llr + out.parity()) > 0).astype(np.uint8))


def test_zero_syst_and_zero_state_equal_none(suite_code):
    """test_soDecode_0systIn / 0stateIn (operations.h:276-342): bit-exact."""
    import fecl_b200 as F
    code, _ = suite_code
    p = code.encode(np.ones(code.msgSize(), np.uint8))
    llr = distort(p, -5.0, 5)
    a = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg().syst().parity())
    b = code.soDecode(F.Codec.Input().parity(llr).syst(np.zeros(code.systSize())), F.Codec.Output().msg().syst().parity())
    c = code.soDecode(F.Codec.Input().parity(llr).state(np.zeros(code.stateSize())), F.Codec.Output().msg().syst().parity())
    for x in (b, c):
        assert np.array_equal(a.msg(), x.msg()) and np.array_equal(a.syst(), x.syst()) and np.array_equal(a.parity(), x.parity())


def test_two_phase_resume(suite_code):
    """test_soDecode_2phases (operations.h:344-383): I iterations, then I more from the
    state, equal 2I iterations in one go, bit for bit."""
    import fecl_b200 as F
    code, alg = suite_code
    code2 = make_code(F.Ldpc.Gallager.matrix(2048, 3, 5, 0), alg, 60)
    p = code.encode(np.ones(code.msgSize(), np.uint8))
    assert np.array_equal(p, code2.encode(np.ones(code.msgSize(), np.uint8)))
    llr = distort(p, -5.0, 6)
    st = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().state()).state()
    a = code.soDecode(F.Codec.Input().parity(llr).state(st), F.Codec.Output().msg().syst().parity())
    b = code2.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg().syst().parity())
    assert np.array_equal(a.msg(), b.msg()) and np.array_equal(a.syst(), b.syst()) and np.array_equal(a.parity(), b.parity())


def test_systOut_is_parityOut_prefix(suite_code):
    """test_ldpc_soDecode_systOut (test/Cpp/Ldpc.cpp:32-49)."""
    import fecl_b200 as F
    code, _ = suite_code
    llr = distort(code.encode(np.ones(code.msgSize(), np.uint8)), -5.0, 7)
    out = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().parity().syst())
    assert np.array_equal(out.syst(), out.parity()[: code.systSize()])


def test_systIn_does_not_hurt(suite_code):
    """test_soDecode_systIn (operations.h:237-274)."""
    import fecl_b200 as F
    code, _ = suite_code
    msg = np.ones(code.msgSize(), np.uint8)
    p = code.encode(msg)
    llr = distort(p, -5.0, 8)
    syst = distort(msg, -5.0, 9)
    a = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg())
    b = code.soDecode(F.Codec.Input().parity(llr).syst(syst), F.Codec.Output().msg())
    e1 = np.sum(msg != (a.msg() > 0))
    e2 = np.sum(msg != (b.msg() > 0))
    assert e2 <= e1


def test_state_resume_matches_oracle_soft(suite_code):
    """soDecode with a-priori and state inputs against the oracle (all four outputs)."""
    import fecl_b200 as F
    from oracle import restated as O
    if not O.available():
        pytest.skip("restated oracle not built")
    code, alg = suite_code
    H = F.Ldpc.Gallager.matrix(2048, 3, 5, 0)
    o = O.Ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx)
    msg = np.ones(code.msgSize() * 3, np.uint8)
    llr = distort(code.encode(msg), 1.0, 10).astype(np.float32).astype(np.float64)
    syst = (0.1 * distort(msg, -5.0, 11)).astype(np.float32).astype(np.float64)
    st = o.so_decode(llr, alg, 30, outputs=("state",))["state"].astype(np.float32).astype(np.float64)
    ref = o.so_decode(llr, alg, 30, syst=syst, state=st)
    out = code.soDecode(F.Codec.Input().parity(llr).syst(syst).state(st), F.Codec.Output().msg().syst().parity().state())
    ok = frame_ok((ref["msg"] >= 0).astype(np.uint8), msg, code.msgSize())
    for k in ("msg", "syst", "parity", "state"):
        size = {"msg": code.msgSize(), "syst": code.systSize(), "parity": code.paritySize(), "state": code.stateSize()}[k]
        assert_soft_parity(getattr(out, k)(), ref[k], ok, size, what=k, exact=alg == F.Exact)


def test_input_dtypes_and_device_memory():
    """float64 / float32 / float16 L-values, host and device memory give the same bits."""
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(16200, Fraction(1, 2))
    code = make_code(H, F.Approximate, 20, 0.75)
    K, N = code.msgSize(), code.paritySize()
    llr = ch.awgn_llr(code.encode(ch.random_bits(4 * K, 12)), 2.0, K / N, 12, np.float16)
    a = code.decode(llr)
    b = code.decode(llr.astype(np.float32))
    c = code.decode(llr.astype(np.float64))
    d = code.decode(torch.from_numpy(llr).cuda()).cpu().numpy()
    assert np.array_equal(a, b) and np.array_equal(b, c) and np.array_equal(c, d)


@pytest.mark.parametrize("alg", [0, 1, 2])
def test_lane_batched_kernel_equals_generic(alg):
    """The lane-batched kernel (32 frames per warp) and the one-CTA-per-frame generic
    kernel compute the same FP32 operations: outputs agree bit for bit, including the
    per-frame iteration counts of the syndrome stop."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(16200, Fraction(1, 2))
    code = make_code(H, alg, 20, 0.75 if alg == 2 else 1.0)
    K, N = code.msgSize(), code.paritySize()
    msg = ch.random_bits(40 * K, 13)
    llr = ch.awgn_llr(code.encode(msg), 1.3, K / N, 13, np.float32)
    syst = ch.awgn_llr(msg, -3.0, 1.0, 14, np.float32) * 0.1
    outs = {}
    for kernel in ("auto", "generic"):
        code.setKernel(kernel)
        bits, its = code.decode(llr, iterations=True)
        so = code.soDecode(F.Codec.Input().parity(llr).syst(syst), F.Codec.Output(np.float32).msg().syst().parity().state())
        st = code.soDecode(F.Codec.Input().parity(llr).state(so.state()), F.Codec.Output(np.float32).msg())
        outs[kernel] = (bits, its, so.msg(), so.syst(), so.parity(), so.state(), st.msg())
    for a, b in zip(outs["auto"], outs["generic"]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [1, 2])
def test_reduced_precision_messages(precision):
    """FP16 and saturated int8 (Q5.2) message storage with FP32 sums, normalized
    min-sum 0.75: frame errors within a few frames of the FP32 path near threshold;
    FP16 error-free where FP32 is, int8 within two frames of 64 there (its step of
    1/4 costs a little)."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(64800, Fraction(1, 2))
    K = 32400
    msg = ch.random_bits(64 * K, 15)
    ref = make_code(H, F.Approximate, 50, 0.75)
    cw = ref.encode(msg)
    low = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(50)
                 .scalingFactor(0.75).precision(precision))
    for ebn0, slack in ((1.0, 6), (2.0, 0 if precision == 1 else 2)):
        llr = ch.awgn_llr(cw, ebn0, 0.5, 16, np.float32)
        fer = [np.sum(~frame_ok(c.decode(llr), msg, K)) for c in (ref, low)]
        assert fer[1] <= fer[0] + slack, (ebn0, fer)


def _all_outputs(code, llr, syst, F):
    bits, its = code.decode(llr, iterations=True)
    so = code.soDecode(F.Codec.Input().parity(llr).syst(syst), F.Codec.Output(np.float32).msg().syst().parity().state())
    st = code.soDecode(F.Codec.Input().parity(llr).state(so.state()), F.Codec.Output(np.float32).msg())
    return bits, its, so.msg(), so.syst(), so.parity(), so.state(), st.msg()


@pytest.mark.parametrize("alg,precision,n,rate,shapes", [
    (0, 0, 16200, (1, 2), [(2, 512), (4, 1024)]),
    (1, 0, 16200, (1, 2), [(2, 1024), (8, 512)]),
    (2, 0, 16200, (1, 2), [(2, 512), (4, 512), (16, 512)]),
    (2, 1, 16200, (1, 2), [(1, 1024), (2, 512)]),
    (2, 2, 16200, (1, 2), [(1, 512), (4, 1024)]),
    (2, 1, 64800, (9, 10), [(8, 512), (8, 256)]),
    (2, 0, 64800, (3, 4), [(8, 1024)]),
])
def test_cluster_kernel_equals_lanes(alg, precision, n, rate, shapes):
    """The cluster-resident kernel (messages in the shared memory of 1 to 16 CTAs,
    neighbours' values over distributed shared memory) and the lane-batched kernel
    compute the same FP32 operations: every output, hard and soft, and the per-frame
    iteration counts agree bit for bit, for every cluster shape."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(n, Fraction(*rate))
    code = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(alg).iterations(20)
                  .scalingFactor(0.75 if alg == 2 else 1.0).precision(precision))
    K, N = code.msgSize(), code.paritySize()
    frames = 37 if n == 16200 else 9
    msg = ch.random_bits(frames * K, 17)
    # half the frames near threshold (some run every iteration), half 1.5 dB above
    # (the syndrome stops them early)
    ebn0 = {(1, 2): 1.2, (3, 4): 2.4, (9, 10): 3.6}[rate]
    cw = code.encode(msg).reshape(frames, N)
    h = frames // 2
    llr = np.concatenate([ch.awgn_llr(cw[:h].ravel(), ebn0, K / N, 17, np.float32),
                          ch.awgn_llr(cw[h:].ravel(), ebn0 + 1.5, K / N, 21, np.float32)])
    syst = ch.awgn_llr(msg, -3.0, 1.0, 18, np.float32) * 0.1
    code.setKernel("lanes")
    ref = _all_outputs(code, llr, syst, F)
    assert ref[1].min() >= 1 and ref[1].max() <= 20 and len(set(ref[1].tolist())) > 1
    code.setKernel("cluster")
    for cl, th in shapes:
        code.setClusterShape(cl, th)
        got = _all_outputs(code, llr, syst, F)
        for what, a, b in zip(("bits", "iterations", "msg", "syst", "parity", "state", "resumed msg"), ref, got):
            assert np.array_equal(a, b), (cl, th, what)


@pytest.mark.parametrize("alg", [0, 2])
def test_cluster_kernel_iteration_dependent_scaling(alg):
    """Scaling that changes with the iteration: the cluster kernel tests the syndrome
    in a pass of its own and runs the final check update with the last iteration's
    scaling, as the reference does; it agrees bit for bit with the generic kernel."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(16200, Fraction(1, 2))
    sf = {0: [0.6 + 0.02 * i for i in range(20)]}
    code = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(alg).iterations(20).scalingFactor(sf))
    K, N = code.msgSize(), code.paritySize()
    msg = ch.random_bits(20 * K, 19)
    llr = ch.awgn_llr(code.encode(msg), 1.3, K / N, 19, np.float32)
    syst = ch.awgn_llr(msg, -3.0, 1.0, 20, np.float32) * 0.1
    code.setKernel("generic")
    ref = _all_outputs(code, llr, syst, F)
    code.setKernel("cluster")
    for cl in (2, 4, 8):
        code.setClusterShape(cl, 512)
        got = _all_outputs(code, llr, syst, F)
        for what, a, b in zip(("bits", "iterations", "msg", "syst", "parity", "state", "resumed msg"), ref, got):
            assert np.array_equal(a, b), (cl, what)


def _nms(H, precision, iterations=50):
    import fecl_b200 as F
    return F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(F.Approximate).iterations(iterations)
                  .scalingFactor(0.75).precision(precision))


def test_packed_fp16_frames_are_independent():
    """The packed FP16 min-sum kernel (two frames per lane, 64 per warp) decodes every
    frame on its own: a frame's bits and iteration count are the same alone, first or
    last in a batch of 65, whatever its neighbours."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(16200, Fraction(3, 5))
    code = _nms(H, 1)
    K, N = code.msgSize(), code.paritySize()
    msg = ch.random_bits(65 * K, 41)
    llr = ch.awgn_llr_per_frame(code.encode(msg), N, np.linspace(1.5, 3.5, 65), K / N, 41, np.float32)
    bits, its = code.decode(llr, iterations=True)
    assert len(set(its.tolist())) > 3
    for f in (0, 31, 32, 63, 64):
        b1, i1 = code.decode(llr[f * N:(f + 1) * N], iterations=True)
        assert np.array_equal(b1, bits[f * K:(f + 1) * K]) and i1[0] == its[f], f


@pytest.mark.parametrize("n,rate", [(16200, (3, 5)), (64800, (1, 2))])
def test_packed_fp16_group_width_does_not_change_results(n, rate):
    """Batches of up to 16 frames run one group of 2, 4 or 8 lanes (2 W frames);
    larger ones groups of 8, 16 or 32 lanes, whichever idles the fewest frame slots:
    every frame's bits, iteration count and soft outputs (a-posteriori, extrinsic,
    edge state) are the same bit for bit in batches of every width (1, 3 and 4
    frames: W = 2; 5: 4; 16 and 37: 8; 17 and 32: 16) as in one of 64 frames
    (W = 32)."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(n, Fraction(*rate))
    code = _nms(H, 1, 30)
    K, N = code.msgSize(), code.paritySize()
    total = 64
    msg = ch.random_bits(total * K, 47)
    lo, hi = (1.6, 3.2) if n == 16200 else (0.9, 1.8)
    llr = ch.awgn_llr_per_frame(code.encode(msg), N, np.linspace(lo, hi, total), K / N, 47, np.float32)
    syst = (0.1 * ch.awgn_llr(msg, -2.0, 1.0, 48, np.float32)).astype(np.float32)

    def run(a, b):
        bits, its = code.decode(llr[a * N:b * N], iterations=True)
        so = code.soDecode(F.Codec.Input().parity(llr[a * N:b * N]).syst(syst[a * K:b * K]),
                           F.Codec.Output(np.float32).msg().syst().parity().state())
        return bits, its, so.msg(), so.syst(), so.parity(), so.state()

    full = run(0, total)
    assert len(set(full[1].tolist())) > 2
    sizes = {"bits": K, "iterations": 1, "msg": K, "syst": K, "parity": N, "state": code.stateSize()}
    for a, b in ((0, 1), (5, 8), (9, 13), (13, 18), (20, 36), (3, 20), (2, 34), (27, 64)):
        got = run(a, b)
        for (what, size), x, y in zip(sizes.items(), full, got):
            assert np.array_equal(np.asarray(x)[a * size:b * size], np.asarray(y)), (a, b, what)


@pytest.mark.parametrize("n,rate,ebn0s", [(16200, (1, 2), (1.2, 1.6, 2.2)), (64800, (9, 10), (3.4, 3.7, 4.2)),
                                          (64800, (1, 2), (1.0, 1.3))])
def test_packed_fp16_fer_matches_fp32(n, rate, ebn0s):
    """FP16 message passing with half2 check-node arithmetic against FP32 message
    passing on the same L-values: the frame error rates agree within a few frames of
    the 96 at each Eb/N0, near threshold and above it."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(n, Fraction(*rate))
    ref, low = _nms(H, 0), _nms(H, 1)
    K, N = ref.msgSize(), ref.paritySize()
    frames = 96
    msg = ch.random_bits(frames * K, 43)
    cw = ref.encode(msg)
    for ebn0 in ebn0s:
        llr = ch.awgn_llr(cw, ebn0, K / N, 44, np.float32)
        fer = [int(np.sum(~frame_ok(c.decode(llr), msg, K))) for c in (ref, low)]
        assert abs(fer[1] - fer[0]) <= max(3, fer[0] // 8), (ebn0, fer)


def test_packed_fp16_soft_state_falls_back_to_fp32_arithmetic():
    """A soft state input is decoded by the lane kernel with FP32 check-node arithmetic
    (FP16 storage), exactly as FECL_KERNEL_LANES does."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(16200, Fraction(1, 2))
    code = _nms(H, 1, 20)
    K, N = code.msgSize(), code.paritySize()
    msg = ch.random_bits(8 * K, 45)
    llr = ch.awgn_llr(code.encode(msg), 1.4, K / N, 45, np.float32)
    st = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output(np.float32).state()).state()
    a = code.soDecode(F.Codec.Input().parity(llr).state(st), F.Codec.Output(np.float32).msg()).msg()
    code.setKernel("lanes")
    b = code.soDecode(F.Codec.Input().parity(llr).state(st), F.Codec.Output(np.float32).msg()).msg()
    assert np.array_equal(a, b)


@pytest.mark.parametrize("alg,precision,frames,n", [(0, 0, 40, 16200), (1, 0, 40, 16200), (2, 0, 200, 16200),
                                                    (2, 1, 130, 16200), (2, 2, 40, 16200), (2, 1, 64, 64800)])
def test_persistent_launch_equals_launch_per_pass(alg, precision, frames, n):
    """A small batch decoded by one persistent launch (check and bit passes separated
    by grid barriers) and by two launches per iteration: the same outputs bit for bit,
    iteration counts and soft outputs included, from device and from host memory (the
    host path decodes its chunks on several streams)."""
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    H = F.Ldpc.DvbS2.matrix(n, Fraction(1, 2))
    code = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(alg).iterations(30)
                  .scalingFactor(0.75 if alg == 2 else 1.0).precision(precision))
    K, N = code.msgSize(), code.paritySize()
    msg = ch.random_bits(frames * K, 40 + alg)
    llr = ch.awgn_llr(code.encode(msg), 1.2 if n == 16200 else 1.0, K / N, 40 + alg, np.float32)
    d_llr = torch.from_numpy(llr).cuda()
    outs = {}
    for mode in (1, -1):
        code.setPersistent(mode)
        bits, its = code.decode(d_llr, iterations=True)
        hbits = code.decode(llr)
        res = [bits.cpu().numpy(), its.cpu().numpy(), hbits]
        if precision == 0:
            so = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output(np.float32).msg().state())
            res += [so.msg(), so.state()]
        outs[mode] = res
    assert np.all(outs[1][1] > 0)
    for a, b in zip(outs[1], outs[-1]):
        assert np.array_equal(a, b)
