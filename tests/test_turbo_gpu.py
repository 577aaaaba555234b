"""Turbo decoding on the GPU, against the FP64 oracle and the reference's own
property tests (test/Cpp/operations.h, test/Cpp/Turbo.cpp), through the C-ABI."""
import numpy as np
import pytest

from goldens import ARRAYS, GOLDEN, SUITE3, T17, case_inputs, hard, turbo_layout
from parity import assert_hard_parity, assert_soft_parity, frame_ok

pytestmark = pytest.mark.gpu

TURBO_CASES = [n for n, c in GOLDEN["cases"].items() if c["kind"] == "turbo"]


def distort(bits, snrdb, seed):
    snr = 10.0 ** (snrdb / 10.0)
    rng = np.random.default_rng(seed)
    return np.where(np.asarray(bits) > 0, 1.0, -1.0) * rng.normal(snr * 4.0, 4.0 * np.sqrt(snr / 2.0), size=len(bits))


def make_turbo(specs, perms, term, alg, iterations, sched, scaling=None):
    import fecl_b200 as F
    dec = F.Turbo.DecoderOptions().algorithm(alg).iterations(iterations).scheduling(sched)
    if scaling is not None:
        dec.scalingFactor(np.asarray(scaling).tolist())
    return F.Turbo(F.Turbo.EncoderOptions([F.Trellis(*s) for s in specs], perms).termination(term), dec)


@pytest.mark.parametrize("kernel", ["auto", "generic"])
@pytest.mark.parametrize("name", TURBO_CASES)
def test_golden_parity(name, kernel):
    import fecl_b200 as F
    c = GOLDEN["cases"][name]
    specs, perms = turbo_layout(c["code"])
    code = make_turbo(specs, perms, c["termination"], c["algorithm"], c["iterations"], c["scheduling"], c["scaling"])
    code.setKernel(kernel)
    msg, cw, llr = case_inputs(name, code.encode)
    K = c["msg_size"]
    ref_hard = hard(name)
    ref_msg = ARRAYS[name + "__msg"]
    bits = code.decode(llr.astype(np.float32))
    assert_hard_parity(bits, ref_hard, msg, K, ref_app=ref_msg)
    if c["scaling"] is None:  # soDecode ignores scaling (TurboDecoderImpl.cpp:75-150); decode applies it
        out = code.soDecode(F.Codec.Input().parity(llr.astype(np.float32)), F.Codec.Output().msg().state())
        ok = frame_ok(ref_hard, msg, K)
        assert_soft_parity(out.msg(), ref_msg, ok, K, what="msg")
        assert_soft_parity(out.state(), ARRAYS[name + "__state"], ok, c["state_size"], what="state")


@pytest.mark.parametrize("alg", [2, 1, 0])
def test_config2_scale_parity(alg):
    """LTE K=6144, 6 iterations, serial, Eb/N0 0.7 dB, 128 frames: the windowed
    kernel against the FP64 oracle on the same FP32 L-values."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    from oracle import checker
    K, n = 6144, 128
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(alg).iterations(6).scheduling(F.Serial))
    msg = ch.random_bits(n * K, 31)
    llr = ch.awgn_llr(code.encode(msg), 0.7, K / code.paritySize(), 31, np.float32)
    bits = code.decode(llr)
    ref_bits, ref_app = checker.turbo_lte_decode(K, alg, 6, F.Serial, llr)
    assert_hard_parity(bits, ref_bits, msg, K, ref_app=ref_app)
    passes, rounds, recomputed = code.windowStats()
    assert passes == n * 12


def test_windowed_equals_generic_kernel():
    """The windowed LTE kernel and the generic kernel (the reference's operation order
    in FP32) under the parity rules, whatever the training length: the same hard
    decisions bit for bit in every frame the generic kernel decodes, the same frames
    failing.  In a failed frame the decisions follow FP32 rounding (the windowed
    kernel normalises its metrics once per 8 steps), so a few of them may differ."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    K, n = 2048, 48
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6))
    msg = ch.random_bits(n * K, 32)
    llr = ch.awgn_llr(code.encode(msg), 0.6, K / code.paritySize(), 32, np.float32)
    code.setKernel("generic")
    ref = code.decode(llr)
    code.setKernel("auto")
    for train in (0, 32, 96, 256):
        code.setWindowTraining(train)
        for segs in (32, 64, 128):
            code.setWindowSegments(segs)
            assert_hard_parity(code.decode(llr), ref, msg, K) > n // 4, (train, segs)


@pytest.mark.parametrize("alg", [2, 1, 0])
def test_balanced_rounds_match_generic_kernel(alg):
    """1024 frames with the segment count left to the launcher run as two launches
    (whole GPU rounds of 32-segment frames, then 64-segment ones, the second launch's
    frame offset applied to every buffer).  With a CRC-24A stop, under the parity
    rules: the decisions equal the generic kernel's in every frame it decodes and the
    same frames fail; every frame of either launch that stopped early passes its
    CRC, each reporting its own iteration count; a single 64-segment launch gives
    the same decisions in the decoded frames."""
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    K, n = 1024, 1024
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(alg).iterations(6).crc(F.CRC24A))
    info = torch.from_numpy(ch.random_bits(n * (K - 24), 35 + alg)).cuda()
    msg = F.crc24_attach(info, F.CRC24A, n).cpu().numpy()
    ebn0 = np.repeat(np.linspace(0.3, 1.5, 8), n // 8)
    llr = ch.awgn_llr_per_frame(code.encode(msg), code.paritySize(), ebn0, K / code.paritySize(), 35 + alg,
                                np.float32)
    code.setKernel("generic")
    ref, ref_it = code.decode(llr, iterations=True)
    code.setKernel("auto")
    split, split_it = code.decode(llr, iterations=True)
    assert assert_hard_parity(split, ref, msg, K) > n // 4
    ok = frame_ok(ref, msg, K)
    early = split_it < 6
    assert early[: n // 2].sum() > n // 16 and early[n // 2:].sum() > n // 16 and len(set(split_it.tolist())) > 2
    crc_ok = F.crc24_check(torch.from_numpy(split).cuda(), F.CRC24A, n).cpu().numpy()
    assert crc_ok[early].all()
    code.setWindowSegments(64)
    single = code.decode(llr)
    assert np.array_equal(split.reshape(n, K)[ok], single.reshape(n, K)[ok])


@pytest.mark.parametrize("K", [40, 1008, 4096, 6144])
def test_lte_sizes(K):
    """Every LTE block size the windowed kernel sees decodes like the generic kernel."""
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(4))
    msg = ch.random_bits(8 * K, K)
    llr = ch.awgn_llr(code.encode(msg), 1.0, K / code.paritySize(), K, np.float32)
    a = code.decode(llr)
    code.setKernel("generic")
    b = code.decode(llr)
    assert np.array_equal(a, b)


SUITE_PARAMS = [(1, 0, 1), (0, 0, 1), (0, 1, 1), (0, 2, 1), (0, 2, 0)]  # (termination, algorithm, scheduling)


@pytest.fixture(scope="module", params=SUITE_PARAMS, ids=["default", "tail", "table", "approximate", "serial"])
def suite_code(request):
    """test/Cpp/Turbo.cpp:89-161: K=1024 random interleaver, Trellis({4},{{017}},{015}), 4 iterations."""
    term, alg, sched = request.param
    perms = [np.arange(1024, dtype=np.uint32), ARRAYS["perm_1024"]]
    mk = lambda it: make_turbo([T17], perms, term, alg, it, sched)
    return mk(4), mk(8)


def test_decode(suite_code):
    code, _ = suite_code
    for n in (1, 5):
        msg = np.ones(code.msgSize() * n, np.uint8)
        assert np.array_equal(code.decode(distort(code.encode(msg), -2.0, n)), msg)


def test_soDecode_agrees_with_decode(suite_code):
    import fecl_b200 as F
    code, _ = suite_code
    llr = distort(code.encode(np.ones(code.msgSize(), np.uint8)), -5.0, 3)
    out = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg())
    assert np.array_equal(code.decode(llr), (out.msg() > 0).astype(np.uint8))


def test_soDecode_parityOut(suite_code):
    import fecl_b200 as F
    code, _ = suite_code
    msg = np.ones(code.msgSize(), np.uint8)
    p = code.encode(msg)
    llr = distort(p, -2.0, 4)
    out = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg().parity())
    assert np.array_equal(msg, (out.msg() > 0).astype(np.uint8))
    assert np.array_equal(p, ((llr + out.parity()) > 0).astype(np.uint8))


def test_zero_syst_and_zero_state_equal_none(suite_code):
    import fecl_b200 as F
    code, _ = suite_code
    llr = distort(code.encode(np.ones(code.msgSize(), np.uint8)), -5.0, 5)
    a = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg().syst().parity())
    b = code.soDecode(F.Codec.Input().parity(llr).syst(np.zeros(code.systSize())), F.Codec.Output().msg().syst().parity())
    c = code.soDecode(F.Codec.Input().parity(llr).state(np.zeros(code.stateSize())), F.Codec.Output().msg().syst().parity())
    for x in (b, c):
        assert np.array_equal(a.msg(), x.msg()) and np.array_equal(a.syst(), x.syst()) and np.array_equal(a.parity(), x.parity())


def test_two_phase_resume(suite_code):
    import fecl_b200 as F
    code, code2 = suite_code
    llr = distort(code.encode(np.ones(code.msgSize(), np.uint8)), -5.0, 6)
    st = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().state()).state()
    a = code.soDecode(F.Codec.Input().parity(llr).state(st), F.Codec.Output().msg().syst().parity())
    b = code2.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg().syst().parity())
    assert np.array_equal(a.msg(), b.msg()) and np.array_equal(a.syst(), b.syst()) and np.array_equal(a.parity(), b.parity())


def test_systOut_is_parityOut_prefix(suite_code):
    import fecl_b200 as F
    code, _ = suite_code
    llr = distort(code.encode(np.ones(code.msgSize(), np.uint8)), -5.0, 7)
    out = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().parity().syst())
    assert np.array_equal(out.syst(), out.parity()[: code.systSize()])


@pytest.mark.parametrize("term", [1, 0])
@pytest.mark.parametrize("sched", [0, 1])
def test_three_variable_length_constituents(term, sched):
    """test/Cpp/Turbo.cpp:143-161: three constituents, one with a 2-input trellis,
    interleavers of lengths 1024, 512 and 512 (even positions)."""
    import fecl_b200 as F
    from oracle import restated as O
    perms = [ARRAYS["perm_1024"], ARRAYS["perm_512"], ARRAYS["perm_even_512"]]
    code = make_turbo(SUITE3, perms, term, F.Exact, 4, sched)
    msg = np.ones(code.msgSize() * 2, np.uint8)
    llr = distort(code.encode(msg), 0.0, 8)
    assert np.array_equal(code.decode(llr), msg)
    if O.available():
        o = O.Turbo([O.trellis(*s) for s in SUITE3], perms, term)
        x = llr.astype(np.float32).astype(np.float64)
        ref = o.so_decode(x, F.Exact, 4, sched)
        out = code.soDecode(F.Codec.Input().parity(x), F.Codec.Output().msg().syst().parity().state())
        ok = frame_ok((ref["msg"] > 0).astype(np.uint8), msg, code.msgSize())
        for k, size in (("msg", code.msgSize()), ("syst", code.systSize()), ("parity", code.paritySize()),
                        ("state", code.stateSize())):
            assert_soft_parity(getattr(out, k)(), ref[k], ok, size, what=k)


def test_device_memory_decode_matches_host():
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    K = 6144
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6))
    llr = ch.awgn_llr(code.encode(ch.random_bits(16 * K, 40)), 0.8, K / code.paritySize(), 40, np.float32)
    a = code.decode(llr)
    b = code.decode(torch.from_numpy(llr).cuda()).cpu().numpy()
    c = code.decode(torch.from_numpy(llr).pin_memory()).numpy()
    assert np.array_equal(a, b) and np.array_equal(a, c)


CUSTOM_SCHEDULES = [
    [([0, 1, 2], [[1, 2], [0, 2], [0, 1]])],                       # all constituents at once (like Parallel)
    [([0], [[1, 2]]), ([2, 1], [[0, 1], [0, 2]])],                 # two stages, activation given out of order
    [([1], [[0]]), ([0], [[1]]), ([2], [[0, 1]])],                 # one constituent per stage, partial transfers
]


@pytest.mark.parametrize("stages", CUSTOM_SCHEDULES)
@pytest.mark.parametrize("alg", [2, 0])
def test_custom_scheduling_matches_reference(stages, alg):
    """Turbo::DecoderOptions::scheduling(Scheduling) (TurboDecoderImpl.cpp:170-189,
    252-289) on the reference suite's three-constituent code, against the compiled
    reference: decode hard decisions and soDecode soft outputs."""
    import fecl_b200 as F
    from oracle import ref
    if not ref.available():
        pytest.skip("reference library not built")
    perms = [ARRAYS["perm_1024"], ARRAYS["perm_512"], ARRAYS["perm_even_512"]]
    sf = [[0.7, 0.8, 0.9, 1.0], [0.75], [0.9]]
    dec = F.Turbo.DecoderOptions().algorithm(alg).iterations(4).scheduling([F.Turbo.Stage(a, t) for a, t in stages])
    dec.scalingFactor(sf)
    code = F.Turbo(F.Turbo.EncoderOptions([F.Trellis(*s) for s in SUITE3], perms).termination(0), dec)
    rc = ref.RefCodec.turbo(SUITE3, perms, 0, alg, 0, 4)
    rc.set_turbo_schedule(stages, alg, 4, np.asarray([[0.7, 0.8, 0.9, 1.0], [0.75] * 4, [0.9] * 4]))
    msg = np.random.default_rng(90).integers(0, 2, 6 * code.msgSize()).astype(np.uint8)
    llr = distort(code.encode(msg), -1.0, 91).astype(np.float32).astype(np.float64)
    want = rc.decode(llr)
    out = rc.so_decode(llr, outputs=("msg", "syst", "parity", "state"))
    assert_hard_parity(code.decode(llr), want, msg, code.msgSize(), ref_app=out["msg"])
    got = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output().msg().syst().parity().state())
    ok = frame_ok((out["msg"] > 0).astype(np.uint8), msg, code.msgSize())
    for k, size in (("msg", code.msgSize()), ("syst", code.systSize()), ("parity", code.paritySize()),
                    ("state", code.stateSize())):
        assert_soft_parity(getattr(got, k)(), out[k], ok, size, what=k, exact=alg == 0)


@pytest.mark.parametrize("sched", [0, 1])
@pytest.mark.parametrize("alg", [2, 1, 0])
def test_windowed_soDecode_and_parallel_match_reference(alg, sched, has_ref):
    """LTE soDecode (with a-priori and state inputs, every soft output) and Parallel
    scheduling on the windowed kernel against the compiled FP64 reference on the same
    L-values, under the parity rules: hard decisions equal in every frame the
    reference decodes, soft outputs within 1e-4 relative there.  With the Linear
    algorithm the windowed kernel's soft outputs are also held to the generic kernel's
    (the reference's operation order in FP32) under the strict tail bound, so the
    Linear tail allowance against FP64 covers FP32 itself, not the windowing."""
    if not has_ref:
        pytest.skip("the compiled reference (oracle/_ref) is not built")
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    from oracle import ref
    K, n = 1024, 24
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(alg).iterations(5).scheduling(sched))
    msg = ch.random_bits(n * K, 70 + alg)
    llr = ch.awgn_llr(code.encode(msg), 1.2, K / code.paritySize(), 70 + alg, np.float32)
    syst = (0.05 * ch.awgn_llr(ch.random_bits(n * code.systSize(), 9), 0.0, 1.0, 9)).astype(np.float32)
    rc = ref.RefCodec.turbo([([4], [[0o15]], [0o13])], [np.arange(K), F.Turbo.Lte3Gpp.interleaver(K)], 0, alg, sched, 5,
                            workgroup=8)
    r_first = rc.so_decode(llr, outputs=("state",))
    state_in = r_first["state"].astype(np.float32)
    r_so = rc.so_decode(llr, syst=syst, state=state_in, outputs=("msg", "syst", "parity", "state"))
    r_bits, r_app = rc.decode(llr), rc.so_decode(llr, outputs=("msg",))["msg"]

    def run(kernel):
        code.setKernel(kernel)
        first = code.soDecode(F.Codec.Input().parity(llr), F.Codec.Output(np.float32).state())
        so = code.soDecode(F.Codec.Input().parity(llr).syst(syst).state(state_in),
                           F.Codec.Output(np.float32).msg().syst().parity().state())
        return code.decode(llr), (first.state(), so.msg(), so.syst(), so.parity(), so.state())

    bits, outs = run("auto")
    assert_hard_parity(bits, r_bits, msg, K, ref_app=r_app)
    ok = frame_ok(r_app > 0, msg, K)
    assert ok.sum() >= n // 3
    names = ("state", "msg", "syst", "parity", "state2")
    sizes = (code.stateSize(), K, code.systSize(), code.paritySize(), code.stateSize())
    refs = (r_first["state"], r_so["msg"], r_so["syst"], r_so["parity"], r_so["state"])
    for name, a, b, size in zip(names, outs, refs, sizes):
        assert_soft_parity(a, b, ok, size, what=name, exact=(alg == 0), linear=(alg == 1))
    if alg == 1:
        _, gen = run("generic")
        for name, a, b, size in zip(names, outs, gen, sizes):
            assert_soft_parity(a, b, ok, size, what=name + " vs generic")


def test_tune_window(has_ref):
    """The window autotuner picks one of the equivalent shapes on the caller's inputs,
    remembers it for the same (K, frames, options), and the tuned decoder still meets
    the parity rules against the FP64 reference."""
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    from oracle import checker
    K, n = 2048, 48
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6).scheduling(F.Serial))
    msg = ch.random_bits(n * K, 91)
    llr = ch.awgn_llr(code.encode(msg), 0.7, K / code.paritySize(), 91, np.float32)
    d_llr = torch.from_numpy(llr).cuda()
    segs, train = code.tuneWindow(d_llr)
    assert segs in (0, 32, 64, 128) and train in (48, 64, 80, 96, 128)
    assert code.tuneWindow(d_llr) == (segs, train)
    bits = code.decode(llr)
    ref_bits, ref_app = checker.turbo_lte_decode(K, F.Approximate, 6, F.Serial, llr)
    assert_hard_parity(bits, ref_bits, msg, K, ref_app=ref_app)
