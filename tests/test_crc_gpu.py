"""CRC-24A / CRC-24B (3GPP TS 36.212 section 5.1.1) on the GPU, and the LTE turbo
decoder's CRC stop: a frame that stops after t iterations has exactly the bits of a
decode with t iterations; frames whose CRC never passes run every iteration."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _crc_ref(bits, poly):
    """Bitwise CRC register over a 0/1 sequence, most significant bit first."""
    r = 0
    for b in bits:
        fb = ((r >> 23) & 1) ^ int(b)
        r = (r << 1) & 0xFFFFFF
        if fb:
            r ^= poly
    return r


@pytest.mark.parametrize("kind,poly", [(1, 0x864CFB), (2, 0x800063)])
def test_attach_and_check(kind, poly):
    import torch
    import fecl_b200 as F
    rng = np.random.default_rng(95)
    n, L = 9, 1000
    bits = torch.from_numpy(rng.integers(0, 2, n * L).astype(np.uint8)).cuda()
    out = F.crc24_attach(bits, kind, n)
    o = out.cpu().numpy().reshape(n, L + 24)
    assert np.array_equal(o[:, :L].ravel(), bits.cpu().numpy())
    for f in range(n):
        r = _crc_ref(o[f, :L], poly)
        assert [int(x) for x in o[f, L:]] == [(r >> (23 - k)) & 1 for k in range(24)]
        assert _crc_ref(o[f], poly) == 0
    assert bool(F.crc24_check(out, kind, n).all())
    bad = out.clone()
    bad[3 * (L + 24) + 17] ^= 1
    ok = F.crc24_check(bad, kind, n).cpu().numpy()
    assert not ok[3] and ok.sum() == n - 1


@pytest.mark.parametrize("K", [40, 1024, 6144])
def test_lte_crc_stop_equals_shorter_decodes(K):
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    I = 8
    dec = F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(I)
    stop = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(I).crc(F.CRC24A))
    full = F.Turbo.lte(K, dec)
    n = 48
    info = torch.from_numpy(ch.random_bits(n * (K - 24), 96)).cuda()
    msg = F.crc24_attach(info, F.CRC24A, n)
    cw = stop.encode(msg)
    ebn0 = np.repeat(np.linspace(0.2, 2.5, 8), n // 8)
    llr = torch.from_numpy(ch.awgn_llr_per_frame(cw.cpu().numpy(), stop.paritySize(), ebn0, K / stop.paritySize(), 97,
                                                 np.float32)).cuda()
    bits, its = stop.decode(llr, iterations=True)
    its = its.cpu().numpy()
    assert its.min() >= 1 and its.max() <= I and len(set(its.tolist())) > 1
    ok = F.crc24_check(bits, F.CRC24A, n).cpu().numpy()
    b = bits.cpu().numpy().reshape(n, K)
    x = llr.cpu().numpy().reshape(n, -1)
    for t in sorted(set(its.tolist())):
        shorter = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(t))
        sel = np.nonzero(its == t)[0]
        ref = shorter.decode(x[sel].ravel()).reshape(len(sel), K)
        assert np.array_equal(b[sel], ref), t
        if t < I:
            assert ok[sel].all()
    # the mixed-K batch kernel (64 segments per frame) applies the same stop: the
    # same bits and counts as a decode with 64 segments (a batch of a few frames
    # decodes with 128 by default, which rounds differently)
    out = torch.zeros_like(bits)
    it2 = torch.zeros(n, dtype=torch.int32, device="cuda")
    F.Batch([(stop, llr, out, it2)]).run()
    torch.cuda.synchronize()
    stop.setWindowSegments(64)
    bits64, its64 = stop.decode(llr, iterations=True)
    assert torch.equal(out, bits64) and np.array_equal(it2.cpu().numpy(), its64.cpu().numpy())
    # without the CRC stop every frame runs all iterations
    assert (full.decode(llr, iterations=True)[1].cpu().numpy() == I).all()


def test_server_applies_the_crc_stop():
    """Requests of a CRC-stopping LTE codec through the decode server: the same bits
    and the same iteration counts as the codec's own decode (so the stop fired in the
    server's batches too), with some frames stopping before the last iteration."""
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    I = 8
    codes = [F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(I).crc(F.CRC24A))
             for K in (1024, 6144)]
    srv = F.Server(device_budget=2 << 30, max_batch_frames=64, slots=2)
    reqs = []
    for i, code in enumerate(codes * 6):
        K = code.msgSize()
        info = ch.random_bits(3 * (K - 24), 200 + i)
        msg = F.crc24_attach(torch.from_numpy(info).cuda(), F.CRC24A, 3).cpu().numpy()
        llr = ch.awgn_llr(code.encode(msg), 0.6 + 0.3 * (i % 5), K / code.paritySize(), 200 + i, np.float32)
        reqs.append((code, llr))
    tickets = [srv.submit(c, llr, iterations=True) for c, llr in reqs]
    stopped_early = 0
    for (c, llr), t in zip(reqs, tickets):
        bits, its, _ = srv.wait(t)
        ref_bits, ref_its = c.decode(llr, iterations=True)
        assert np.array_equal(bits, ref_bits) and np.array_equal(its, ref_its)
        stopped_early += int(np.sum(its < I))
    srv.close()
    assert stopped_early > 0


def _generic_code(which, iterations, crc):
    import fecl_b200 as F
    from goldens import ARRAYS, T17
    if which == "lte-parallel":
        d = F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(iterations).scheduling(F.Parallel)
        if crc:
            d = d.crc(F.CRC24A)
        return F.Turbo.lte(1024, d)
    d = F.Turbo.DecoderOptions().algorithm(F.Linear).iterations(iterations).scheduling(F.Serial)
    if crc:
        d = d.crc(F.CRC24A)
    perms = [np.arange(1024, dtype=np.uint32), ARRAYS["perm_1024"]]
    return F.Turbo(F.Turbo.EncoderOptions([F.Trellis(*T17)], perms).termination(0), d)


@pytest.mark.parametrize("which", ["lte-parallel", "t17-serial-linear"])
def test_generic_kernel_crc_stop_equals_shorter_decodes(which):
    """The CRC stop in the generic turbo kernel (any code, any scheduling): a frame
    that stops after t iterations has exactly the bits of a decode with t iterations,
    its CRC passes, and frames whose CRC never passes run every iteration."""
    import torch
    import fecl_b200 as F
    from fecl_b200 import channel as ch
    I = 8
    stop = _generic_code(which, I, True)
    K, P = stop.msgSize(), stop.paritySize()
    n = 40
    info = torch.from_numpy(ch.random_bits(n * (K - 24), 210)).cuda()
    msg = F.crc24_attach(info, F.CRC24A, n).cpu().numpy()
    ebn0 = np.repeat(np.linspace(0.0, 2.5, 8), n // 8)
    llr = ch.awgn_llr_per_frame(stop.encode(msg), P, ebn0, K / P, 211, np.float32)
    bits, its = stop.decode(llr, iterations=True)
    assert its.min() >= 1 and its.max() <= I and len(set(its.tolist())) > 1
    ok = F.crc24_check(torch.from_numpy(bits).cuda(), F.CRC24A, n).cpu().numpy()
    b = bits.reshape(n, K)
    x = llr.reshape(n, -1)
    for t in sorted(set(its.tolist())):
        sel = np.nonzero(its == t)[0]
        ref = _generic_code(which, t, False).decode(x[sel].ravel()).reshape(len(sel), K)
        assert np.array_equal(b[sel], ref), t
        if t < I:
            assert ok[sel].all()
