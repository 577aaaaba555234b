"""The allocation-free LTE turbo entry point, fecl_lte_turbo_decode_noalloc.

It exists for callers that cannot allocate device memory once running (a pipeline
with a memory budget fixed at start-up, a real-time thread that must not block in
cudaMalloc, a plug-in host that owns the memory pool).  Called through the C-ABI, it
must give the same bits as the allocating entry point (fecl_decode on an LTE codec),
on two calls in a row over the shared static scratch -- also when a small block
follows a large one, so that nothing a previous call left beyond the new K is read --
and reject batches beyond its scratch.  This file sorts last so that a run stopping
at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DTYPES = {"f32": (np.float32, "F32"), "f16": (np.float16, "F16"), "f64": (np.float64, "F64")}


def _decode_pair(K, n, alg, dtype, seed, ebn0):
    """(allocating decode, allocation-free decode) of the same L-values."""
    import torch
    import fecl_b200 as F
    from fecl_b200 import _lib
    from fecl_b200 import channel as ch
    np_t, lib_t = DTYPES[dtype]
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(alg).iterations(6).scheduling(F.Serial))
    msg = ch.random_bits(n * K, seed)
    llr = ch.awgn_llr(code.encode(msg), ebn0, K / code.paritySize(), seed, np_t)
    d_llr = torch.from_numpy(llr).cuda()
    expected = code.decode(d_llr).cpu().numpy()
    out = torch.full((n * K,), 7, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _lib.lib.fecl_lte_turbo_decode_noalloc(K, alg, 6, C.c_void_p(d_llr.data_ptr()), getattr(_lib, lib_t), n,
                                                C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == _lib.OK, _lib.lib.fecl_last_error()
    torch.cuda.synchronize()
    return expected, out.cpu().numpy()


def test_noalloc_matches_allocating_decode_on_two_calls():
    import fecl_b200 as F
    K, n = 6144, 48
    for call, seed in enumerate((501, 502)):
        expected, got = _decode_pair(K, n, F.Approximate, "f32", seed, 0.7 + 0.2 * call)
        assert np.array_equal(got, expected), "call %d: %d bits differ" % (call, int(np.sum(got != expected)))


@pytest.mark.parametrize("alg,dtype", [("Exact", "f16"), ("Linear", "f64"), ("Approximate", "f16")])
def test_noalloc_small_block_after_a_large_one(alg, dtype):
    """K=6144 then K=40 (whose padded tables are shorter) then K=1008, each equal to
    the allocating decode of the same L-values."""
    import fecl_b200 as F
    a = getattr(F, alg)
    for call, (K, n) in enumerate(((6144, 20), (40, 64), (1008, 33))):
        expected, got = _decode_pair(K, n, a, dtype, 600 + call, 0.8)
        assert np.array_equal(got, expected), "K=%d: %d bits differ" % (K, int(np.sum(got != expected)))


def test_noalloc_capacity_edge():
    """At K=6144 the scratch holds exactly the frame count the error message names:
    that many frames decode, one more is rejected."""
    import re
    import torch
    import fecl_b200 as F
    from fecl_b200 import _lib
    K = 6144
    big = torch.zeros(1, dtype=torch.float32, device="cuda")
    rc = _lib.lib.fecl_lte_turbo_decode_noalloc(K, 2, 6, C.c_void_p(big.data_ptr()), _lib.F32, 1 << 20,
                                                C.c_void_p(big.data_ptr()), None)
    assert rc == _lib.EINVAL
    cap = int(re.search(rb"at most (\d+) frames", _lib.lib.fecl_last_error()).group(1))
    assert cap >= 32
    expected, got = _decode_pair(K, cap, F.Approximate, "f32", 777, 0.7)
    assert np.array_equal(got, expected)
    llr = torch.zeros((cap + 1) * (3 * K + 12), dtype=torch.float32, device="cuda")
    out = torch.zeros((cap + 1) * K, dtype=torch.uint8, device="cuda")
    rc = _lib.lib.fecl_lte_turbo_decode_noalloc(K, 2, 6, C.c_void_p(llr.data_ptr()), _lib.F32, cap + 1,
                                                C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.EINVAL


def test_noalloc_rejects_batches_beyond_its_scratch():
    import torch
    from fecl_b200 import _lib
    K, n = 6144, 4096
    llr = torch.zeros(n * (3 * K + 12), dtype=torch.float32, device="cuda")
    out = torch.zeros(n * K, dtype=torch.uint8, device="cuda")
    rc = _lib.lib.fecl_lte_turbo_decode_noalloc(K, 2, 6, C.c_void_p(llr.data_ptr()), _lib.F32, n,
                                                C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.EINVAL
    assert b"scratch" in _lib.lib.fecl_last_error()
    assert _lib.lib.fecl_lte_turbo_decode_noalloc(41, 2, 6, C.c_void_p(llr.data_ptr()), _lib.F32, 1,
                                                  C.c_void_p(out.data_ptr()), None) == _lib.EINVAL
