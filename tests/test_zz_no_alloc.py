"""The allocation-free LTE turbo entry point, fecl_lte_turbo_decode_noalloc.

It exists for callers that cannot allocate device memory once running (a pipeline
with a memory budget fixed at start-up, a real-time thread that must not block in
cudaMalloc, a plug-in host that owns the memory pool).  Called through the C-ABI, it
must give the same bits as the allocating entry point (fecl_decode on an LTE codec),
on two calls in a row over the shared static scratch, and reject batches beyond its
scratch.  This file sorts last so that a run stopping at the first failure has run
every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_decode_on_two_calls():
    import torch
    import fecl_b200 as F
    from fecl_b200 import _lib
    from fecl_b200 import channel as ch

    K, n = 6144, 48
    code = F.Turbo.lte(K, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6).scheduling(F.Serial))
    stream = torch.cuda.current_stream()
    for call, seed in enumerate((501, 502)):
        msg = ch.random_bits(n * K, seed)
        llr = ch.awgn_llr(code.encode(msg), 0.7 + 0.2 * call, K / code.paritySize(), seed, np.float32)
        d_llr = torch.from_numpy(llr).cuda()
        expected = code.decode(d_llr).cpu().numpy()
        out = torch.full((n * K,), 7, dtype=torch.uint8, device="cuda")
        rc = _lib.lib.fecl_lte_turbo_decode_noalloc(K, F.Approximate, 6, C.c_void_p(d_llr.data_ptr()), _lib.F32, n,
                                                    C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == _lib.OK, _lib.lib.fecl_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got, expected), "call %d: %d bits differ" % (call, int(np.sum(got != expected)))


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
