"""The C-ABI library: it loads, exports every symbol include/fecl_b200.h declares,
and reports the reference's errors on the host-side calls (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "fecl_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fecl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import fecl_b200
    lib = C.CDLL(fecl_b200.lib_path)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from fecl_b200 import _lib
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_version_and_errors():
    from fecl_b200 import _lib
    assert b"sm_100a" in _lib.lib.fecl_version()
    assert _lib.lib.fecl_strerror(_lib.EINVAL) == b"invalid argument"


def test_sizes_of_the_lte_code():
    import fecl_b200 as F
    t = F.Turbo.lte(6144)
    # src/Turbo.h:38-53 layout: msg K, syst K+6, parity 3K+12, state 2(K+3)
    assert (t.msgSize(), t.systSize(), t.paritySize(), t.stateSize()) == (6144, 6150, 18444, 12294)


def test_bad_sizes_raise_like_the_reference():
    """test/Cpp/operations.h:94-104, :147-157, :385-432: size mismatches throw."""
    import fecl_b200 as F
    t = F.Turbo.lte(40)
    with pytest.raises(ValueError):
        t.encode(np.zeros(t.msgSize() + 1, np.uint8))
    with pytest.raises(ValueError):
        t.decode(np.zeros(t.paritySize() + 1))
    with pytest.raises(ValueError):
        t.soDecode(F.Codec.Input().parity(np.zeros(t.paritySize() + 1)), F.Codec.Output().syst())
    with pytest.raises(ValueError):
        t.soDecode(F.Codec.Input().parity(np.zeros(t.paritySize())).syst(np.zeros(t.systSize() + 1)),
                   F.Codec.Output().syst())
    with pytest.raises(ValueError):
        t.soDecode(F.Codec.Input().parity(np.zeros(t.paritySize())).state(np.zeros(t.stateSize() + 1)),
                   F.Codec.Output().syst())
    with pytest.raises(ValueError):
        t.soDecode(F.Codec.Input(), F.Codec.Output().syst())


def test_invalid_options_raise():
    import fecl_b200 as F
    with pytest.raises(ValueError):
        F.Turbo.Lte3Gpp.interleaver(41)
    with pytest.raises(ValueError):
        F.Ldpc.DvbS2.matrix(16200, 0.9)  # 9/10 exists only for normal frames
    with pytest.raises(ValueError):
        F.Ldpc.DvbS2.matrix(1000, 0.5)
    H = F.Ldpc.Gallager.matrix(96, 3, 6, 1)
    # src/detail/Ldpc.cpp:71-73: a scaling vector must have 1 or `iterations` entries
    with pytest.raises(ValueError):
        F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().iterations(5).scalingFactor({0: [1.0, 0.5]}))
    # src/detail/Turbo.cpp:127-135: one row, or one row per constituent of 1 or `iterations` entries
    with pytest.raises(ValueError):
        F.Turbo.lte(40, F.Turbo.DecoderOptions().iterations(4).scalingFactor([[1.0], [0.5], [0.7]]))
    with pytest.raises(ValueError):
        F.Turbo.lte(40, F.Turbo.DecoderOptions().iterations(4).scalingFactor([[1.0, 0.5], [0.5, 1.0]]))
    F.Turbo.lte(40, F.Turbo.DecoderOptions().iterations(4).scalingFactor([[1.0, 0.5]]))  # accepted, cycled
    # src/detail/Turbo.cpp:106-124: custom schedules need one transfer list per
    # activation and valid constituent ids
    with pytest.raises(ValueError):
        F.Turbo.lte(40, F.Turbo.DecoderOptions().scheduling([F.Turbo.Stage([0, 1], [[1]])]))
    with pytest.raises(ValueError):
        F.Turbo.lte(40, F.Turbo.DecoderOptions().scheduling([F.Turbo.Stage([2], [[0]])]))
    F.Turbo.lte(40, F.Turbo.DecoderOptions().scheduling([F.Turbo.Stage([1, 0], [[0], [1]])]))
    t = F.Turbo.lte(40)
    with pytest.raises(ValueError):
        t.setWindowTraining(12)
    for segs in (0, 32, 64, 128):  # the window shapes the decoder has
        t.setWindowSegments(segs)
    for segs in (16, 48, 96, 256):
        with pytest.raises(ValueError):
            t.setWindowSegments(segs)


def test_decode_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import fecl_b200 as F
    t = F.Turbo.lte(40)
    with pytest.raises(F.FeclError):
        t.decode(np.zeros(t.paritySize()))


def test_noalloc_rejects_a_frame_count_that_would_wrap_the_scratch_size():
    """A frame count whose byte size wraps around 2^64 (K=40: 1056 B a frame, so
    2^59 + 1 frames wrap to 1056 B) must be rejected before anything is launched."""
    from fecl_b200 import _lib
    dummy = C.c_void_p(256)  # never dereferenced: the call returns before any device work
    for K, n in ((40, (1 << 59) + 1), (6144, (1 << 64) - 1), (6144, 69)):
        rc = _lib.lib.fecl_lte_turbo_decode_noalloc(K, 2, 6, dummy, _lib.F32, n, dummy, None)
        assert rc == _lib.EINVAL, (K, n, rc)
        assert b"scratch" in _lib.lib.fecl_last_error()
