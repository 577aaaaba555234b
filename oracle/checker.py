"""Test infrastructure: the CPU checker the smoke test, the test-suite and bench.py's
CPU baseline compare against.

It runs the reference decoder compiled from FeCl's sources (oracle/_ref, via
ref.py).  Where that library is absent it runs the C restatement (fecl_oracle.c,
via restated.py), which the test-suite pins to the reference's outputs.
"""
import numpy as np

from . import ref

TIE_REL = 1e-9  # a-posteriori magnitudes below TIE_REL * max |APP| are flagged ties


def _backend():
    if ref.available():
        return "reference"
    from . import restated
    if restated.available():
        return "restated"
    raise RuntimeError("no CPU oracle is built (make -C oracle)")


def ldpc_decode(H, algorithm, iterations, scaling, llr, workgroup=8):
    """Hard bits and a-posteriori message L-values of the reference BP decoder."""
    llr = np.asarray(llr, dtype=np.float64)
    if _backend() == "reference":
        rc = ref.RefCodec.ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx, algorithm, iterations, (scaling,), workgroup)
        return rc.decode(llr), rc.so_decode(llr, outputs=("msg",))["msg"]
    from . import restated
    return restated.ldpc_decode(H, algorithm, iterations, scaling, llr)


def turbo_lte_decode(K, algorithm, iterations, scheduling, llr, workgroup=8):
    from fecl_b200 import Turbo
    llr = np.asarray(llr, dtype=np.float64)
    perm = Turbo.Lte3Gpp.interleaver(K)
    if _backend() == "reference":
        rc = ref.RefCodec.turbo([([4], [[0o15]], [0o13])], [np.arange(K), perm], 0, algorithm, scheduling, iterations,
                                workgroup=workgroup)
        return rc.decode(llr), rc.so_decode(llr, outputs=("msg",))["msg"]
    from . import restated
    return restated.turbo_lte_decode(K, algorithm, iterations, scheduling, llr)


def flagged_ties(app):
    """Outputs whose reference a-posteriori value is (near) zero: hard decisions
    there are a coin toss between FP32 and FP64 and are not compared."""
    a = np.abs(np.asarray(app, dtype=np.float64))
    fin = a[np.isfinite(a)]
    m = fin.max() if fin.size else 0.0
    return (a == 0.0) | (a < TIE_REL * m)


def assert_hard_match(bits, ref_bits, ref_app, what="", strict_positive=False):
    bits = np.asarray(bits).ravel()
    ref_bits = np.asarray(ref_bits).ravel()
    ties = flagged_ties(ref_app)
    bad = (bits != ref_bits) & ~ties
    if bad.any():
        idx = np.nonzero(bad)[0][:8]
        raise AssertionError("%s: %d hard decisions differ from the oracle outside flagged ties (first at %s)"
                             % (what, int(bad.sum()), idx.tolist()))
