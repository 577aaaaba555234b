"""Parity rules of the GPU tests against the FP64 oracle.

Hard decisions.  In every frame the oracle decodes correctly (its bits equal the
transmitted message), the GPU's FP32 hard decisions must equal the oracle's bit for
bit, outside flagged ties (|APP| below 1e-9 of the frame's largest |APP|, or zero).
Frames the oracle fails to decode are chaotic under any change of rounding: there
the GPU must fail too (matched frame errors) and its bit disagreements must stay a
small fraction of the frame.

Soft outputs.  In oracle-decoded frames, at least 99.9% of the FP32 soft outputs
must agree with the oracle within |gpu - ref| <= rtol * max(|ref|, 1), rtol = 1e-4,
and every one within 1e-2 on the same scale; the floor of 1 keeps values near
zero, where a relative error is meaningless, to an absolute 1e-4.  The tail
allowance is what FP32 itself costs: an FP32 build of the C restatement, which
keeps the reference's operation order exactly, lands on the FP64 reference with
p99.9 errors of 2e-6 (Linear) to 6e-5 (min-sum) but single outliers up to ~1e-3,
from decisions that flip on rounding: the min/max selections of min-sum and
max-log, and the step of the Linear table at |x| = 3.5 (src/detail/LinearTable.h:68-74).  The reference's Exact boxplus works in the tanh domain, whose product
rounds to +-1 once every other input of a check exceeds ~38 in magnitude, and then
returns +-inf (src/detail/LlrMetrics.h:136-138); the FP32 kernel computes the same
boxplus in the phi domain and stays finite, so reference infinities compare by
sign and by magnitude above SATURATED.  The Linear table (src/detail/LinearTable.h:56-81) is discontinuous
at 3.5, where it drops by log(1 + e^-3.5) = 0.0297: an FP32 log-sum whose argument
lands on the other side of the step than the reference's jumps by that much, and in a
turbo decode the jump spreads over the iterations, so with the Linear algorithm the
tail bound is LINEAR_TAIL_MAX (see there).  Below the rounding to +-1 the tanh form is
already inexact: with FP64 the boxplus output c carries an error of about
1e-16 * exp(|c|) / 2, above 1e-4 relative once |c| > 32, so with the Exact
algorithm every reference value beyond EXACT_RELIABLE compares the same way.
"""
import numpy as np

RTOL = 1e-4
TIE_REL = 1e-9
SATURATED = 30.0
EXACT_RELIABLE = 32.0


def frame_ok(bits, msg, k):
    return ~np.any(np.asarray(bits).reshape(-1, k) != np.asarray(msg).reshape(-1, k), axis=1)


def ties(app, k):
    a = np.abs(np.asarray(app, np.float64)).reshape(-1, k)
    m = a.max(axis=1, keepdims=True)
    return ((a == 0) | (a < TIE_REL * m)).ravel()


def assert_hard_parity(gpu_bits, ref_bits, msg, k, ref_app=None, max_bad_fraction=0.02):
    gpu_bits = np.asarray(gpu_bits).ravel()
    ref_bits = np.asarray(ref_bits).ravel()
    ok = frame_ok(ref_bits, msg, k)
    diff = (gpu_bits != ref_bits)
    if ref_app is not None:
        diff &= ~ties(ref_app, k)
    diff = diff.reshape(-1, k)
    bad_converged = diff[ok].sum()
    assert bad_converged == 0, "%d hard decisions differ in %d oracle-decoded frames" % (bad_converged, int(ok.sum()))
    gpu_ok = frame_ok(gpu_bits, msg, k)
    assert np.array_equal(gpu_ok, ok), "frame errors differ: gpu %s ref %s" % (np.nonzero(~gpu_ok)[0], np.nonzero(~ok)[0])
    if (~ok).any():
        frac = diff[~ok].mean()
        assert frac <= max_bad_fraction, "%.4f of bits differ in failed frames" % frac
    return int(ok.sum())


def soft_error(gpu, ref, frame_mask=None, size=None, reliable=np.inf):
    g = np.asarray(gpu, np.float64).ravel()
    r = np.asarray(ref, np.float64).ravel()
    inf = ~np.isfinite(r) | (np.abs(r) > reliable)
    rr = np.where(inf, 0.0, r)
    err = np.abs(g - rr) / np.maximum(np.abs(rr), 1.0)
    err[inf] = np.where((np.sign(g[inf]) == np.sign(r[inf])) & (np.abs(g[inf]) >= SATURATED), 0.0, np.inf)
    if frame_mask is not None:
        err = err.reshape(-1, size)[frame_mask].ravel()
    return err


TAIL_FRACTION = 1e-3
TAIL_MAX = 1e-2
# The Linear log-sum table (src/detail/LinearTable.h:56-81) steps from log(1 + e^-3.5)
# to 0 at |x| = 3.5.  Where rounding puts an FP32 argument on the other side of the
# step than the FP64 reference's, that log-sum jumps by 0.0297, and over the
# iterations of a turbo decode the jump spreads to the a-posteriori values of nearby
# bits: both FP32 turbo kernels (the reference's operation order and the windowed
# one, with identical values) show single tail values up to 2.4e-2 scaled error
# against the FP64 reference.  With the Linear algorithm the tail bound is therefore
# LINEAR_TAIL_MAX; the bulk rule (99.9 % within 1e-4 relative) is unchanged.
LINEAR_TAIL_MAX = 5e-2


def assert_soft_parity(gpu, ref, frame_mask=None, size=None, rtol=RTOL, what="", exact=False, linear=False):
    err = soft_error(gpu, ref, frame_mask, size, EXACT_RELIABLE if exact else np.inf)
    if err.size == 0:
        return 0.0
    worst = float(err.max())
    over = float(np.mean(err > rtol))
    tail_ok = worst <= (LINEAR_TAIL_MAX if linear else TAIL_MAX)
    assert over <= TAIL_FRACTION and tail_ok, "%s: %.2e of values beyond %.0e (max scaled error %.3g, p99.9 %.3g)" % (
        what, over, rtol, worst, float(np.quantile(err, 0.999)))
    return worst
