"""Frame-error-rate sweep of the DVB-S2 normal-frame decoder across message precisions.

The sweep: DVB-S2 normal frames (n = 64800) at rates 1/2, 3/4 and 9/10, 512 frames
per point, seeded BPSK/AWGN at Eb/N0 = 1.0, 1.25, ..., 4.0 dB, normalised min-sum
(scaling 0.75), at most 50 iterations with the syndrome stop, FP32 L-values.  The
same frames are decoded with FP32, FP16 and saturated int8 message storage, and by
the FP64 CPU decoder of the reference (the oracle).

How precision loss is stated in dB: every frame's noise draws are fixed by its
seed, so `sweep_llr(..., shift_db=d)` is the same noise realisation at a
(d dB) better channel.  "Loses at most d dB" is then checked pointwise and with
low variance: the decoder's FER at Eb/N0 + d is no larger than the oracle's FER at
Eb/N0, on the same noise.  `threshold_db` interpolates the Eb/N0 where a FER curve
crosses a target, for reporting.

The reference's benchmark harness likewise decodes random frames at each point of
an SNR grid (benchmark/Cpp/main.cpp:73-83, :244-254); it times the decodes and
keeps no error counts.
"""
import math

import numpy as np

from . import channel as ch

RATES = ((1, 2), (3, 4), (9, 10))
EBN0_DB = tuple(1.0 + 0.25 * i for i in range(13))
FRAMES = 512
N = 64800
ITERATIONS = 50
SCALING = 0.75
SHIFT_DB = 0.1


def seed(rate_index, point_index):
    """Seed of the message bits and of the noise at one sweep point."""
    return 70001 + 1000 * int(rate_index) + int(point_index)


def code(rate_index, precision=0):
    """The sweep's decoder for one rate: normalised min-sum, at most 50 iterations,
    message storage `precision` (0 FP32, 1 FP16, 2 int8)."""
    from fractions import Fraction

    from . import Approximate, Ldpc
    num, den = RATES[rate_index]
    H = Ldpc.DvbS2.matrix(N, Fraction(num, den))
    dec = Ldpc.DecoderOptions().algorithm(Approximate).iterations(ITERATIONS).scalingFactor(SCALING).precision(precision)
    return Ldpc(Ldpc.EncoderOptions(H), dec)


def sweep_msg(K, rate_index, point_index, frames=FRAMES):
    return ch.random_bits(frames * K, seed(rate_index, point_index))


def sweep_llr(codeword, K, rate_index, point_index, shift_db=0.0, dtype=np.float32):
    """FP32 L-values of one sweep point; shift_db moves Eb/N0 with the same draws."""
    ebn0 = EBN0_DB[point_index] + shift_db
    return ch.awgn_llr(codeword, ebn0, K / N, seed(rate_index, point_index), dtype)


def frame_fails(bits, msg, frames):
    """Per-frame failure flags: any decided message bit differs."""
    b = np.asarray(bits, dtype=np.uint8).reshape(frames, -1)
    m = np.asarray(msg, dtype=np.uint8).reshape(frames, -1)
    return np.any(b != m, axis=1)


def pack_fails(fails):
    """Failure flags as a hex string (frame i is bit i % 8 of byte i // 8)."""
    return np.packbits(np.asarray(fails, dtype=np.uint8), bitorder="little").tobytes().hex()


def unpack_fails(hexstr, frames):
    b = np.frombuffer(bytes.fromhex(hexstr), dtype=np.uint8)
    return np.unpackbits(b, bitorder="little")[:frames].astype(bool)


def threshold_db(ebn0, fer, target, frames=FRAMES):
    """Eb/N0 where a FER curve first falls to `target`, by linear interpolation of
    log10(FER) between the two grid points that bracket it.  A FER of zero counts
    as half a frame error (the curve's resolution).  None when the curve never
    reaches the target; the first grid point when it starts below it."""
    floor = 0.5 / frames
    lf = [math.log10(max(float(f), floor)) for f in fer]
    lt = math.log10(target)
    if lf[0] <= lt:
        return float(ebn0[0])
    for i in range(1, len(lf)):
        if lf[i] <= lt:
            x0, x1, y0, y1 = ebn0[i - 1], ebn0[i], lf[i - 1], lf[i]
            return float(x0 + (x1 - x0) * (lt - y0) / (y1 - y0))
    return None


def loss_check(fer_shifted, fer_oracle, frames=FRAMES, slack=2):
    """Points where the decoder at Eb/N0 + shift has more frame errors than the
    oracle at Eb/N0, beyond `slack` frames: [(point index, decoder errors, oracle
    errors)].  Empty means the decoder loses at most the shift."""
    bad = []
    for i, (a, b) in enumerate(zip(fer_shifted, fer_oracle)):
        ea, eb = int(round(a * frames)), int(round(b * frames))
        if ea > eb + slack:
            bad.append((i, ea, eb))
    return bad
