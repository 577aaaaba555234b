#!/usr/bin/env python3
"""Generate fer_sweep_oracle.json: the frame failures of the reference FeCl decoder
(compiled from its sources, oracle/_ref; FP64 arithmetic) on the FER sweep defined
in fecl_b200/fer.py.

For each rate (1/2, 3/4, 9/10 of the DVB-S2 normal frame) and each Eb/N0 point
(1.0 to 4.0 dB in 0.25 dB steps) it decodes the 512 seeded frames with normalised
min-sum (0.75, at most 50 iterations, syndrome stop), from the FP32-rounded
L-values the GPU decoders see, and records which frames fail (packed bit flags).
The GPU tests compare the decoders at FP32, FP16 and int8 message precision with
these flags, so they need neither the reference sources nor its compiled library.

The reference's own DVB-S2 builder is correct only for (64800, 1/2), so the check
matrix given to it is the standard one from fecl_b200's tables (identical edge for
edge at (64800, 1/2)); its encoder and decoder are the reference's.

Run from the repository root (about 5 minutes on 8 threads):
    python tests/golden/make_fer_sweep.py
"""
import json
import os
import sys
import time
from fractions import Fraction

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from fecl_b200 import fer  # noqa: E402  (host-side code builders only; no GPU needed)
from oracle import ref as R  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    import fecl_b200 as F
    out = {"generator": "tests/golden/make_fer_sweep.py",
           "decoder": "reference FeCl compiled from its sources, FP64, Approximate (min-sum), scaling 0.75, "
                      "<=50 iterations with its syndrome stop, 8 worker threads",
           "n": fer.N, "frames": fer.FRAMES, "iterations": fer.ITERATIONS, "scaling": fer.SCALING,
           "ebn0_db": list(fer.EBN0_DB), "rates": {}}
    for r, (num, den) in enumerate(fer.RATES):
        H = F.Ldpc.DvbS2.matrix(fer.N, Fraction(num, den))
        rc = R.RefCodec.ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx, F.Approximate, fer.ITERATIONS, (fer.SCALING,),
                             workgroup=8)
        K = rc.msg
        fails, rates = [], []
        for p in range(len(fer.EBN0_DB)):
            t = time.time()
            msg = fer.sweep_msg(K, r, p)
            cw = rc.encode(msg)
            llr = fer.sweep_llr(cw, K, r, p).astype(np.float64)
            f = fer.frame_fails(rc.decode(llr), msg, fer.FRAMES)
            fails.append(fer.pack_fails(f))
            rates.append(float(f.mean()))
            print("rate %d/%d  Eb/N0 %.2f dB  FER %.4f  (%.1f s)" % (num, den, fer.EBN0_DB[p], f.mean(), time.time() - t),
                  flush=True)
        out["rates"]["%d/%d" % (num, den)] = {"K": K, "fails": fails, "fer": rates}
    with open(os.path.join(HERE, "fer_sweep_oracle.json"), "w") as fo:
        json.dump(out, fo, indent=1)
        fo.write("\n")


if __name__ == "__main__":
    main()
