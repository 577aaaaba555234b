"""Golden fixtures made by tests/golden/make_golden.py from the reference FeCl
library compiled from its sources, plus helpers that rebuild each case's inputs
from its recipe (code, seed, Eb/N0, frames)."""
import hashlib
import json
import os
from fractions import Fraction

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(HERE, "golden.json")) as _f:
    GOLDEN = json.load(_f)
ARRAYS = np.load(os.path.join(HERE, "golden_arrays.npz"))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def check_matrix(spec):
    import fecl_b200 as F
    if spec["family"] == "dvbs2":
        return F.Ldpc.DvbS2.matrix(spec["n"], Fraction(*spec["rate"]))
    if spec["family"] == "gallager":
        return F.Ldpc.Gallager.matrix(spec["n"], spec["wc"], spec["wr"], spec["seed"])
    raise KeyError(spec["family"])


LTE = ([4], [[0o15]], [0o13])
T17 = ([4], [[0o17]], [0o15])
SUITE3 = [T17, ([3, 3], [[0o5, 0o3, 0], [0, 0o3, 0o7]], [0o7, 0o5]), ([4], [[0o17, 0o13]], [0o15])]


def turbo_layout(spec):
    """(trellis specs, interleavers) of a golden turbo case."""
    import fecl_b200 as F
    fam = spec["family"]
    if fam == "lte":
        K = spec["K"]
        return [LTE], [np.arange(K, dtype=np.uint32), F.Turbo.Lte3Gpp.interleaver(K)]
    if fam == "suite2":
        return [T17], [np.arange(1024, dtype=np.uint32), ARRAYS["perm_1024"]]
    if fam == "suite3":
        return SUITE3, [ARRAYS["perm_1024"], ARRAYS["perm_512"], ARRAYS["perm_even_512"]]
    raise KeyError(fam)


def case_inputs(name, encode):
    """Message bits, codeword bits and FP32-rounded L-values (as float64) of a case;
    `encode` maps message bits to codeword bits."""
    from fecl_b200 import channel as ch
    c = GOLDEN["cases"][name]
    msg = ch.random_bits(c["frames"] * c["msg_size"], c["seed"])
    cw = encode(msg)
    llr = ch.awgn_llr(cw, c["ebn0_db"], c["msg_size"] / c["parity_size"], c["seed"], np.float32).astype(np.float64)
    return msg, cw, llr


def hard(name):
    c = GOLDEN["cases"][name]
    return np.unpackbits(ARRAYS[name + "__hard"])[: c["frames"] * c["msg_size"]]
