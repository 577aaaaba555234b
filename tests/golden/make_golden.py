#!/usr/bin/env python3
"""Generate the golden fixtures in this directory from the reference FeCl library
compiled from its sources (oracle/_ref, built by `make -C oracle ref`).

The reference ships no golden vectors or fixtures of its own, so these are made by
running it on seeded inputs: every case records its inputs by recipe (code,
seed, Eb/N0, frames), SHA-256 digests of the reference outputs as float64 / byte
arrays (to pin the C restatement bit for bit), packed hard decisions, and FP32
copies of the main soft outputs (for the GPU tolerance tests, which run where the
reference is not available).

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys
from fractions import Fraction

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import fecl_b200 as F  # noqa: E402  (host-side code builders only; no GPU needed)
from fecl_b200 import channel as ch  # noqa: E402
from oracle import ref as R  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def ldpc_case(name, H, algorithm, iterations, scaling, ebn0, frames, seed, keep_state=False):
    rc = R.RefCodec.ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx, algorithm, iterations, (scaling,), workgroup=8)
    msg = ch.random_bits(frames * rc.msg, seed)
    cw = rc.encode(msg)
    llr = ch.awgn_llr(cw, ebn0, rc.msg / rc.parity, seed, np.float32).astype(np.float64)
    hard = rc.decode(llr)
    so = rc.so_decode(llr, outputs=("msg", "syst", "parity", "state"))
    meta = {"kind": "ldpc", "algorithm": algorithm, "iterations": iterations, "scaling": scaling, "ebn0_db": ebn0,
            "frames": frames, "seed": seed, "msg_size": rc.msg, "parity_size": rc.parity, "state_size": rc.state,
            "sha": {"codeword": sha(cw), "hard": sha(hard), **{k: sha(v) for k, v in so.items()}}}
    arrays = {name + "__hard": np.packbits(hard), name + "__msg": so["msg"].astype(np.float32),
              name + "__parity": so["parity"].astype(np.float32)}
    if keep_state:
        arrays[name + "__state"] = so["state"].astype(np.float32)
    return meta, arrays


def turbo_case(name, specs, perms, termination, algorithm, iterations, scheduling, ebn0, frames, seed, scaling=None):
    rc = R.RefCodec.turbo(specs, perms, termination, algorithm, scheduling, iterations, scaling=scaling, workgroup=8)
    msg = ch.random_bits(frames * rc.msg, seed)
    cw = rc.encode(msg)
    llr = ch.awgn_llr(cw, ebn0, rc.msg / rc.parity, seed, np.float32).astype(np.float64)
    hard = rc.decode(llr)
    so = rc.so_decode(llr, outputs=("msg", "syst", "parity", "state"))
    meta = {"kind": "turbo", "algorithm": algorithm, "iterations": iterations, "scheduling": scheduling,
            "termination": termination, "ebn0_db": ebn0, "frames": frames, "seed": seed,
            "scaling": None if scaling is None else np.asarray(scaling).tolist(),
            "msg_size": rc.msg, "syst_size": rc.syst, "parity_size": rc.parity, "state_size": rc.state,
            "sha": {"codeword": sha(cw), "hard": sha(hard), **{k: sha(v) for k, v in so.items()}}}
    arrays = {name + "__hard": np.packbits(hard), name + "__msg": so["msg"].astype(np.float32),
              name + "__state": so["state"].astype(np.float32)}
    return meta, arrays


def main():
    if not R.available():
        raise SystemExit("build the reference first: make -C oracle ref")
    cases, arrays = {}, {}

    def add(name, res, code_spec):
        meta, arr = res
        meta["code"] = code_spec
        cases[name] = meta
        arrays.update(arr)

    # -- LDPC: DVB-S2 short frame, rate 1/2 (the CPU-runnable configuration), three algorithms
    H = F.Ldpc.DvbS2.matrix(16200, Fraction(1, 2))
    for alg, tag in ((F.Exact, "exact"), (F.Linear, "linear"), (F.Approximate, "approx")):
        add("s2short_%s" % tag, ldpc_case("s2short_%s" % tag, H, alg, 20, 1.0, 1.5, 2, 101),
            {"family": "dvbs2", "n": 16200, "rate": [1, 2]})
    # -- LDPC: Gallager(2048, 3, 5, 0), the reference test-suite code, at the suite SNR and at -5 dB
    G = F.Ldpc.Gallager.matrix(2048, 3, 5, 0)
    for alg, tag in ((F.Exact, "exact"), (F.Linear, "linear"), (F.Approximate, "approx")):
        for ebn0, st in ((2.0, "2db"), (-5.0, "m5db")):
            add("gallager_%s_%s" % (tag, st), ldpc_case("gallager_%s_%s" % (tag, st), G, alg, 30, 1.0, ebn0, 2, 102,
                                                         keep_state=True),
                {"family": "gallager", "n": 2048, "wc": 3, "wr": 5, "seed": 0})
    # -- LDPC: DVB-S2 normal frame, rate 1/2, normalized min-sum 0.75, 50 iterations
    H2 = F.Ldpc.DvbS2.matrix(64800, Fraction(1, 2))
    add("s2normal_nms", ldpc_case("s2normal_nms", H2, F.Approximate, 50, 0.75, 1.5, 1, 103),
        {"family": "dvbs2", "n": 64800, "rate": [1, 2]})

    # -- DVB-S2 structures: the reference's transform of each standard matrix, and its encoder
    structures = {}
    rates = {16200: [(1, 4), (1, 3), (2, 5), (1, 2), (3, 5), (2, 3), (3, 4), (4, 5), (5, 6), (8, 9)],
             64800: [(1, 4), (1, 3), (2, 5), (1, 2), (3, 5), (2, 3), (3, 4), (4, 5), (5, 6), (8, 9), (9, 10)]}
    for n, rs in rates.items():
        for num, den in rs:
            Hs = F.Ldpc.DvbS2.matrix(n, Fraction(num, den))
            rc = R.RefCodec.ldpc(Hs.rows(), Hs.cols(), Hs.row_ptr, Hs.col_idx, 2, 10)
            rows, cols, rp, ri = rc.checks()
            m = ch.random_bits(rc.msg, 104)
            structures["%d_%d_%d" % (n, num, den)] = {
                "H_sha": sha(np.concatenate([Hs.row_ptr, Hs.col_idx])),
                "checks_sha": sha(np.concatenate([rp, ri])), "msg_size": rc.msg, "edges": rc.state,
                "encode_sha": sha(rc.encode(m))}
    rows, cols, rp, ri = R.dvbs2_builtin_64800_half()
    structures["reference_builder_64800_1_2_sha"] = sha(np.concatenate([rp, ri]))
    r_, n_, gp, gi = R.gallager(2048, 3, 5, 0)
    structures["gallager_2048_3_5_0_sha"] = sha(np.concatenate([gp, gi]))

    # -- Turbo: LTE K=6144 (the benchmark configuration), three algorithms, serial
    K = 6144
    lte = ([4], [[0o15]], [0o13])
    perms = [np.arange(K), R.lte_interleaver(K)]
    for alg, tag in ((F.Approximate, "approx"), (F.Linear, "linear"), (F.Exact, "exact")):
        add("lte6144_%s" % tag, turbo_case("lte6144_%s" % tag, [lte], perms, 0, alg, 6, F.Serial, 0.7, 2, 201),
            {"family": "lte", "K": K})
    # -- Turbo: LTE K=1024, parallel, per-constituent scaling (decode applies it, soDecode does not)
    K2 = 1024
    add("lte1024_parallel_scaled",
        turbo_case("lte1024_parallel_scaled", [lte], [np.arange(K2), R.lte_interleaver(K2)], 0, F.Approximate, 6,
                   F.Parallel, 0.5, 2, 202, scaling=np.array([[0.7], [0.9]])),
        {"family": "lte", "K": K2})
    # -- Turbo: the reference test-suite shapes (random interleavers stored here)
    rng = np.random.default_rng(0)
    p1 = rng.permutation(1024).astype(np.uint32)
    p2 = rng.permutation(512).astype(np.uint32)
    p3 = (2 * rng.permutation(512)).astype(np.uint32)
    arrays["perm_1024"] = p1
    arrays["perm_512"] = p2
    arrays["perm_even_512"] = p3
    t17 = ([4], [[0o17]], [0o15])
    for term, tag in ((1, "truncate"), (0, "tail")):
        add("suite_%s" % tag, turbo_case("suite_%s" % tag, [t17], [np.arange(1024), p1], term, F.Exact, 4, F.Parallel,
                                          0.0, 2, 203),
            {"family": "suite2", "trellis": "17/15", "perms": ["identity", "perm_1024"]})
    specs = [t17, ([3, 3], [[0o5, 0o3, 0], [0, 0o3, 0o7]], [0o7, 0o5]), ([4], [[0o17, 0o13]], [0o15])]
    add("suite_3var_serial", turbo_case("suite_3var_serial", specs, [p1, p2, p3], 0, F.Exact, 4, F.Serial, 0.0, 2, 204),
        {"family": "suite3", "perms": ["perm_1024", "perm_512", "perm_even_512"]})

    # -- trellis tables of the reference
    trellises = {}
    for key, spec in (("lte_15_13", lte), ("17_15", t17), ("33_5307_75", specs[1]), ("17_13_15", specs[2])):
        sc, ic, osz, ns, out = R.trellis_tables(spec)
        trellises[key] = {"spec": [spec[0], spec[1], spec[2]], "state_count": sc, "input_count": ic,
                          "output_size": osz, "next_state": ns.tolist(), "output": out.tolist()}
    lte_perms = {str(k): sha(R.lte_interleaver(k)) for k in (40, 512, 1024, 4096, 6144)}

    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases, "dvbs2": structures,
                   "trellis": trellises, "lte_interleaver_sha": lte_perms}, f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "golden_arrays.npz"), **arrays)
    print("wrote %d cases, %d arrays" % (len(cases), len(arrays)))


if __name__ == "__main__":
    main()
