"""Test infrastructure: ctypes binding of oracle/_ref/libfecl_ref.so, the reference
FeCl library compiled from its own sources with the shim in ref_shim.cpp.

Only tests/, the smoke check and bench.py's CPU baseline use this module; the
product never does.  `available()` is False where the library was not built
(the reference tree is not present on every machine; the built .so travels).
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libfecl_ref.so")
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/libfecl_ref.so is not built (make -C oracle ref)")
        L = C.CDLL(LIB_PATH)
        L.fref_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _chk(rc):
    if rc != 0:
        raise ValueError(lib().fref_last_error().decode())


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


class fref_trellis(C.Structure):
    _fields_ = [
        ("ninputs", C.c_size_t),
        ("constraint_lengths", C.c_void_p),
        ("noutputs", C.c_size_t),
        ("generators", C.c_void_p),
        ("feedback", C.c_void_p),
    ]


def gallager(n, wc, wr, seed=0):
    rows, nnz = C.c_size_t(), C.c_size_t()
    _chk(lib().fref_gallager(C.c_size_t(n), C.c_size_t(wc), C.c_size_t(wr), C.c_uint64(seed), C.byref(rows),
                             C.byref(nnz), None, None))
    ptr = np.zeros(rows.value + 1, np.uint32)
    idx = np.zeros(nnz.value, np.uint32)
    _chk(lib().fref_gallager(C.c_size_t(n), C.c_size_t(wc), C.c_size_t(wr), C.c_uint64(seed), C.byref(rows),
                             C.byref(nnz), _p(ptr), _p(idx)))
    return rows.value, n, ptr, idx


def dvbs2_builtin_64800_half():
    rows, cols, nnz = C.c_size_t(), C.c_size_t(), C.c_size_t()
    L = lib()
    _chk(L.fref_dvbs2_builtin(C.c_size_t(64800), C.c_double(0.5), C.byref(rows), C.byref(cols), C.byref(nnz), None, None))
    ptr = np.zeros(rows.value + 1, np.uint32)
    idx = np.zeros(nnz.value, np.uint32)
    _chk(L.fref_dvbs2_builtin(C.c_size_t(64800), C.c_double(0.5), C.byref(rows), C.byref(cols), C.byref(nnz), _p(ptr),
                              _p(idx)))
    return rows.value, cols.value, ptr, idx


def lte_interleaver(K):
    p = np.zeros(K, np.uint32)
    _chk(lib().fref_lte_interleaver(C.c_size_t(K), _p(p)))
    return p


def _trellis_struct(spec, keep):
    cl, gens, fb = spec
    cl = np.asarray(cl, dtype=np.uint64).astype(np.uintp)
    g = np.asarray(gens, dtype=np.uint64)
    f = None if fb is None else np.asarray(fb, dtype=np.uint64)
    keep += [cl, g, f]
    return fref_trellis(cl.size, cl.ctypes.data, g.shape[1], g.ctypes.data, f.ctypes.data if f is not None else None)


def trellis_tables(spec):
    keep = []
    t = _trellis_struct(spec, keep)
    sc, ic, osz = C.c_size_t(), C.c_size_t(), C.c_size_t()
    L = lib()
    _chk(L.fref_trellis_tables(C.byref(t), C.byref(sc), C.byref(ic), C.byref(osz), None, None))
    ns = np.zeros(sc.value * ic.value, np.uint32)
    out = np.zeros(sc.value * ic.value, np.uint32)
    _chk(L.fref_trellis_tables(C.byref(t), C.byref(sc), C.byref(ic), C.byref(osz), _p(ns), _p(out)))
    return sc.value, ic.value, osz.value, ns, out


class RefCodec:
    """A reference fec::Ldpc or fec::Turbo driven through the shim."""

    def __init__(self, handle):
        self.h = C.c_void_p(handle)
        s = (C.c_size_t * 4)()
        _chk(lib().fref_codec_sizes(self.h, s))
        self.msg, self.syst, self.parity, self.state = list(s)

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value and _lib is not None:
            _lib.fref_codec_destroy(self.h)
            self.h = C.c_void_p(0)

    @classmethod
    def ldpc(cls, rows, cols, row_ptr, col_idx, algorithm, iterations, scaling=(1.0,), workgroup=1):
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        ci = np.ascontiguousarray(col_idx, np.uint32)
        sf = np.ascontiguousarray(scaling, np.float64)
        h = C.c_void_p()
        _chk(lib().fref_ldpc_create(C.c_size_t(rows), C.c_size_t(cols), _p(rp), _p(ci), C.c_int(algorithm),
                                    C.c_size_t(iterations), _p(sf), C.c_size_t(sf.size), C.c_int(workgroup), C.byref(h)))
        return cls(h.value)

    @classmethod
    def turbo(cls, trellis_specs, perms, termination, algorithm, scheduling, iterations, scaling=None, workgroup=1):
        keep = []
        arr = (fref_trellis * len(trellis_specs))(*[_trellis_struct(s, keep) for s in trellis_specs])
        lens = np.asarray([len(p) for p in perms], dtype=np.uintp)
        data = np.ascontiguousarray(np.concatenate([np.asarray(p, np.uint32) for p in perms]) if sum(lens) else np.zeros(1, np.uint32))
        if scaling is None:
            sf = np.zeros(1, np.float64)
            rows_, cols_ = 0, 0
        else:
            sf = np.ascontiguousarray(scaling, np.float64)
            rows_, cols_ = sf.shape
        h = C.c_void_p()
        _chk(lib().fref_turbo_create(C.c_size_t(len(perms)), arr, C.c_size_t(len(trellis_specs)), _p(data), _p(lens),
                                     C.c_int(termination), C.c_int(algorithm), C.c_int(scheduling), C.c_size_t(iterations),
                                     _p(sf), C.c_size_t(rows_), C.c_size_t(cols_), C.c_int(workgroup), C.byref(h)))
        return cls(h.value)

    @classmethod
    def conv(cls, trellis_spec, length, termination, algorithm=2, scaling=1.0, workgroup=1):
        keep = []
        t = _trellis_struct(trellis_spec, keep)
        h = C.c_void_p()
        _chk(lib().fref_conv_create(C.byref(t), C.c_size_t(length), C.c_int(termination), C.c_int(algorithm),
                                    C.c_double(scaling), C.c_int(workgroup), C.byref(h)))
        return cls(h.value)

    def conv_puncturing(self, mask=(), tail_mask=()):
        """Convolutional::Structure::puncturing: (sequence, input size)."""
        m = np.asarray(list(mask) or [0], np.uint8)
        t = np.asarray(list(tail_mask) or [0], np.uint8)
        n, ins = C.c_size_t(), C.c_size_t()
        L = lib()
        args = (self.h, _p(m), C.c_size_t(len(mask)), _p(t), C.c_size_t(len(tail_mask)))
        _chk(L.fref_conv_puncturing(*args, None, C.byref(n), C.byref(ins)))
        seq = np.zeros(max(n.value, 1), np.uint32)
        _chk(L.fref_conv_puncturing(*args, _p(seq), C.byref(n), C.byref(ins)))
        return seq[: n.value], ins.value

    def set_turbo_schedule(self, stages, algorithm, iterations, scaling=None):
        """A custom schedule: stages = [(activation, [transfer, ...]), ...]."""
        counts = np.asarray([len(a) for a, _ in stages] or [0], np.uint32)
        act = np.asarray([x for a, _ in stages for x in a] or [0], np.uint32)
        tc = np.asarray([len(t) for _, tr in stages for t in tr] or [0], np.uint32)
        tr = np.asarray([x for _, trs in stages for t in trs for x in t] or [0], np.uint32)
        if scaling is None:
            sf, r, c = np.zeros(1, np.float64), 0, 0
        else:
            sf = np.ascontiguousarray(scaling, np.float64)
            r, c = sf.shape
        _chk(lib().fref_turbo_set_schedule(self.h, C.c_int(algorithm), C.c_size_t(iterations), _p(sf), C.c_size_t(r),
                                           C.c_size_t(c), C.c_size_t(len(stages)), _p(counts), _p(act), _p(tc), _p(tr)))

    def set_workgroup(self, n):
        _chk(lib().fref_codec_set_workgroup(self.h, C.c_int(n)))

    def checks(self):
        rows, cols, nnz = C.c_size_t(), C.c_size_t(), C.c_size_t()
        L = lib()
        _chk(L.fref_ldpc_checks(self.h, C.byref(rows), C.byref(cols), C.byref(nnz), None, None))
        ptr = np.zeros(rows.value + 1, np.uint32)
        idx = np.zeros(nnz.value, np.uint32)
        _chk(L.fref_ldpc_checks(self.h, C.byref(rows), C.byref(cols), C.byref(nnz), _p(ptr), _p(idx)))
        return rows.value, cols.value, ptr, idx

    def encode(self, msg):
        m = np.ascontiguousarray(msg, np.uint8)
        n = m.size // self.msg
        out = np.zeros(n * self.parity, np.uint8)
        _chk(lib().fref_codec_encode(self.h, _p(m), C.c_size_t(n), _p(out)))
        return out

    def check(self, parity):
        p = np.ascontiguousarray(parity, np.uint8)
        r = lib().fref_codec_check(self.h, _p(p), C.c_size_t(p.size // self.parity))
        if r < 0:
            raise ValueError(lib().fref_last_error().decode())
        return bool(r)

    def decode(self, llr):
        x = np.ascontiguousarray(llr, np.float64)
        n = x.size // self.parity
        out = np.zeros(n * self.msg, np.uint8)
        _chk(lib().fref_codec_decode(self.h, _p(x), C.c_size_t(n), _p(out)))
        return out

    def so_decode(self, parity, syst=None, state=None, outputs=("msg",)):
        x = np.ascontiguousarray(parity, np.float64)
        n = x.size // self.parity
        s = None if syst is None else np.ascontiguousarray(syst, np.float64)
        st = None if state is None else np.ascontiguousarray(state, np.float64)
        size = {"msg": self.msg, "syst": self.syst, "parity": self.parity, "state": self.state}
        out = {k: np.zeros(n * size[k], np.float64) for k in outputs}
        _chk(lib().fref_codec_so_decode(self.h, C.c_size_t(n), _p(x), _p(s), _p(st), _p(out.get("msg")),
                                        _p(out.get("syst")), _p(out.get("parity")), _p(out.get("state"))))
        return out

    def ldpc_puncturing(self, mask=(), syst_mask=()):
        """Ldpc::Structure::puncturing (src/detail/Ldpc.cpp:333-353): (sequence, input size)."""
        m = np.ascontiguousarray(np.asarray(mask, np.uint8).reshape(-1)) if len(mask) else np.zeros(1, np.uint8)
        sm = np.ascontiguousarray(np.asarray(syst_mask, np.uint8).reshape(-1)) if len(syst_mask) else np.zeros(1, np.uint8)
        n, ins = C.c_size_t(), C.c_size_t()
        L = lib()
        _chk(L.fref_ldpc_puncturing(self.h, _p(m), C.c_size_t(len(mask)), _p(sm), C.c_size_t(len(syst_mask)), None,
                                    C.byref(n), C.byref(ins)))
        seq = np.zeros(max(n.value, 1), np.uint32)
        _chk(L.fref_ldpc_puncturing(self.h, _p(m), C.c_size_t(len(mask)), _p(sm), C.c_size_t(len(syst_mask)), _p(seq),
                                    C.byref(n), C.byref(ins)))
        return seq[: n.value], ins.value

    def turbo_puncturing(self, masks=(), tails=(), ordering=0):
        """Turbo::Structure::puncturing (src/detail/Turbo.cpp:200-320): (sequence, input size)."""
        def flat(ms):
            data = np.asarray([b for x in ms for b in x] or [0], np.uint8)
            lens = np.asarray([len(x) for x in ms] or [0], np.uintp)
            return data, lens
        md, ml = flat(masks)
        td, tl = flat(tails)
        n, ins = C.c_size_t(), C.c_size_t()
        L = lib()
        args = (self.h, _p(md), _p(ml), C.c_size_t(len(masks)), _p(td), _p(tl), C.c_size_t(len(tails)), C.c_int(ordering))
        _chk(L.fref_turbo_puncturing(*args, None, C.byref(n), C.byref(ins)))
        seq = np.zeros(max(n.value, 1), np.uint32)
        _chk(L.fref_turbo_puncturing(*args, _p(seq), C.byref(n), C.byref(ins)))
        return seq[: n.value], ins.value
