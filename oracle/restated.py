"""Test infrastructure: ctypes binding of oracle/_build/libfecl_oracle.so, the C
restatement of FeCl's decode path (fecl_oracle.c).

Used by tests/ (pinned against golden vectors made with the compiled reference),
by the smoke check and by bench.py's CPU baseline when the compiled reference
is absent.  Never by the product.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libfecl_oracle.so")
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_build/libfecl_oracle.so is not built (make -C oracle oracle)")
        L = C.CDLL(LIB_PATH)
        L.fo_ldpc_create.restype = C.c_void_p
        L.fo_turbo_create.restype = C.c_void_p
        for fn in ("fo_ldpc_destroy", "fo_turbo_destroy"):
            getattr(L, fn).argtypes = [C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


def _threads(threads):
    return int(threads or os.cpu_count() or 1)


def dvbs2_matrix(n, num, den):
    rows, cols, nnz = C.c_uint32(), C.c_uint32(), C.c_uint64()
    if lib().fo_dvbs2_matrix(n, num, den, C.byref(rows), C.byref(cols), C.byref(nnz), None, None) != 0:
        raise ValueError("unknown DVB-S2 code")
    ptr = np.zeros(rows.value + 1, np.uint32)
    idx = np.zeros(nnz.value, np.uint32)
    lib().fo_dvbs2_matrix(n, num, den, C.byref(rows), C.byref(cols), C.byref(nnz), _p(ptr), _p(idx))
    return rows.value, cols.value, ptr, idx


def lte_interleaver(K):
    p = np.zeros(K, np.uint32)
    if lib().fo_lte_interleaver(C.c_uint32(K), _p(p)) != 0:
        raise ValueError("Invalid length")
    return p


def trellis(constraint_lengths, generators, feedback=None):
    cl = np.asarray(constraint_lengths, np.uint32)
    g = np.ascontiguousarray(np.asarray(generators, np.uint64))
    fb = None if feedback is None else np.asarray(feedback, np.uint64)
    sc, ic = C.c_uint32(), C.c_uint32()
    L = lib()
    if L.fo_trellis(cl.size, _p(cl), g.shape[1], _p(g), _p(fb), C.byref(sc), C.byref(ic), None, None) != 0:
        raise ValueError("Invalid trellis")
    ns = np.zeros(sc.value * ic.value, np.uint32)
    out = np.zeros(sc.value * ic.value, np.uint32)
    L.fo_trellis(cl.size, _p(cl), g.shape[1], _p(g), _p(fb), C.byref(sc), C.byref(ic), _p(ns), _p(out))
    return sc.value, ic.value, int(g.shape[1]), ns, out


class Ldpc:
    """The restated LDPC code: transform, encoder and BP decoder."""

    def __init__(self, rows, cols, row_ptr, col_idx):
        self._ptr = np.ascontiguousarray(row_ptr, np.uint32)
        self._idx = np.ascontiguousarray(col_idx, np.uint32)
        self.h = lib().fo_ldpc_create(C.c_uint32(rows), C.c_uint32(cols), _p(self._ptr), _p(self._idx))
        if not self.h:
            raise ValueError("Invalid check matrix")
        m, p, s, d = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint32()
        lib().fo_ldpc_sizes(C.c_void_p(self.h), C.byref(m), C.byref(p), C.byref(s), C.byref(d))
        self.msg, self.parity, self.state, self.max_degree = m.value, p.value, s.value, d.value
        self.rows = rows

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fo_ldpc_destroy(C.c_void_p(self.h))
            self.h = None

    def checks(self):
        ptr = np.zeros(self.rows + 1, np.uint32)
        idx = np.zeros(self.state, np.uint32)
        lib().fo_ldpc_checks(C.c_void_p(self.h), _p(ptr), _p(idx))
        return ptr, idx

    def encode(self, msg):
        m = np.ascontiguousarray(msg, np.uint8).reshape(-1, self.msg)
        out = np.zeros((m.shape[0], self.parity), np.uint8)
        for f in range(m.shape[0]):
            lib().fo_ldpc_encode(C.c_void_p(self.h), _p(m[f]), _p(out[f]))
        return out.ravel()

    def check(self, parity):
        p = np.ascontiguousarray(parity, np.uint8).reshape(-1, self.parity)
        return all(lib().fo_ldpc_check(C.c_void_p(self.h), _p(p[f])) == 1 for f in range(p.shape[0]))

    def _table(self, scaling):
        t = np.asarray(scaling, np.float64)
        if t.ndim == 0:
            t = np.full((1, self.max_degree - 1), float(t))
        elif t.ndim == 1:
            t = np.tile(t[:, None], (1, self.max_degree - 1))
        return np.ascontiguousarray(t)

    def decode(self, llr, algorithm, iterations, scaling=1.0, threads=None):
        x = np.ascontiguousarray(llr, np.float64)
        n = x.size // self.parity
        out = np.zeros(n * self.msg, np.uint8)
        its = np.zeros(n, np.int32)
        t = self._table(scaling)
        lib().fo_ldpc_decode(C.c_void_p(self.h), algorithm, C.c_uint32(iterations), _p(t), C.c_uint32(t.shape[0]),
                             _p(x), C.c_uint64(n), _p(out), _p(its), _threads(threads))
        return out, its

    def so_decode(self, parity, algorithm, iterations, scaling=1.0, syst=None, state=None,
                  outputs=("msg", "syst", "parity", "state"), threads=None):
        x = np.ascontiguousarray(parity, np.float64)
        n = x.size // self.parity
        s = None if syst is None else np.ascontiguousarray(syst, np.float64)
        st = None if state is None else np.ascontiguousarray(state, np.float64)
        size = {"msg": self.msg, "syst": self.msg, "parity": self.parity, "state": self.state}
        out = {k: np.zeros(n * size[k], np.float64) for k in outputs}
        t = self._table(scaling)
        lib().fo_ldpc_so_decode(C.c_void_p(self.h), algorithm, C.c_uint32(iterations), _p(t), C.c_uint32(t.shape[0]),
                                _p(x), _p(s), _p(st), C.c_uint64(n), _p(out.get("msg")), _p(out.get("syst")),
                                _p(out.get("parity")), _p(out.get("state")), _threads(threads))
        return out


class Turbo:
    """The restated turbo code: structure, encoder and turbo/MAP decoder.
    trellises: list of (state_count, input_count, output_size, next_state, output)."""

    def __init__(self, trellises, perms, termination):
        n = len(perms)
        tr = list(trellises)
        self._keep = []
        sc = np.asarray([t[0] for t in tr], np.uint32)
        ic = np.asarray([t[1] for t in tr], np.uint32)
        osz = np.asarray([t[2] for t in tr], np.uint32)
        ns = [np.ascontiguousarray(t[3], np.uint32) for t in tr]
        out = [np.ascontiguousarray(t[4], np.uint32) for t in tr]
        ns_arr = (C.c_void_p * len(tr))(*[a.ctypes.data for a in ns])
        out_arr = (C.c_void_p * len(tr))(*[a.ctypes.data for a in out])
        lens = np.asarray([len(p) for p in perms], np.uint32)
        data = np.ascontiguousarray(np.concatenate([np.asarray(p, np.uint32) for p in perms])
                                    if lens.sum() else np.zeros(1, np.uint32))
        term = np.asarray(termination if isinstance(termination, (list, tuple)) else [termination], np.int32)
        self._keep = [sc, ic, osz, ns, out, ns_arr, out_arr, lens, data, term]
        self.h = lib().fo_turbo_create(C.c_uint32(n), _p(sc), _p(ic), _p(osz), ns_arr, out_arr, C.c_uint32(len(tr)),
                                       _p(data), _p(lens), _p(term), C.c_uint32(term.size))
        if not self.h:
            raise ValueError("Invalid turbo structure")
        m, s, p, st = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib().fo_turbo_sizes(C.c_void_p(self.h), C.byref(m), C.byref(s), C.byref(p), C.byref(st))
        self.msg, self.syst, self.parity, self.state = m.value, s.value, p.value, st.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fo_turbo_destroy(C.c_void_p(self.h))
            self.h = None

    def encode(self, msg):
        m = np.ascontiguousarray(msg, np.uint8).reshape(-1, self.msg)
        out = np.zeros((m.shape[0], self.parity), np.uint8)
        for f in range(m.shape[0]):
            lib().fo_turbo_encode(C.c_void_p(self.h), _p(m[f]), _p(out[f]))
        return out.ravel()

    def decode(self, llr, algorithm, iterations, scheduling, scaling=None, threads=None):
        x = np.ascontiguousarray(llr, np.float64)
        n = x.size // self.parity
        out = np.zeros(n * self.msg, np.uint8)
        if scaling is None:
            sf, rows, cols = None, 0, 0
        else:
            sf = np.ascontiguousarray(np.atleast_2d(np.asarray(scaling, np.float64)))
            rows, cols = sf.shape
        lib().fo_turbo_decode(C.c_void_p(self.h), algorithm, C.c_uint32(iterations), scheduling, _p(sf),
                              C.c_uint32(rows), C.c_uint32(cols), _p(x), C.c_uint64(n), _p(out), _threads(threads))
        return out

    def so_decode(self, parity, algorithm, iterations, scheduling, syst=None, state=None,
                  outputs=("msg", "syst", "parity", "state"), threads=None):
        x = np.ascontiguousarray(parity, np.float64)
        n = x.size // self.parity
        s = None if syst is None else np.ascontiguousarray(syst, np.float64)
        st = None if state is None else np.ascontiguousarray(state, np.float64)
        size = {"msg": self.msg, "syst": self.syst, "parity": self.parity, "state": self.state}
        out = {k: np.zeros(n * size[k], np.float64) for k in outputs}
        lib().fo_turbo_so_decode(C.c_void_p(self.h), algorithm, C.c_uint32(iterations), scheduling, _p(x), _p(s),
                                 _p(st), C.c_uint64(n), _p(out.get("msg")), _p(out.get("syst")),
                                 _p(out.get("parity")), _p(out.get("state")), _threads(threads))
        return out


LTE_RSC = ([4], [[0o15]], [0o13])


def lte_turbo(K):
    t = trellis(*LTE_RSC)
    return Turbo([t], [np.arange(K, dtype=np.uint32), lte_interleaver(K)], 0)


def ldpc_decode(H, algorithm, iterations, scaling, llr, threads=None):
    """Hard bits and a-posteriori message L-values (checker interface)."""
    code = Ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx)
    bits, _ = code.decode(llr, algorithm, iterations, scaling, threads)
    return bits, code.so_decode(llr, algorithm, iterations, scaling, outputs=("msg",), threads=threads)["msg"]


def turbo_lte_decode(K, algorithm, iterations, scheduling, llr, threads=None):
    code = lte_turbo(K)
    bits = code.decode(llr, algorithm, iterations, scheduling, threads=threads)
    return bits, code.so_decode(llr, algorithm, iterations, scheduling, outputs=("msg",), threads=threads)["msg"]
