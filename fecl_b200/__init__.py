"""fecl_b200: B200-native batched soft-decision decoding with FeCl's API.

A Python mirror of the FeCl C++ interface (src/Codec.h, src/Ldpc.h, src/Turbo.h,
src/Trellis.h) on top of the C-ABI in include/fecl_b200.h.  Names, argument
meaning and error behaviour follow the reference:

    code = Ldpc(Ldpc.EncoderOptions(Ldpc.DvbS2.matrix(16200, Fraction(1, 2))),
                Ldpc.DecoderOptions().algorithm(Exact).iterations(20))
    bits = code.decode(llr)                       # Codec::decode, src/Codec.h:210-238
    out = Codec.Output().msg().state()
    code.soDecode(Codec.Input().parity(llr), out)  # Codec::soDecode, src/Codec.h:249-307

Host numpy arrays go through FECL_HOST_MEMORY (the call copies in, decodes on
the GPU and copies out); torch CUDA tensors go through FECL_DEVICE_MEMORY on the
current torch stream.  Size mismatches raise ValueError, as the reference throws
std::invalid_argument.  Bits are uint8 0/1 (the reference uses BitField<size_t>).
"""
import ctypes as C
from fractions import Fraction

import numpy as np

from . import _lib
from ._lib import check as _check
from ._lib import lib as _L

__all__ = [
    "Exact", "Linear", "Approximate", "Serial", "Parallel", "Custom", "CRC24A", "CRC24B", "crc24_attach", "crc24_check",
    "SparseBitMatrix", "Trellis", "Codec", "Ldpc", "Turbo", "Convolutional", "Batch", "Server", "Permutation", "FeclError", "lib_path",
]

# DecoderAlgorithm (src/DecoderAlgorithm.h:30-34) and SchedulingType (src/SchedulingType.h:32-39)
Exact, Linear, Approximate = 0, 1, 2
Serial, Parallel, Custom = 0, 1, 2
# CRC polynomials of 3GPP TS 36.212 section 5.1.1 (an extension)
CRC24A, CRC24B = 1, 2


def crc24_attach(bits, kind, nframes=1):
    """Extension: appends to each of `nframes` frames of the torch CUDA uint8 tensor
    `bits` its 24 CRC bits (fecl_crc24_attach); returns a CUDA tensor."""
    import torch
    b = bits.contiguous().view(-1)
    n = int(nframes)
    if n <= 0 or b.numel() % n:
        raise ValueError("Invalid size for message")
    L = b.numel() // n
    out = torch.empty(n * (L + 24), dtype=torch.uint8, device=b.device)
    _check(_L.fecl_crc24_attach(C.c_void_p(b.data_ptr()), L, n, int(kind), C.c_void_p(out.data_ptr()),
                                C.c_void_p(torch.cuda.current_stream(b.device).cuda_stream)))
    return out


def crc24_check(bits, kind, nframes=1):
    """Extension: per frame, whether its bits (CRC included) pass (fecl_crc24_check)."""
    import torch
    b = bits.contiguous().view(-1)
    n = int(nframes)
    if n <= 0 or b.numel() % n:
        raise ValueError("Invalid size")
    ok = torch.empty(n, dtype=torch.int32, device=b.device)
    _check(_L.fecl_crc24_check(C.c_void_p(b.data_ptr()), b.numel() // n, n, int(kind), C.c_void_p(ok.data_ptr()),
                               C.c_void_p(torch.cuda.current_stream(b.device).cuda_stream)))
    return ok.bool()
FeclError = _lib.FeclError
lib_path = _lib.LIB_PATH


def _u32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None and a.size else C.c_void_p(0)


class SparseBitMatrix:
    """A binary matrix in CSR form (SparseBitMatrix, src/BitMatrix.h:42-624)."""

    def __init__(self, rows, cols, row_ptr, col_idx):
        self._rows, self._cols = int(rows), int(cols)
        self.row_ptr = _u32(row_ptr)
        self.col_idx = _u32(col_idx)
        if self.row_ptr.size != self._rows + 1:
            raise ValueError("row_ptr must hold rows + 1 entries")

    @classmethod
    def from_dense(cls, dense):
        d = np.asarray(dense) != 0
        rows = [np.nonzero(r)[0] for r in d]
        ptr = np.zeros(len(rows) + 1, dtype=np.uint32)
        ptr[1:] = np.cumsum([len(r) for r in rows])
        idx = np.concatenate(rows) if rows else np.zeros(0, np.uint32)
        return cls(d.shape[0], d.shape[1], ptr, idx)

    def rows(self):
        return self._rows

    def cols(self):
        return self._cols

    def size(self):
        return int(self.col_idx.size)

    def row(self, r):
        return self.col_idx[self.row_ptr[r]:self.row_ptr[r + 1]]

    def rowSizes(self):
        return np.diff(self.row_ptr.astype(np.int64))

    def to_dense(self):
        d = np.zeros((self._rows, self._cols), dtype=np.uint8)
        for r in range(self._rows):
            d[r, self.row(r)] = 1
        return d

    def __eq__(self, other):
        return (self._rows, self._cols) == (other._rows, other._cols) and np.array_equal(
            self.row_ptr, other.row_ptr) and np.array_equal(self.col_idx, other.col_idx)


class Trellis:
    """Trellis(constraintLengths, generator, feedback) -- src/Trellis.cpp:76-143.
    Tables are indexed [state * inputCount + input] (src/Trellis.h:131-172)."""
    Tail, Truncate = 0, 1

    def __init__(self, constraintLengths, generator, feedback=None):
        cl = _u32(constraintLengths)
        gen = np.ascontiguousarray(np.asarray(generator, dtype=np.uint64))
        if gen.ndim != 2 or gen.shape[0] != cl.size:
            raise ValueError("Invalid number of generators")
        fb = None if not feedback else np.ascontiguousarray(np.asarray(feedback, dtype=np.uint64))
        sc, ic, osz = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(_L.fecl_trellis_build(cl.size, _ptr(cl), gen.shape[1], _ptr(gen), _ptr(fb), C.byref(sc), C.byref(ic),
                                     C.byref(osz), None, None))
        self.next_state = np.zeros(sc.value * ic.value, dtype=np.uint32)
        self.output = np.zeros(sc.value * ic.value, dtype=np.uint32)
        _check(_L.fecl_trellis_build(cl.size, _ptr(cl), gen.shape[1], _ptr(gen), _ptr(fb), C.byref(sc), C.byref(ic),
                                     C.byref(osz), _ptr(self.next_state), _ptr(self.output)))
        self._sc, self._ic, self._os = sc.value, ic.value, osz.value

    def stateCount(self):
        return self._sc

    def inputCount(self):
        return self._ic

    def outputSize(self):
        return self._os

    def getNextState(self, s, u):
        return int(self.next_state[s * self._ic + u])

    def getOutput(self, s, u):
        return int(self.output[s * self._ic + u])

    def _c(self):
        return _lib.fecl_trellis(self._sc, self._ic, self._os, self.next_state.ctypes.data_as(C.POINTER(C.c_uint32)),
                                 self.output.ctypes.data_as(C.POINTER(C.c_uint32)))


def _is_device(x):
    return hasattr(x, "is_cuda") and x.is_cuda


def _contiguous(x):
    if hasattr(x, "is_contiguous"):
        return x.is_contiguous()
    return np.asarray(x).flags["C_CONTIGUOUS"]


def _dtype_code(a):
    if hasattr(a, "data_ptr"):
        import torch
        m = {torch.float64: _lib.F64, torch.float32: _lib.F32, torch.float16: _lib.F16}
    else:
        m = {np.dtype(np.float64): _lib.F64, np.dtype(np.float32): _lib.F32, np.dtype(np.float16): _lib.F16}
    try:
        return m[a.dtype]
    except KeyError:
        raise ValueError("L-values must be float64, float32 or float16")


class Codec:
    """fec::Codec (src/Codec.h:46-127): the operations every code family offers."""

    class Input:
        """Codec::Input (src/detail/Codec.h:142-171): parity (required), syst, state."""

        def __init__(self):
            self._v = {}

        def parity(self, x):
            self._v["parity"] = x
            return self

        def syst(self, x):
            self._v["syst"] = x
            return self

        def state(self, x):
            self._v["state"] = x
            return self

        def msg(self, x):
            self._v["msg"] = x
            return self

    class Output:
        """Codec::Output: name the outputs wanted; after soDecode, call them without
        argument to read the arrays (host) or tensors (device)."""

        def __init__(self, dtype=np.float64):
            self._want = []
            self._v = {}
            self.dtype = dtype

        def _get_or_want(self, name):
            if name in self._v:
                return self._v[name]
            self._want.append(name)
            return self

        def msg(self):
            return self._get_or_want("msg")

        def syst(self):
            return self._get_or_want("syst")

        def parity(self):
            return self._get_or_want("parity")

        def state(self):
            return self._get_or_want("state")

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        s = _lib.fecl_sizes()
        _check(_L.fecl_codec_sizes(self._h, C.byref(s)))
        self._sizes = (s.msg, s.syst, s.parity, s.state)
        self._work_group = 8

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _L is not None:
            try:
                _L.fecl_destroy(h)
            except Exception:
                pass
            self._h = C.c_void_p(0)

    def msgSize(self):
        return self._sizes[0]

    def systSize(self):
        return self._sizes[1]

    def paritySize(self):
        return self._sizes[2]

    def stateSize(self):
        return self._sizes[3]

    def setKernel(self, kernel):
        """Extension: 'auto' (fastest kernel for the code), 'generic' (the kernels that
        walk the reference's operation order in FP32), and for LDPC 'lanes' (32 frames
        per warp, messages in device memory) or 'cluster' (each frame's messages in the
        shared memory of a thread-block cluster)."""
        sel = {"auto": 0, "generic": 1, "lanes": 2, "cluster": 3}
        if kernel not in sel:
            raise ValueError("Invalid kernel selection")
        _check(_L.fecl_set_kernel(self._h, sel[kernel]))

    # Codec::getWorkGroupSize / setWorkGroupSize (src/Codec.h:65-66): a CPU thread count
    # in the reference; kept for API compatibility, the device decoder ignores it.
    def getWorkGroupSize(self):
        return self._work_group

    def setWorkGroupSize(self, n):
        self._work_group = int(n)

    def _frames(self, n, size, what):
        blocks = n // size
        if n != blocks * size:
            raise ValueError("Invalid size for %s" % what)
        return blocks

    def encode(self, msg):
        """Codec::encode -- src/Codec.h:171-198.  A torch CUDA tensor of message bits is
        encoded on the GPU (asynchronous on the current stream) and returns a CUDA tensor."""
        if _is_device(msg):
            import torch
            m = msg.contiguous().view(-1)
            if m.dtype != torch.uint8:
                raise ValueError("message bits must be uint8")
            n = self._frames(m.numel(), self.msgSize(), "message")
            parity = torch.empty(n * self.paritySize(), dtype=torch.uint8, device=m.device)
            stream = torch.cuda.current_stream(m.device).cuda_stream
            _check(_L.fecl_encode(self._h, C.c_void_p(m.data_ptr()), n, C.c_void_p(parity.data_ptr()),
                                  _lib.DEVICE_MEMORY, C.c_void_p(stream)))
            return parity
        m = np.ascontiguousarray(np.asarray(msg, dtype=np.uint8).ravel())
        n = self._frames(m.size, self.msgSize(), "message")
        parity = np.zeros(n * self.paritySize(), dtype=np.uint8)
        _check(_L.fecl_encode(self._h, _ptr(m), n, _ptr(parity), _lib.HOST_MEMORY, None))
        return parity

    def check(self, parity):
        """Codec::check -- src/Codec.h:137-145."""
        p = np.ascontiguousarray(np.asarray(parity, dtype=np.uint8).ravel())
        n = self._frames(p.size, self.paritySize(), "parity")
        ok = C.c_int32(0)
        _check(_L.fecl_check(self._h, _ptr(p), n, C.byref(ok)))
        return bool(ok.value)

    def decode(self, parity, iterations=False, out=None):
        """Codec::decode -- src/Codec.h:210-238.  Returns the hard message bits and,
        with iterations=True, the per-frame iteration counts.

        parity may be a numpy array (host memory), a torch CUDA tensor (device memory,
        asynchronous on the current stream) or a torch CPU tensor, ideally pinned (host
        memory; the call copies in, decodes and copies out).  `out` optionally receives
        the bits (same kind of memory as parity)."""
        if _is_device(parity):
            import torch
            x = parity.contiguous().view(-1)
            n = self._frames(x.numel(), self.paritySize(), "parity")
            msg = out if out is not None else torch.empty(n * self.msgSize(), dtype=torch.uint8, device=x.device)
            it = torch.empty(n, dtype=torch.int32, device=x.device) if iterations else None
            stream = torch.cuda.current_stream(x.device).cuda_stream
            _check(_L.fecl_decode(self._h, C.c_void_p(x.data_ptr()), _dtype_code(x), n, C.c_void_p(msg.data_ptr()),
                                  C.c_void_p(it.data_ptr()) if it is not None else None, _lib.DEVICE_MEMORY,
                                  C.c_void_p(stream)))
            return (msg, it) if iterations else msg
        if hasattr(parity, "data_ptr"):  # torch CPU tensor
            import torch
            x = parity.contiguous().view(-1)
            n = self._frames(x.numel(), self.paritySize(), "parity")
            msg = out if out is not None else torch.empty(n * self.msgSize(), dtype=torch.uint8)
            it = torch.empty(n, dtype=torch.int32) if iterations else None
            _check(_L.fecl_decode(self._h, C.c_void_p(x.data_ptr()), _dtype_code(x), n, C.c_void_p(msg.data_ptr()),
                                  C.c_void_p(it.data_ptr()) if it is not None else None, _lib.HOST_MEMORY, None))
            return (msg, it) if iterations else msg
        x = np.asarray(parity)
        if x.dtype not in (np.float64, np.float32, np.float16):
            x = x.astype(np.float64)
        x = np.ascontiguousarray(x.ravel())
        n = self._frames(x.size, self.paritySize(), "parity")
        msg = np.zeros(n * self.msgSize(), dtype=np.uint8)
        it = np.zeros(n, dtype=np.int32) if iterations else None
        _check(_L.fecl_decode(self._h, _ptr(x), _dtype_code(x), n, _ptr(msg), _ptr(it) if it is not None else None,
                              _lib.HOST_MEMORY, None))
        return (msg, it) if iterations else msg

    def soDecode(self, input, output, out=None):
        """Codec::soDecode -- src/Codec.h:249-307.  `out` optionally maps output names
        to preallocated buffers (numpy arrays or torch tensors in the input's kind of
        memory, of the output dtype and size) that receive them."""
        v = input._v
        if "parity" not in v:
            raise ValueError("Input must contains parity")
        if "msg" in v:
            raise ValueError("Input should not contain msg")
        par = v["parity"]
        device = _is_device(par)
        n_par = par.numel() if device else np.asarray(par).size
        n = self._frames(n_par, self.paritySize(), "parity")
        if "syst" in v and (v["syst"].numel() if device else np.asarray(v["syst"]).size) != n * self.systSize():
            raise ValueError("Invalid size for msg")
        if "state" in v and (v["state"].numel() if device else np.asarray(v["state"]).size) != n * self.stateSize():
            raise ValueError("Invalid size for state")
        sizes = {"msg": self.msgSize(), "syst": self.systSize(), "parity": self.paritySize(), "state": self.stateSize()}
        io = _lib.fecl_so_io()
        keep = []
        if device:
            import torch
            dt = par.dtype
            ins = {k: v[k].contiguous().view(-1).to(dt) for k in ("parity", "syst", "state") if k in v}
            odt = torch.float64 if output.dtype == np.float64 else torch.float32
            outs = {k: torch.empty(n * sizes[k], dtype=odt, device=par.device) for k in output._want
                    if not (out and k in out)}
            ptr = lambda t: t.data_ptr()
            flags = _lib.DEVICE_MEMORY
            stream = C.c_void_p(torch.cuda.current_stream(par.device).cuda_stream)
            io.in_dtype = _dtype_code(ins["parity"])
        else:
            x = np.asarray(par)
            dt = x.dtype if x.dtype in (np.float64, np.float32, np.float16) else np.float64
            ins = {k: np.ascontiguousarray(np.asarray(v[k], dtype=dt).ravel()) for k in ("parity", "syst", "state") if k in v}
            odt = np.float64 if output.dtype == np.float64 else np.float32
            outs = {k: np.zeros(n * sizes[k], dtype=odt) for k in output._want if not (out and k in out)}
            ptr = lambda a: a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data
            flags = _lib.HOST_MEMORY
            stream = None
            io.in_dtype = _dtype_code(ins["parity"])
        io.out_dtype = _lib.F64 if output.dtype == np.float64 else _lib.F32
        for k in output._want:
            if out and k in out:
                t = out[k]
                nbytes = t.numel() * t.element_size() if hasattr(t, "data_ptr") else np.asarray(t).nbytes
                if nbytes != n * sizes[k] * (8 if io.out_dtype == _lib.F64 else 4) or not _contiguous(t):
                    raise ValueError("Invalid size for " + k)
                outs[k] = t
        for k, t in ins.items():
            setattr(io, k, ptr(t))
            keep.append(t)
        for k, t in outs.items():
            setattr(io, {"msg": "msg", "syst": "syst_out", "parity": "parity_out", "state": "state_out"}[k], ptr(t))
        _check(_L.fecl_so_decode(self._h, C.byref(io), n, flags, stream))
        output._v.update(outs)
        output._want = []
        return output


class Ldpc(Codec):
    """fec::Ldpc -- src/Ldpc.h:59-108."""

    class EncoderOptions:
        def __init__(self, checkMatrix):
            self._H = checkMatrix

        def checkMatrix(self):
            return self._H

    class DecoderOptions:
        """Ldpc::DecoderOptions -- src/detail/Ldpc.h:56-74 (iterations defaults to 50
        here; the reference leaves it uninitialised)."""

        def __init__(self):
            self._alg = Approximate
            self._it = 50
            self._sf = {0: [1.0]}
            self._precision = _lib.MSG_F32
            self._fixed = False

        def algorithm(self, a=None):
            if a is None:
                return self._alg
            self._alg = int(a)
            return self

        def iterations(self, n=None):
            if n is None:
                return self._it
            self._it = int(n)
            return self

        def scalingFactor(self, f=None):
            if f is None:
                return self._sf
            self._sf = dict(f) if isinstance(f, dict) else {0: [float(f)]}
            return self

        def precision(self, p=None):
            if p is None:
                return self._precision
            self._precision = int(p)
            return self

        def fixedIterations(self, on=None):
            if on is None:
                return self._fixed
            self._fixed = bool(on)
            return self

    class PunctureOptions:
        """Ldpc::PunctureOptions -- src/detail/Ldpc.h (mask, systMask: repeating bit masks)."""

        def __init__(self):
            self._mask, self._syst = [], []

        def mask(self, m=None):
            if m is None:
                return list(self._mask)
            self._mask = [bool(x) for x in m]
            return self

        def systMask(self, m=None):
            if m is None:
                return list(self._syst)
            self._syst = [bool(x) for x in m]
            return self

    def puncturing(self, options):
        """Ldpc::puncturing -- src/Ldpc.h:94: the fec::Permutation of the kept code bits."""
        m = np.asarray(options._mask, np.uint8)
        sm = np.asarray(options._syst, np.uint8)
        n = C.c_uint64()
        _check(_L.fecl_ldpc_puncturing(self._h, _ptr(m), m.size, _ptr(sm), sm.size, None, C.byref(n)))
        seq = np.zeros(n.value, np.uint32)
        _check(_L.fecl_ldpc_puncturing(self._h, _ptr(m), m.size, _ptr(sm), sm.size, _ptr(seq), C.byref(n)))
        return Permutation(seq, self.paritySize())

    class Gallager:
        @staticmethod
        def matrix(n, wc, wr, seed=0):
            """Ldpc::Gallager::matrix -- src/Ldpc.cpp:77-102."""
            rows, nnz = C.c_uint32(), C.c_uint64()
            _check(_L.fecl_gallager_matrix(n, wc, wr, seed, C.byref(rows), C.byref(nnz), None, None))
            ptr = np.zeros(rows.value + 1, np.uint32)
            idx = np.zeros(nnz.value, np.uint32)
            _check(_L.fecl_gallager_matrix(n, wc, wr, seed, C.byref(rows), C.byref(nnz), _ptr(ptr), _ptr(idx)))
            return SparseBitMatrix(rows.value, n, ptr, idx)

    class DvbS2:
        @staticmethod
        def matrix(n, rate):
            """Standard DVB-S2 check matrix for n in {16200, 64800} (Ldpc::DvbS2::matrix,
            src/DvbS2.cpp:1595-1645).  rate is a Fraction or one of the listed floats."""
            fr = Fraction(rate).limit_denominator(16)
            rows, cols, nnz = C.c_uint32(), C.c_uint32(), C.c_uint64()
            _check(_L.fecl_dvbs2_matrix(n, fr.numerator, fr.denominator, C.byref(rows), C.byref(cols), C.byref(nnz), None, None))
            ptr = np.zeros(rows.value + 1, np.uint32)
            idx = np.zeros(nnz.value, np.uint32)
            _check(_L.fecl_dvbs2_matrix(n, fr.numerator, fr.denominator, C.byref(rows), C.byref(cols), C.byref(nnz),
                                        _ptr(ptr), _ptr(idx)))
            return SparseBitMatrix(rows.value, cols.value, ptr, idx)

    def __init__(self, encoder, decoder=None, workGroupSize=8):
        H = encoder.checkMatrix() if isinstance(encoder, Ldpc.EncoderOptions) else encoder
        decoder = decoder or Ldpc.DecoderOptions()
        self._degrees = H.rowSizes()
        opts, keep = self._options(decoder)
        h = C.c_void_p()
        _check(_L.fecl_ldpc_create(H.rows(), H.cols(), _ptr(H.row_ptr), _ptr(H.col_idx), C.byref(opts), C.byref(h)))
        super().__init__(h.value)
        self._decoder = decoder
        self._work_group = workGroupSize

    def _options(self, d):
        """scalingMapToVector (src/detail/Ldpc.cpp:64-112): map {degree: [per-iteration]}
        with key 0 as default -> table [iterations or 1][maxDegree-1]."""
        deg = self._degrees
        maxd = int(deg.max())
        m = d.scalingFactor()
        if 0 in m:
            default = list(m[0])
            if len(default) != 1 and len(default) != d.iterations():
                raise ValueError("Wrong size for scaling factor")
            vec = [[default[i]] * (maxd - 1) for i in range(len(default))]
            for key, vals in m.items():
                if 2 <= key and key - 2 < maxd - 1:
                    if len(vals) != len(vec):
                        raise ValueError("Wrong size for scaling factor")
                    for j in range(len(vec)):
                        vec[j][key - 2] = vals[j]
        else:
            length = max(len(v) for v in m.values())
            if length != 1 and length != d.iterations():
                raise ValueError("Wrong size for scaling factor")
            vec = [[0.0] * (maxd - 1) for _ in range(length)]
            for dg in deg:
                if int(dg) not in m:
                    raise ValueError("Scaling factor not defined and no default")
                vals = m[int(dg)]
                if len(vals) != length:
                    raise ValueError("Wrong size for scaling factor")
                for j in range(length):
                    vec[j][int(dg) - 2] = vals[j]
        table = np.ascontiguousarray(np.asarray(vec, dtype=np.float64))
        o = _lib.fecl_ldpc_options()
        o.algorithm = d.algorithm()
        o.iterations = d.iterations()
        o.scaling = table.ctypes.data_as(C.POINTER(C.c_double))
        o.scaling_iterations = table.shape[0]
        o.scaling_degrees = table.shape[1]
        o.precision = d.precision()
        o.fixed_iterations = 1 if d.fixedIterations() else 0
        self._table = table
        return o, table

    def setDecoderOptions(self, decoder):
        opts, keep = self._options(decoder)
        _check(_L.fecl_ldpc_set_options(self._h, C.byref(opts)))
        self._decoder = decoder

    def getDecoderOptions(self):
        return self._decoder

    def setClusterShape(self, cluster=0, threads=0):
        """Extension: CTAs per frame (1, 2, 4, 8, 16) and threads per CTA (256, 512,
        1024) of the cluster-resident decoder; 0 restores the built-in choice."""
        _check(_L.fecl_ldpc_set_cluster_shape(self._h, int(cluster), int(threads)))
        return self

    def setWave(self, groups=0):
        """Extension: frame groups of 32 the lane-batched decoder runs together through
        every iteration (0 restores the built-in choice)."""
        _check(_L.fecl_ldpc_set_wave(self._h, int(groups)))
        return self

    def setPersistent(self, mode=0):
        """Extension: run small batches as one persistent launch (1: wherever it
        applies, 0: built-in choice, -1: never); results are identical either way."""
        _check(_L.fecl_ldpc_set_persistent(self._h, int(mode)))
        return self

    def checks(self):
        """The transformed check matrix (detail::Ldpc::Structure::checks); its edge
        order is the layout of the soft state."""
        rows, cols, nnz = C.c_uint32(), C.c_uint32(), C.c_uint64()
        _check(_L.fecl_ldpc_checks(self._h, C.byref(rows), C.byref(cols), C.byref(nnz), None, None))
        ptr = np.zeros(rows.value + 1, np.uint32)
        idx = np.zeros(nnz.value, np.uint32)
        _check(_L.fecl_ldpc_checks(self._h, C.byref(rows), C.byref(cols), C.byref(nnz), _ptr(ptr), _ptr(idx)))
        return SparseBitMatrix(rows.value, cols.value, ptr, idx)


class Turbo(Codec):
    """fec::Turbo -- src/Turbo.h:55-116."""

    class Lte3Gpp:
        @staticmethod
        def interleaver(length):
            """Turbo::Lte3Gpp::interleaver -- src/Lte3Gpp.cpp:219-237."""
            p = np.zeros(int(length), np.uint32)
            _check(_L.fecl_lte_interleaver(int(length), _ptr(p)))
            return p

        @staticmethod
        def sizes():
            """The 188 message lengths of the LTE QPP table (3GPP TS 36.212 Table 5.1.3-3):
            40..512 step 8, 528..1024 step 16, 1056..2048 step 32, 2112..6144 step 64."""
            return (list(range(40, 513, 8)) + list(range(528, 1025, 16)) + list(range(1056, 2049, 32))
                    + list(range(2112, 6145, 64)))

    class EncoderOptions:
        """Turbo::EncoderOptions -- src/detail/Turbo.h:59-72."""

        def __init__(self, trellis, interleaver):
            self._trellis = list(trellis) if isinstance(trellis, (list, tuple)) else [trellis]
            self._perm = [np.asarray(p, dtype=np.uint32) for p in interleaver]
            self._term = [Trellis.Tail]

        def interleaver(self, perms):
            self._perm = [np.asarray(p, dtype=np.uint32) for p in perms]
            return self

        def termination(self, t):
            self._term = list(t) if isinstance(t, (list, tuple)) else [t]
            return self

    Alternate, Group = 0, 1  # Turbo::BitOrdering, src/detail/Turbo.h:54-57

    class Stage:
        """Turbo::Stage -- src/detail/Turbo.h:38-48: constituents decoded in the stage and,
        for each, the constituents whose extrinsic values form its a-priori input."""

        def __init__(self, activation, transfer):
            self.activation = [int(a) for a in activation]
            self.transfer = [[int(t) for t in lst] for lst in transfer]

    class PunctureOptions:
        """Turbo::PunctureOptions -- src/detail/Turbo.h: mask (one repeating mask per
        stream: systematic, then each constituent's parity), tailMask (two per
        constituent), bitOrdering (Alternate or Group)."""

        def __init__(self):
            self._mask, self._tail, self._ordering = [], [], 0

        def mask(self, m=None):
            if m is None:
                return [list(x) for x in self._mask]
            self._mask = [[bool(b) for b in x] for x in m]
            return self

        def tailMask(self, m=None):
            if m is None:
                return [list(x) for x in self._tail]
            self._tail = [[bool(b) for b in x] for x in m]
            return self

        def bitOrdering(self, o=None):
            if o is None:
                return self._ordering
            self._ordering = int(o)
            return self

    class DecoderOptions:
        """Turbo::DecoderOptions -- src/detail/Turbo.h:77-101."""

        def __init__(self):
            self._it, self._sched, self._alg, self._sf = 6, Serial, Linear, [[1.0]]
            self._precision = _lib.MSG_F32

        def iterations(self, n=None):
            if n is None:
                return self._it
            self._it = int(n)
            return self

        def scheduling(self, s=None):
            """Serial, Parallel, or a custom schedule: a list of Turbo.Stage (then the
            scheduling type is Custom, as DecoderOptions::scheduling(Scheduling) sets it)."""
            if s is None:
                return self._sched
            if isinstance(s, (list, tuple)):
                self._stages = [st if isinstance(st, Turbo.Stage) else Turbo.Stage(*st) for st in s]
                self._sched = Custom
            else:
                self._sched = int(s)
            return self

        def schedule(self):
            return list(getattr(self, "_stages", []))

        def crc(self, kind=None):
            """Extension: CRC24A / CRC24B when the message ends with that CRC of the rest;
            decode then stops each frame at the first iteration whose decisions pass it."""
            if kind is None:
                return getattr(self, "_crc", 0)
            self._crc = int(kind)
            return self

        def algorithm(self, a=None):
            if a is None:
                return self._alg
            self._alg = int(a)
            return self

        def scalingFactor(self, f=None):
            if f is None:
                return self._sf
            self._sf = [list(map(float, r)) for r in f] if isinstance(f, (list, tuple)) else [[float(f)]]
            return self

        def precision(self, p=None):
            if p is None:
                return self._precision
            self._precision = int(p)
            return self

    def __init__(self, encoder, decoder=None, workGroupSize=8, lte_length=None):
        decoder = decoder or Turbo.DecoderOptions()
        opts, keep = self._options(decoder)
        h = C.c_void_p()
        if lte_length is not None:
            _check(_L.fecl_turbo_create_lte(int(lte_length), C.byref(opts), C.byref(h)))
        else:
            tr = (_lib.fecl_trellis * len(encoder._trellis))(*[t._c() for t in encoder._trellis])
            lens = _u32([p.size for p in encoder._perm])
            data = _u32(np.concatenate(encoder._perm)) if sum(p.size for p in encoder._perm) else np.zeros(1, np.uint32)
            term = np.ascontiguousarray(np.asarray(encoder._term, dtype=np.int32))
            _check(_L.fecl_turbo_create(len(encoder._perm), tr, len(encoder._trellis), _ptr(data), _ptr(lens), _ptr(term),
                                        term.size, C.byref(opts), C.byref(h)))
        super().__init__(h.value)
        self._decoder = decoder
        self._work_group = workGroupSize

    @classmethod
    def lte(cls, K, decoder=None):
        """The LTE turbo code of 3GPP TS 36.212 for block size K: RSC (13, 15) octal,
        Tail, {identity, Lte3Gpp.interleaver(K)}."""
        return cls(None, decoder, lte_length=K)

    def _options(self, d):
        rows = [list(np.atleast_1d(np.asarray(r, dtype=np.float64))) for r in d.scalingFactor()]
        width = max((len(r) for r in rows), default=0)
        # rows of 1 entry cycle like rows of `iterations` entries (src/detail/Turbo.cpp:148-153):
        # widen them so that the table is rectangular
        if any(len(r) not in (1, width) for r in rows):
            raise ValueError("Wrong size for scaling factor")
        sf = np.ascontiguousarray(np.asarray([r * width if len(r) == 1 else r for r in rows], dtype=np.float64))
        if sf.ndim != 2 or sf.size == 0:
            raise ValueError("Wrong size for scaling factor")
        o = _lib.fecl_turbo_options()
        o.algorithm = d.algorithm()
        o.iterations = d.iterations()
        o.scheduling = d.scheduling()
        o.scaling = sf.ctypes.data_as(C.POINTER(C.c_double))
        o.scaling_rows, o.scaling_cols = sf.shape
        o.precision = d.precision()
        self._sf_table = sf
        o.crc = d.crc()
        stages = d.schedule() if d.scheduling() == Custom else []
        for st in stages:  # src/detail/Turbo.cpp:109-111 (the C-ABI pairs one transfer list with each activation)
            if len(st.activation) != len(st.transfer):
                raise ValueError("Invalid scheduling : activation and transfer not the same size")
        if stages:
            counts = _u32([len(st.activation) for st in stages])
            act = _u32([a for st in stages for a in st.activation] or [0])
            tcounts = _u32([len(t) for st in stages for t in st.transfer] or [0])
            tr = _u32([v for st in stages for t in st.transfer for v in t] or [0])
            self._sched_arrays = (counts, act, tcounts, tr)
            o.n_stages = len(stages)
            o.stage_counts, o.activation = counts.ctypes.data, act.ctypes.data
            o.transfer_counts, o.transfer = tcounts.ctypes.data, tr.ctypes.data
        return o, sf

    def setDecoderOptions(self, decoder):
        opts, keep = self._options(decoder)
        _check(_L.fecl_turbo_set_options(self._h, C.byref(opts)))
        self._decoder = decoder

    def puncturing(self, options):
        """Turbo::puncturing -- src/Turbo.h:102: the fec::Permutation of the kept code bits."""
        def flat(ms):
            data = np.asarray([b for x in ms for b in x], np.uint8)
            lens = np.asarray([len(x) for x in ms], np.uint32)
            return data, lens
        md, ml = flat(options._mask)
        td, tl = flat(options._tail)
        n = C.c_uint64()
        args = (_ptr(md), _ptr(ml), ml.size, _ptr(td), _ptr(tl), tl.size, options._ordering)
        _check(_L.fecl_turbo_puncturing(self._h, *args, None, C.byref(n)))
        seq = np.zeros(n.value, np.uint32)
        _check(_L.fecl_turbo_puncturing(self._h, *args, _ptr(seq), C.byref(n)))
        return Permutation(seq, self.paritySize())

    def setWindowTraining(self, steps):
        """Extension: training steps of the windowed LTE decoder (multiple of 8, -1 default)."""
        _check(_L.fecl_turbo_set_window_training(self._h, int(steps)))

    def setWindowSegments(self, segments):
        """Extension: forward/backward segments per frame of the windowed LTE decoder
        (32, 64 or 128, 0 for the built-in choice)."""
        _check(_L.fecl_turbo_set_window_segments(self._h, int(segments)))

    def tuneWindow(self, llr, out=None):
        """Extension: time the windowed LTE decoder's equivalent window shapes on these
        device L-values (a torch CUDA tensor) and keep the fastest; returns (segments,
        training steps).  `out` (uint8 CUDA tensor of the decisions) is optional."""
        import torch
        if not _is_device(llr):
            raise ValueError("tuneWindow needs L-values in device memory")
        n = self._frames(llr.numel(), self.paritySize(), "parity")
        if out is None:
            out = torch.empty(n * self.msgSize(), dtype=torch.uint8, device=llr.device)
        segs, train = C.c_int32(), C.c_int32()
        stream = torch.cuda.current_stream(llr.device).cuda_stream
        _check(_L.fecl_turbo_tune_window(self._h, C.c_void_p(llr.data_ptr()), _dtype_code(llr), n,
                                         C.c_void_p(out.data_ptr()), C.c_void_p(stream), C.byref(segs), C.byref(train)))
        return segs.value, train.value

    def windowStats(self):
        """Extension: (passes, fix-up rounds, recomputed segments) since the last call."""
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(_L.fecl_turbo_window_stats(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def getDecoderOptions(self):
        return self._decoder


class Convolutional(Codec):
    """fec::Convolutional -- src/Convolutional.h:40-81: decode by Viterbi, soDecode by
    the MAP decoder, on the GPU."""

    class EncoderOptions:
        """Convolutional::EncoderOptions -- src/detail/Convolutional.h:36-46 (termination
        defaults to Truncate)."""

        def __init__(self, trellis, length):
            self._trellis = trellis
            self._length = int(length)
            self._term = Trellis.Truncate

        def termination(self, t=None):
            if t is None:
                return self._term
            self._term = int(t)
            return self

    class DecoderOptions:
        """Convolutional::DecoderOptions -- src/detail/Convolutional.h:48-62."""

        def __init__(self):
            self._alg = Approximate
            self._sf = 1.0

        def algorithm(self, a=None):
            if a is None:
                return self._alg
            self._alg = int(a)
            return self

        def scalingFactor(self, f=None):
            if f is None:
                return self._sf
            self._sf = float(f)
            return self

    class PunctureOptions:
        """Convolutional::PunctureOptions -- src/detail/Convolutional.h:64-75."""

        def __init__(self):
            self._mask, self._tail = [], []

        def mask(self, m=None):
            if m is None:
                return list(self._mask)
            self._mask = [bool(x) for x in m]
            return self

        def tailMask(self, m=None):
            if m is None:
                return list(self._tail)
            self._tail = [bool(x) for x in m]
            return self

    def __init__(self, encoder, decoder=None, workGroupSize=8):
        decoder = decoder or Convolutional.DecoderOptions()
        o = _lib.fecl_conv_options(decoder._alg, decoder._sf)
        tr = encoder._trellis._c()
        h = C.c_void_p()
        _check(_L.fecl_conv_create(C.byref(tr), encoder._length, encoder._term, C.byref(o), C.byref(h)))
        super().__init__(h.value)
        self._decoder = decoder
        self._work_group = workGroupSize

    def setDecoderOptions(self, decoder):
        o = _lib.fecl_conv_options(decoder._alg, decoder._sf)
        _check(_L.fecl_conv_set_options(self._h, C.byref(o)))
        self._decoder = decoder

    def getDecoderOptions(self):
        return self._decoder

    def puncturing(self, options):
        """Convolutional::puncturing -- src/Convolutional.h:73."""
        m = np.asarray(options._mask, np.uint8)
        t = np.asarray(options._tail, np.uint8)
        n = C.c_uint64()
        _check(_L.fecl_conv_puncturing(self._h, _ptr(m), m.size, _ptr(t), t.size, None, C.byref(n)))
        seq = np.zeros(n.value, np.uint32)
        _check(_L.fecl_conv_puncturing(self._h, _ptr(m), m.size, _ptr(t), t.size, _ptr(seq), C.byref(n)))
        return Permutation(seq, self.paritySize())


class Permutation:
    """fec::Permutation -- src/Permutation.h: a sequence of input indices.  permute()
    gathers out[i] = in[seq[i]] block by block; dePermute() scatters back and leaves
    zeros (erasures) where nothing maps.  Both run on the GPU: torch CUDA tensors stay
    there (asynchronous on the current stream); numpy arrays are copied through."""

    def __init__(self, sequence, inputSize=None):
        self._seq = np.ascontiguousarray(np.asarray(sequence, np.uint32).ravel())
        self._in = int(inputSize) if inputSize is not None else (int(self._seq.max()) + 1 if self._seq.size else 0)
        self._h = None

    def inputSize(self):
        return self._in

    def outputSize(self):
        return int(self._seq.size)

    def __getitem__(self, i):
        return int(self._seq[i])

    def sequence(self):
        return self._seq.copy()

    def _handle(self):
        if self._h is None:
            h = C.c_void_p()
            _check(_L.fecl_permutation_create(_ptr(self._seq), self._seq.size, self._in, C.byref(h)))
            self._h = h
        return self._h

    def _apply(self, x, inverse):
        import torch
        host = not _is_device(x)
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(x))).cuda() if host else x.contiguous()
        t = t.view(-1)
        codes = {torch.float64: _lib.F64, torch.float32: _lib.F32, torch.float16: _lib.F16, torch.uint8: _lib.U8}
        if t.dtype not in codes:
            raise ValueError("unsupported element type")
        size_in, size_out = (self.outputSize(), self._in) if inverse else (self._in, self.outputSize())
        if size_in == 0 or t.numel() % size_in:
            raise ValueError("Invalid input size")
        nb = t.numel() // size_in
        out = torch.empty(nb * size_out, dtype=t.dtype, device=t.device)
        stream = torch.cuda.current_stream(t.device).cuda_stream
        _check(_L.fecl_permute(self._handle(), C.c_void_p(t.data_ptr()), codes[t.dtype], nb, C.c_void_p(out.data_ptr()),
                               1 if inverse else 0, C.c_void_p(stream)))
        return out.cpu().numpy() if host else out

    def permute(self, x):
        return self._apply(x, False)

    def dePermute(self, x):
        return self._apply(x, True)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _L.fecl_permutation_destroy(h)
            self._h = None


class Batch:
    """Extension: frames of several codecs decoded by one CUDA graph launch
    (fecl_batch_create in include/fecl_b200.h).

    jobs is a list of (codec, llr, msg) or (codec, llr, msg, iterations) with torch
    CUDA tensors: llr [nframes * paritySize] (float16/32/64), msg [nframes * msgSize]
    uint8, iterations [nframes] int32.  The tensors stay bound to the batch: write new
    L-values into them and call run() again.  Results equal each codec's decode()
    bit for bit.  autotune=True times the equivalent LDPC kernel shapes on these
    inputs at creation and keeps the fastest.  shared_ldpc="passes" runs the FP16
    LDPC jobs with shared launches per pass, "persistent" with one shared persistent
    launch per check-degree class, instead of their own launches (same results)."""

    def __init__(self, jobs, autotune=False, shared_ldpc=None):
        self._keep = []
        arr = (_lib.fecl_batch_job * len(jobs))()
        for i, job in enumerate(jobs):
            codec, llr, msg = job[:3]
            it = job[3] if len(job) > 3 else None
            if not (_is_device(llr) and _is_device(msg) and (it is None or _is_device(it))):
                raise ValueError("batch buffers must be CUDA tensors")
            n = codec._frames(llr.numel(), codec.paritySize(), "parity")
            if msg.numel() != n * codec.msgSize():
                raise ValueError("Invalid size for message")
            if it is not None and it.numel() != n:
                raise ValueError("Invalid size for iterations")
            arr[i].codec = codec._h
            arr[i].nframes = n
            arr[i].llr = llr.data_ptr()
            arr[i].llr_dtype = _dtype_code(llr)
            arr[i].msg = msg.data_ptr()
            arr[i].iterations = it.data_ptr() if it is not None else None
            self._keep.append((codec, llr, msg, it))
        h = C.c_void_p()
        flags = _lib.BATCH_AUTOTUNE if autotune else 0
        if shared_ldpc == "passes":
            flags |= _lib.BATCH_SHARED_LDPC
        elif shared_ldpc == "persistent":
            flags |= _lib.BATCH_SHARED_PERSISTENT
        elif shared_ldpc not in (None, False):
            raise ValueError("shared_ldpc must be None, 'passes' or 'persistent'")
        _check(_L.fecl_batch_create(arr, len(jobs), flags, C.byref(h)))
        self._h = h
        self._device = jobs[0][1].device

    def run(self, stream=None):
        """Launches the batch on `stream` (default: torch's current stream)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self._device)
        _check(_L.fecl_batch_run(self._h, C.c_void_p(s.cuda_stream)))

    def describe(self):
        """One line per job: the kernel it runs."""
        buf = C.create_string_buffer(1 << 16)
        _check(_L.fecl_batch_describe(self._h, buf, len(buf)))
        return buf.value.decode()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value:
            _L.fecl_batch_destroy(h)
            self._h = None


class Server:
    """Extension: a decode server with continuous batching (fecl_server_* in
    include/fecl_b200.h).  Requests are numpy arrays of host L-values; the server
    batches whatever is waiting whenever one of its `slots` in-flight batches
    finishes, within device_budget bytes of device memory."""

    def __init__(self, device_budget=40 << 30, max_batch_frames=2048, slots=3):
        o = _lib.fecl_server_options(int(device_budget), int(max_batch_frames), int(slots))
        h = C.c_void_p()
        _check(_L.fecl_server_create(C.byref(o), C.byref(h)))
        self._h = h
        self._pending = {}

    def submit(self, codec, llr, iterations=False):
        """Queues the frames in `llr` (numpy, float16/32/64); returns a ticket."""
        x = np.asarray(llr)
        if x.dtype not in (np.float64, np.float32, np.float16):
            x = x.astype(np.float64)
        x = np.ascontiguousarray(x.ravel())
        n = codec._frames(x.size, codec.paritySize(), "parity")
        msg = np.zeros(n * codec.msgSize(), np.uint8)
        it = np.zeros(n, np.int32) if iterations else None
        t = C.c_uint64()
        _check(_L.fecl_server_submit(self._h, codec._h, _ptr(x), _dtype_code(x), n, _ptr(msg),
                                     _ptr(it) if it is not None else None, C.byref(t)))
        self._pending[t.value] = (codec, x, msg, it)
        return t.value

    def wait(self, ticket, timeout=600.0):
        """The request's decisions (and iteration counts when asked), and its latency in seconds."""
        lat = C.c_double()
        try:
            _check(_L.fecl_server_wait(self._h, int(ticket), float(timeout), C.byref(lat)))
        finally:
            entry = self._pending.pop(int(ticket), None)
        _, _, msg, it = entry
        return (msg, it, lat.value) if it is not None else (msg, lat.value)

    def report(self):
        st = _lib.fecl_server_stats()
        _check(_L.fecl_server_report(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def reset_stats(self):
        _check(_L.fecl_server_reset_stats(self._h))

    def replay(self, arrivals, requests):
        """Native load generator: request i = (codec, llr numpy) is submitted at
        arrivals[i] seconds after the call starts; returns (decisions, latencies)."""
        n = len(requests)
        arr = np.ascontiguousarray(np.asarray(arrivals, np.float64))
        codecs = (C.c_void_p * n)()
        llrs = (C.c_void_p * n)()
        msgs = (C.c_void_p * n)()
        dts = np.zeros(n, np.int32)
        nfr = np.zeros(n, np.uint64)
        keep, outs = [], []
        for i, (codec, llr) in enumerate(requests):
            x = np.ascontiguousarray(np.asarray(llr).ravel())
            nf = codec._frames(x.size, codec.paritySize(), "parity")
            m = np.zeros(nf * codec.msgSize(), np.uint8)
            codecs[i] = codec._h.value
            llrs[i] = x.ctypes.data
            msgs[i] = m.ctypes.data
            dts[i] = _dtype_code(x)
            nfr[i] = nf
            keep.append(x)
            outs.append(m)
        lat = np.zeros(n, np.float64)
        _check(_L.fecl_server_replay(self._h, n, _ptr(arr), C.cast(codecs, C.c_void_p), C.cast(llrs, C.c_void_p),
                                     _ptr(dts), _ptr(nfr), C.cast(msgs, C.c_void_p), None, _ptr(lat)))
        return outs, lat

    def close(self):
        h = getattr(self, "_h", None)
        if h and h.value:
            _L.fecl_server_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

