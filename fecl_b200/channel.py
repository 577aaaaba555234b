"""Seeded synthetic inputs: random message bits and BPSK over AWGN L-values.

Model (FeCl's sign convention, L = ln p(x=1)/p(x=0)):
  bit b -> x = 2b - 1;  Es/N0 = (Eb/N0) * R with R = message bits / transmitted bits;
  sigma^2 = 1 / (2 Es/N0);  y = x + N(0, sigma^2);  L = 2 y / sigma^2, in float64,
  then cast to the requested dtype.
The reference's own test channel (test/Cpp/operations.h:42-59) is the same model
written as L = (+-1) * N(4 snr, 4 sqrt(snr / 2)) with snr = Es/N0.

Draws come from numpy's counter-based Philox generator keyed by `seed`, so every
consumer (GPU decoder, CPU oracle, bench) sees identical inputs.
"""
import numpy as np


def _rng(seed, stream):
    return np.random.Generator(np.random.Philox(key=[int(seed) & 0xFFFFFFFFFFFFFFFF, int(stream)]))


def random_bits(n, seed):
    return _rng(seed, 1).integers(0, 2, size=int(n), dtype=np.uint8)


def awgn_llr(bits, ebn0_db, rate, seed, dtype=np.float64):
    bits = np.asarray(bits, dtype=np.uint8)
    esn0 = 10.0 ** (float(ebn0_db) / 10.0) * float(rate)
    sigma2 = 1.0 / (2.0 * esn0)
    y = (2.0 * bits.astype(np.float64) - 1.0) + _rng(seed, 2).normal(0.0, np.sqrt(sigma2), size=bits.size)
    return (2.0 * y / sigma2).astype(dtype)


def awgn_llr_per_frame(bits, frame_size, ebn0_db, rate, seed, dtype=np.float64):
    """Like awgn_llr, with one Eb/N0 per frame (ebn0_db: array of nframes)."""
    bits = np.asarray(bits, dtype=np.uint8).reshape(-1, frame_size)
    esn0 = (10.0 ** (np.asarray(ebn0_db, dtype=np.float64) / 10.0) * float(rate))[:, None]
    sigma2 = 1.0 / (2.0 * esn0)
    y = (2.0 * bits.astype(np.float64) - 1.0) + _rng(seed, 2).normal(0.0, 1.0, size=bits.shape) * np.sqrt(sigma2)
    return (2.0 * y / sigma2).astype(dtype).ravel()


def awgn_llr_device(bits, ebn0_db, rate, seed, dtype=None):
    """BPSK/AWGN L-values computed on the GPU (fecl_awgn_llr): bits is a torch CUDA
    uint8 tensor; returns a CUDA tensor of `dtype` (float32 by default).  Same model
    as awgn_llr, different generator (Philox-4x32-10 on the device)."""
    import ctypes as C
    import torch
    from . import _lib
    dtype = dtype or torch.float32
    code = {torch.float64: _lib.F64, torch.float32: _lib.F32, torch.float16: _lib.F16}[dtype]
    b = bits.contiguous().view(-1)
    out = torch.empty(b.numel(), dtype=dtype, device=b.device)
    stream = torch.cuda.current_stream(b.device).cuda_stream
    _lib.check(_lib.lib.fecl_awgn_llr(C.c_void_p(b.data_ptr()), b.numel(), float(ebn0_db), float(rate), int(seed) & (2**64 - 1),
                                      code, C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
    return out

