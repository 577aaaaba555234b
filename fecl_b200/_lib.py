"""ctypes binding of libfecl_b200.so (the C-ABI declared in include/fecl_b200.h).

The library is loaded from this package directory.  There is no fallback: if the
library is missing or fails to load, importing fecl_b200 raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfecl_b200.so")

OK, EINVAL, ECUDA, ENOMEM, ETIMEDOUT, EUNSUPPORTED, ENODEV = 0, -1, -2, -3, -4, -5, -6
F64, F32, F16, U8 = 0, 1, 2, 3
MSG_F32, MSG_F16, MSG_I8 = 0, 1, 2
HOST_MEMORY, DEVICE_MEMORY = 0, 1
KERNEL_AUTO, KERNEL_GENERIC = 0, 1


class fecl_sizes(C.Structure):
    _fields_ = [("msg", C.c_uint64), ("syst", C.c_uint64), ("parity", C.c_uint64), ("state", C.c_uint64)]


class fecl_ldpc_options(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int32),
        ("iterations", C.c_uint32),
        ("scaling", C.POINTER(C.c_double)),
        ("scaling_iterations", C.c_uint32),
        ("scaling_degrees", C.c_uint32),
        ("precision", C.c_int32),
        ("fixed_iterations", C.c_int32),
    ]


class fecl_trellis(C.Structure):
    _fields_ = [
        ("state_count", C.c_uint32),
        ("input_count", C.c_uint32),
        ("output_size", C.c_uint32),
        ("next_state", C.POINTER(C.c_uint32)),
        ("output", C.POINTER(C.c_uint32)),
    ]


class fecl_turbo_options(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int32),
        ("iterations", C.c_uint32),
        ("scheduling", C.c_int32),
        ("scaling", C.POINTER(C.c_double)),
        ("scaling_rows", C.c_uint32),
        ("scaling_cols", C.c_uint32),
        ("precision", C.c_int32),
        ("n_stages", C.c_uint32),
        ("stage_counts", C.c_void_p),
        ("activation", C.c_void_p),
        ("transfer_counts", C.c_void_p),
        ("transfer", C.c_void_p),
        ("crc", C.c_int32),
    ]


class fecl_conv_options(C.Structure):
    _fields_ = [("algorithm", C.c_int32), ("scaling", C.c_double)]


class fecl_so_io(C.Structure):
    _fields_ = [
        ("parity", C.c_void_p),
        ("syst", C.c_void_p),
        ("state", C.c_void_p),
        ("in_dtype", C.c_int32),
        ("msg", C.c_void_p),
        ("syst_out", C.c_void_p),
        ("parity_out", C.c_void_p),
        ("state_out", C.c_void_p),
        ("out_dtype", C.c_int32),
    ]


class fecl_batch_job(C.Structure):
    _fields_ = [
        ("codec", C.c_void_p),
        ("nframes", C.c_uint64),
        ("llr", C.c_void_p),
        ("llr_dtype", C.c_int32),
        ("msg", C.c_void_p),
        ("iterations", C.c_void_p),
    ]


BATCH_AUTOTUNE = 1
BATCH_SHARED_LDPC = 2
BATCH_SHARED_PERSISTENT = 4


class fecl_server_options(C.Structure):
    _fields_ = [("device_budget_bytes", C.c_uint64), ("max_batch_frames", C.c_uint32), ("slots", C.c_uint32)]


class fecl_server_stats(C.Structure):
    _fields_ = [
        ("requests", C.c_uint64), ("frames", C.c_uint64), ("info_bits", C.c_uint64), ("batches", C.c_uint64),
        ("p50_s", C.c_double), ("p99_s", C.c_double), ("max_s", C.c_double), ("wall_s", C.c_double),
        ("batch_gpu_s", C.c_double), ("batch_host_s", C.c_double), ("batch_frames", C.c_double),
    ]


# (name, restype, argtypes) for every symbol include/fecl_b200.h declares.
SIGNATURES = [
    ("fecl_ldpc_create", C.c_int, [C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.POINTER(fecl_ldpc_options), C.POINTER(C.c_void_p)]),
    ("fecl_ldpc_set_options", C.c_int, [C.c_void_p, C.POINTER(fecl_ldpc_options)]),
    ("fecl_ldpc_checks", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.c_void_p, C.c_void_p]),
    ("fecl_dvbs2_matrix", C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.c_void_p, C.c_void_p]),
    ("fecl_gallager_matrix", C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.c_void_p, C.c_void_p]),
    ("fecl_trellis_build", C.c_int, [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p]),
    ("fecl_turbo_create", C.c_int, [C.c_uint32, C.POINTER(fecl_trellis), C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(fecl_turbo_options), C.POINTER(C.c_void_p)]),
    ("fecl_turbo_create_lte", C.c_int, [C.c_uint32, C.POINTER(fecl_turbo_options), C.POINTER(C.c_void_p)]),
    ("fecl_lte_interleaver", C.c_int, [C.c_uint32, C.c_void_p]),
    ("fecl_turbo_set_options", C.c_int, [C.c_void_p, C.POINTER(fecl_turbo_options)]),
    ("fecl_conv_create", C.c_int, [C.POINTER(fecl_trellis), C.c_uint32, C.c_int32, C.POINTER(fecl_conv_options),
                                   C.POINTER(C.c_void_p)]),
    ("fecl_conv_set_options", C.c_int, [C.c_void_p, C.POINTER(fecl_conv_options)]),
    ("fecl_conv_puncturing", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                       C.POINTER(C.c_uint64)]),
    ("fecl_codec_sizes", C.c_int, [C.c_void_p, C.POINTER(fecl_sizes)]),
    ("fecl_encode", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_int32, C.c_void_p]),
    ("fecl_check", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_int32)]),
    ("fecl_awgn_llr", C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.c_double, C.c_uint64, C.c_int32, C.c_void_p,
                                C.c_void_p]),
    ("fecl_decode", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    ("fecl_so_decode", C.c_int, [C.c_void_p, C.POINTER(fecl_so_io), C.c_uint64, C.c_int32, C.c_void_p]),
    ("fecl_destroy", None, [C.c_void_p]),
    ("fecl_crc24_attach", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p]),
    ("fecl_crc24_check", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p]),
    ("fecl_ldpc_puncturing", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                       C.POINTER(C.c_uint64)]),
    ("fecl_turbo_puncturing", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                        C.c_uint32, C.c_int32, C.c_void_p, C.POINTER(C.c_uint64)]),
    ("fecl_permutation_create", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(C.c_void_p)]),
    ("fecl_permute", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_uint64, C.c_void_p, C.c_int32, C.c_void_p]),
    ("fecl_permutation_destroy", None, [C.c_void_p]),
    ("fecl_set_kernel", C.c_int, [C.c_void_p, C.c_int32]),
    ("fecl_ldpc_set_cluster_shape", C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    ("fecl_ldpc_set_wave", C.c_int, [C.c_void_p, C.c_int32]),
    ("fecl_ldpc_set_persistent", C.c_int, [C.c_void_p, C.c_int32]),
    ("fecl_turbo_set_window_training", C.c_int, [C.c_void_p, C.c_int32]),
    ("fecl_turbo_set_window_segments", C.c_int, [C.c_void_p, C.c_int32]),
    ("fecl_turbo_tune_window", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_uint64, C.c_void_p, C.c_void_p,
                                         C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("fecl_turbo_window_stats", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("fecl_lte_turbo_decode_noalloc", C.c_int, [C.c_uint32, C.c_int32, C.c_uint32, C.c_void_p, C.c_int32, C.c_uint64, C.c_void_p, C.c_void_p]),
    ("fecl_batch_create", C.c_int, [C.POINTER(fecl_batch_job), C.c_uint32, C.c_int32, C.POINTER(C.c_void_p)]),
    ("fecl_batch_run", C.c_int, [C.c_void_p, C.c_void_p]),
    ("fecl_batch_describe", C.c_int, [C.c_void_p, C.c_char_p, C.c_uint64]),
    ("fecl_batch_destroy", None, [C.c_void_p]),
    ("fecl_server_create", C.c_int, [C.POINTER(fecl_server_options), C.POINTER(C.c_void_p)]),
    ("fecl_server_submit", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_uint64, C.c_void_p, C.c_void_p,
                                     C.POINTER(C.c_uint64)]),
    ("fecl_server_wait", C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(C.c_double)]),
    ("fecl_server_report", C.c_int, [C.c_void_p, C.POINTER(fecl_server_stats)]),
    ("fecl_server_reset_stats", C.c_int, [C.c_void_p]),
    ("fecl_server_replay", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    ("fecl_server_destroy", None, [C.c_void_p]),
    ("fecl_strerror", C.c_char_p, [C.c_int]),
    ("fecl_last_error", C.c_char_p, []),
    ("fecl_version", C.c_char_p, []),
]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("libfecl_b200.so is not built (run __graft_entry__.build() or make -C fecl_b200/csrc)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class FeclError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (%s)" % (message, lib.fecl_strerror(status).decode()))
        self.status = status


def check(status):
    """Raise on a non-zero status; invalid arguments raise ValueError like the
    reference's std::invalid_argument."""
    if status != OK:
        msg = lib.fecl_last_error().decode()
        if status == EINVAL:
            raise ValueError(msg)
        raise FeclError(status, msg)
