"""ctypes bindings of the engine's C ABI (include/pava_gpu.h, include/pava_host.h).

The CUDA library is the product path: if ``lib/libpava_gpu.so`` is missing, importing the
GPU entry points raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")

_GPU = None
_HOST = None

c_int, c_ll, c_dbl, c_void_p, c_char_p = (ctypes.c_int, ctypes.c_longlong, ctypes.c_double,
                                          ctypes.c_void_p, ctypes.c_char_p)
c_u64 = ctypes.c_uint64
c_size_t = ctypes.c_size_t

# status codes (include/pava_gpu.h)
SUCCESS = 0
E_UNKNOWN_FORMAT = -1
E_UNSUPPORTED_PARAMS = -2
E_CONVERT_FAILED = -3
E_NOT_CONVERTED = -4
E_UNSUPPORTED_VALUE_TYPE = -5
E_INVALID_ARG = -10
E_INVALID_CSR = -11
E_CUDA = -12
E_NOMEM = -13
E_TIMEOUT = -14
E_TOO_LARGE = -15

FORMAT_CSR, FORMAT_CSR5, FORMAT_CVR, FORMAT_SELL = 0, 1, 3, 4
PREC_FP64, PREC_FP32C = 0, 1
INDEX_I32, INDEX_DELTA16, INDEX_AUTO = 0, 1, 2


class PavaCsr(ctypes.Structure):
    _fields_ = [("m", c_int), ("n", c_int), ("nnz", c_int), ("row_ptr", c_void_p),
                ("col_idx", c_void_p), ("vals", c_void_p), ("on_device", c_int)]


class PavaOpts(ctypes.Structure):
    _fields_ = [("steps", c_int), ("sigma", c_int), ("tiles_per_chunk", c_int),
                ("precision", c_int), ("index_mode", c_int), ("lanes_per_row", c_int),
                ("col_lanes", c_int), ("cols_per_lane", c_int), ("rows_per_tile", c_int),
                ("x_window", c_int)]


class PavaInfo(ctypes.Structure):
    _fields_ = [("format", c_int), ("precision", c_int), ("index_mode", c_int), ("m", c_int),
                ("n", c_int), ("nnz", c_int), ("n_empty", c_int), ("chunks", c_ll),
                ("elems_per_chunk", c_ll), ("convert_ms", c_dbl), ("device_bytes", c_size_t),
                ("alg_bytes", c_dbl), ("format_bytes", c_dbl)]


class PavaRunRecord(ctypes.Structure):
    _fields_ = [("status", c_int), ("format", c_int), ("precision", c_int),
                ("index_mode", c_int), ("steps", c_int), ("sigma", c_int),
                ("tiles_per_chunk", c_int), ("lanes_per_row", c_int), ("sm_count", c_int),
                ("iterations", c_int), ("chunks", c_ll), ("convert_s", c_dbl),
                ("exec_s", c_dbl), ("alg_bytes", c_dbl), ("format_bytes", c_dbl)]


class PavaTuneEntry(ctypes.Structure):
    _fields_ = [("format", c_int), ("opts", PavaOpts), ("ms", c_dbl), ("status", c_int)]


class PavaGenParams(ctypes.Structure):
    _fields_ = [("family", c_int), ("m", c_int), ("n", c_int), ("p0", c_dbl), ("p1", c_dbl),
                ("p2", c_dbl), ("p3", c_dbl)]


GEN_STENCIL, GEN_BANDED, GEN_POWERLAW, GEN_BLOCKDIAG = 0, 1, 2, 3
NVARIANTS, NFAMILIES, MLP_IN, MLP_HIDDEN, MLP_OUT, MLP_NPARAM = 32, 7, 12, 64, 32, 7072
TILES_WAVE = -1


class PavaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"pava status {status}: {msg}")
        self.status = status


# exported symbols and their prototypes: (name, restype, argtypes)
GPU_SYMBOLS = [
    ("pava_init", c_int, [c_int]),
    ("pava_set_device_memory_limit", c_int, [ctypes.c_ulonglong]),
    ("pava_bounds_checked", c_int, []),
    ("pava_bounds_report", c_int, [c_void_p, c_int]),
    ("pava_wait_report", c_int, [c_void_p, c_int]),
    ("pava_get_device_memory_limit", ctypes.c_ulonglong, []),
    ("pava_create", c_int, [ctypes.POINTER(PavaCsr), c_int, ctypes.POINTER(PavaOpts), c_void_p,
                            ctypes.POINTER(c_void_p)]),
    ("pava_spmv", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("pava_spmv_stage", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    ("pava_spmm", c_int, [c_void_p, c_int, c_void_p, c_ll, c_void_p, c_ll, c_void_p]),
    ("pava_spmv_host", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("pava_spmv_host_async", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("pava_spmv_host_wait", c_int, [c_void_p]),
    ("pava_get_info", c_int, [c_void_p, ctypes.POINTER(PavaInfo)]),
    ("pava_destroy", c_int, [c_void_p]),
    ("pava_last_error", c_char_p, []),
    ("pava_status_string", c_char_p, [c_int]),
    ("pava_spmv_csr_noalloc", c_int, [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                      c_void_p, c_void_p, c_void_p]),
    ("pava_batch_create", c_int, [c_int, ctypes.POINTER(PavaCsr), c_int,
                                  ctypes.POINTER(PavaOpts), c_void_p, ctypes.POINTER(c_void_p)]),
    ("pava_batch_create_spmm", c_int, [c_int, ctypes.POINTER(PavaCsr), c_int, c_int,
                                       ctypes.POINTER(PavaOpts), c_void_p,
                                       ctypes.POINTER(c_void_p)]),
    ("pava_batch_layout", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("pava_batch_get", c_int, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(PavaOpts),
                               ctypes.POINTER(PavaInfo)]),
    ("pava_batch_spmv", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("pava_batch_spmm", c_int, [c_void_p, c_int, c_void_p, c_ll, c_void_p, c_ll, c_void_p]),
    ("pava_batch_capture", c_int, [c_void_p, c_void_p, c_void_p]),
    ("pava_batch_capture_spmm", c_int, [c_void_p, c_int, c_void_p, c_ll, c_void_p, c_ll]),
    ("pava_batch_replay", c_int, [c_void_p, c_void_p]),
    ("pava_batch_destroy", c_int, [c_void_p]),
    ("pava_autotune", c_int, [ctypes.POINTER(PavaCsr), c_int, c_int, c_int,
                              ctypes.POINTER(PavaTuneEntry), c_int, ctypes.POINTER(c_int),
                              ctypes.POINTER(c_int)]),
    ("pava_gen_device", c_int, [ctypes.POINTER(PavaGenParams), c_u64, c_void_p,
                                ctypes.POINTER(PavaCsr)]),
    ("pava_free_device_csr", c_int, [ctypes.POINTER(PavaCsr)]),
    ("pava_features", c_int, [ctypes.POINTER(PavaCsr), c_void_p, c_void_p]),
    ("pava_variant", c_int, [c_int, ctypes.POINTER(c_int), ctypes.POINTER(PavaOpts)]),
    ("pava_variant_family", c_int, [c_int]),
    ("pava_time_variants", c_int, [ctypes.POINTER(PavaCsr), c_int, c_void_p,
                                   ctypes.POINTER(c_int)]),
    ("pava_mlp_create", c_int, [c_u64, ctypes.POINTER(c_void_p)]),
    ("pava_mlp_get_params", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("pava_mlp_set_params", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("pava_mlp_set_batch", c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    ("pava_mlp_forward", c_int, [c_void_p, c_void_p]),
    ("pava_mlp_gradient", c_int, [c_void_p, c_void_p, c_void_p]),
    ("pava_mlp_train", c_int, [c_void_p, c_int, ctypes.c_float, c_void_p]),
    ("pava_mlp_destroy", c_int, [c_void_p]),
    ("pava_select", c_int, [c_void_p, ctypes.POINTER(PavaCsr), ctypes.POINTER(c_int),
                            c_void_p]),
    ("pava_create_selected", c_int, [ctypes.POINTER(PavaCsr), c_void_p, c_void_p,
                                     ctypes.POINTER(c_void_p), ctypes.POINTER(c_int)]),
    ("pava_coo_to_csr_device", c_int, [c_int, c_int, c_ll, c_void_p, c_void_p, c_void_p, c_int,
                                       c_int, c_void_p, ctypes.POINTER(PavaCsr)]),
    ("pava_conduct", c_int, [c_int, ctypes.POINTER(PavaCsr), c_void_p, c_void_p, c_char_p, c_int,
                             ctypes.POINTER(PavaOpts), ctypes.POINTER(PavaRunRecord)]),
    ("conduct_cvr_gpu", c_int, [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_int, c_char_p, c_int]),
    ("conduct_csr5_gpu", c_int, [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_void_p, c_dbl, c_char_p, c_int]),
]

HOST_SYMBOLS = [
    ("pava_gen_laplace2d_rowptr", c_int, [c_int, c_void_p]),
    ("pava_gen_laplace2d_fill", c_int, [c_int, c_void_p, c_void_p, c_void_p]),
    ("pava_gen_powerlaw_rowptr", c_int, [c_int, c_int, c_dbl, c_dbl, c_int, c_dbl, c_u64,
                                         c_void_p]),
    ("pava_gen_powerlaw_fill", c_int, [c_int, c_int, c_u64, c_void_p, c_void_p, c_void_p]),
    ("pava_gen_stencil27_rowptr", c_int, [c_int, c_void_p]),
    ("pava_gen_stencil27_fill", c_int, [c_int, c_u64, c_void_p, c_void_p, c_void_p]),
    ("pava_gen_banded_rowptr", c_int, [c_int, c_int, c_int, c_void_p]),
    ("pava_gen_banded_fill", c_int, [c_int, c_int, c_u64, c_void_p, c_void_p, c_void_p]),
    ("pava_gen_random_rowptr", c_int, [c_int, c_int, c_dbl, c_u64, c_void_p]),
    ("pava_gen_random_fill", c_int, [c_int, c_int, c_u64, c_void_p, c_void_p, c_void_p]),
    ("pava_gen_blockdiag_rowptr", c_int, [c_int, c_int, c_int, c_u64, c_void_p]),
    ("pava_gen_blockdiag_fill", c_int, [c_int, c_u64, c_void_p, c_void_p, c_void_p]),
    ("pava_gen_uniform", c_int, [c_int, c_dbl, c_dbl, c_u64, c_int, c_void_p]),
    ("pava_init_vectors", None, [c_int, c_int, c_void_p, c_void_p, c_void_p]),
    ("pava_mtx_info", c_int, [c_char_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                              ctypes.POINTER(c_ll), ctypes.POINTER(c_int),
                              ctypes.POINTER(c_int)]),
    ("pava_mtx_read", c_int, [c_char_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_ll)]),
    ("pava_mtx_write", c_int, [c_char_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    ("pava_coo_to_csr", c_int, [c_int, c_int, c_ll, c_void_p, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_void_p]),
]

PROBE_SYMBOLS = [
    ("pava_probe_floor", c_int, [c_int, c_void_p, c_void_p, c_void_p, c_ll, c_int, c_u64, c_int,
                                 c_int, c_void_p, c_void_p]),
    ("pava_probe_floor_out_len", c_ll, [c_int, c_int]),
    ("pava_probe_gather_tma", c_int, [c_void_p, c_ll, c_int, c_u64, c_int, c_void_p, c_void_p,
                                      c_void_p]),
]
_PROBE = None


def _bind(lib, symbols):
    for name, res, args in symbols:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def gpu_lib_path() -> str:
    """The engine library; PAVA_GPU_LIB names an alternative build (e.g. one compiled with
    other launch bounds for a tuning sweep)."""
    return os.environ.get("PAVA_GPU_LIB") or os.path.join(LIBDIR, "libpava_gpu.so")


def host_lib_path() -> str:
    return os.path.join(LIBDIR, "libpava_host.so")


def probe_lib_path() -> str:
    return os.path.join(LIBDIR, "libpava_probe.so")


def gpu():
    """The CUDA engine.  Raises if the library is not built (no CPU fallback exists)."""
    global _GPU
    if _GPU is None:
        path = gpu_lib_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python -m pava_b200.build`")
        _GPU = _bind(ctypes.CDLL(path), GPU_SYMBOLS)
    return _GPU


def host():
    global _HOST
    if _HOST is None:
        path = host_lib_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python -m pava_b200.build`")
        _HOST = _bind(ctypes.CDLL(path), HOST_SYMBOLS)
    return _HOST


def probe():
    """The floor kernels of include/pava_probe.h (measurement aids, not the product path)."""
    global _PROBE
    if _PROBE is None:
        path = probe_lib_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python -m pava_b200.build`")
        _PROBE = _bind(ctypes.CDLL(path), PROBE_SYMBOLS)
    return _PROBE


def check(status: int) -> None:
    if status != SUCCESS:
        msg = gpu().pava_last_error().decode(errors="replace")
        raise PavaError(status, msg or gpu().pava_status_string(status).decode())
