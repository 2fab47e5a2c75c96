"""ctypes binding of the C ABI in ``include/srf_b200.h`` (``libsrf_b200.so``).

The library is the only compute path: if it cannot be loaded (or built with nvcc when
it is missing) every op raises. Device pointers come from torch tensors; the CUDA
stream is torch's current stream on the tensors' device.
"""

import ctypes as C
import os
import threading

from . import build as _build

_p = C.c_void_p
_f = C.c_float
_int = C.c_int
_i64 = C.c_int64

# (name, argtypes) of every entry point declared in include/srf_b200.h.
_TOR_COLS = [_p] * 10
_SID_COLS = [_p] * 7
SIGNATURES = {
    "srf_status_string": ([_int], C.c_char_p),
    "srf_last_cuda_error": ([], _int),
    "srf_version": ([], _int),
    "srf_launch_count": ([], _i64),
    "srf_release_scratch": ([], _int),
    "srf_tor_projection": (_TOR_COLS + [_int, _p, _p, _p, _p, _f, _f, _f, _p, _i64, _i64, _p],
                           _int),
    "srf_tor_backprojection": (_TOR_COLS + [_int, _p, _p, _p, _p, _f, _f, _f, _p, _i64, _i64,
                                            _int, _p], _int),
    "srf_tor_projection_backprojection": (_TOR_COLS + [_int, _p, _p, _p, _p, _f, _f, _f, _p, _p,
                                                   _i64, _i64, _int, _p], _int),
    "srf_tor_maplors": ([_p] * 7 + [_int, _p, _p, _p, _p, _f, _p, _i64, _i64, _int, _p], _int),
    "srf_tor_backproject_adjoint": (_TOR_COLS + [_int, _p, _p, _p, _p, _f, _f, _f, _p, _i64,
                                                 _i64, _int, _p], _int),
    "srf_siddon_projection": (_SID_COLS + [_p, _p, _p, _p, _f, _f, _p, _i64, _i64, _p], _int),
    "srf_siddon_backprojection": (_SID_COLS + [_p, _p, _p, _p, _f, _f, _p, _i64, _i64, _int,
                                               _p], _int),
    "srf_siddon_maplors": ([_p] * 6 + [_p, _p, _p, _p, _p, _i64, _i64, _int, _p], _int),
    "srf_siddon_backproject_adjoint": (_SID_COLS + [_p, _p, _p, _p, _f, _f, _p, _i64, _i64,
                                                    _int, _p], _int),
    "srf_tor_projection_batched": (_TOR_COLS + [_int, _p, _int, _i64, _p, _p, _p, _p, _f, _f, _f,
                                                _p, _i64, _i64, _p], _int),
    "srf_tor_backprojection_batched": (_TOR_COLS + [_int, _p, _int, _i64, _p, _p, _p, _p, _f, _f,
                                                    _f, _p, _i64, _i64, _int, _p], _int),
    "srf_tor_projection_backprojection_batched": (_TOR_COLS + [_int, _p, _int, _i64, _p, _p, _p,
                                                               _p, _f, _f, _f, _p, _p, _i64,
                                                               _i64, _int, _p], _int),
    "srf_tor_projection_backprojection_batched_strided": (
        _TOR_COLS + [_int, _p, _int, _i64, _p, _p, _p, _p, _f, _f, _f, _p, _p, _p, _i64, _i64,
                     _int, _p], _int),
    "srf_tor_backproject_adjoint_batched": (_TOR_COLS + [_int, _p, _int, _i64, _p, _p, _p, _p,
                                                         _f, _f, _f, _p, _i64, _i64, _int, _p],
                                            _int),
    "srf_tor_set_tuning": ([_int, _int, _int], _int),
    "srf_siddon_set_tuning": ([_int], _int),
    "srf_tor_set_scratch_limit": ([_i64], _int),
    "srf_tor_maplors_generated": ([_int, _p, _int, _int, _int, C.c_uint64, _i64, _i64, _int,
                                   _int, _p, _p, _p, _f, _p, _int, _p], _int),
    "srf_tor_count_samples": ([_p] * 7 + [_int, _p, _p, _p, _f, _p, _i64, _i64, _p], _int),
    "srf_siddon_count_samples": ([_p] * 6 + [_p, _p, _p, _p, _i64, _i64, _p], _int),
    "srf_mlem_update": ([_p, _p, _p, _i64, _p], _int),
    "srf_preprocess_workspace_size": ([_i64], _i64),
    "srf_recon_process": ([_p, _i64, _i64, C.c_double, _p, _p, _p, _i64, _p], _int),
    "srf_map_process": ([_p, _i64, _i64, _p, _p, _p, _i64, _p], _int),
    "srf_recon_process_noalloc": ([_p, _i64, _i64, C.c_double, _p, _p, _p], _int),
    "srf_csr_spmm": ([_p, _p, _p, _i64, _i64, _p, _int, _p, _int, _p], _int),
    "srf_psf_apply": ([_p, _p, _p, _i64, _i64, _p, _int, _p, _int, _p, _int, _p], _int),
    "srf_order_by_direction": ([_p, _i64, _int, _i64, _p, _p], _int),
    "srf_probe_threads": ([_p], _int),
    "srf_probe_l2_read": ([_p, _i64, _int, _p, _p], _int),
    "srf_probe_ex2": ([_int, _p, _p], _int),
    "srf_probe_smem_threads": ([_p], _int),
    "srf_probe_smem_read": ([_int, _p, _p], _int),
    "srf_probe_smem_atomic": ([_int, _int, _p, _p], _int),
}


class SRFError(RuntimeError):
    """A non-zero status from the CUDA library."""

    def __init__(self, func, status, lib):
        msg = lib.srf_status_string(status).decode()
        cuda = lib.srf_last_cuda_error() if status == 2 else 0
        super().__init__(f"{func} failed: {msg} (status {status}"
                         + (f", cuda error {cuda})" if cuda else ")"))
        self.status = status
        self.cuda_error = cuda


_LOCK = threading.Lock()
_LIB = None


def library_path():
    return _build.LIBPATH


def load():
    """Load (building first if needed) libsrf_b200.so and declare its signatures."""
    global _LIB
    if _LIB is not None:
        return _LIB
    with _LOCK:
        if _LIB is None:
            if not _build.up_to_date():
                _build.build()
            lib = C.CDLL(_build.LIBPATH)
            for name, (args, res) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.argtypes = args
                fn.restype = res
            _LIB = lib
    return _LIB


def call(name, *args):
    lib = load()
    st = getattr(lib, name)(*args)
    if st != 0:
        raise SRFError(name, st, lib)
    return st


def call_raw(name, *args):
    """Call an entry point that returns a value rather than a status."""
    return getattr(load(), name)(*args)


def exported_symbols():
    return list(SIGNATURES)
