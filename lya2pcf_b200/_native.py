"""ctypes binding of ``liblya2pcf.so`` (the C ABI declared in ``include/lya2pcf.h``).

The library is built in-tree by :mod:`lya2pcf_b200.build`.  Every call checks the
returned status and raises :class:`LyaError` with the library's message; there
is no fallback: without the library (or without a GPU) the calls fail loudly.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'liblya2pcf.so')

LYA_OK = 0
KERNEL_FP32_GUARDED = 0
KERNEL_FP64_DIAGONAL = 1
KERNEL_FP64_PLAIN = 2
VARIANT_TWO_DIAGONALS = 2   # lya_corr_opts.variant: FP32 kernel without its lean walk
NQ = 5
Q_W, Q_DW, Q_RP, Q_RT, Q_Z = range(NQ)

ERROR_NAMES = {1: 'ARG', 2: 'CUDA', 3: 'ALLOC', 4: 'STATE', 5: 'DATA', 6: 'GUARD', 7: 'DEVICE'}

# Every entry point of include/lya2pcf.h with its ctypes signature.
P = C.c_void_p
SIGNATURES = {
    'lya_ctx_create': ([C.c_int, C.POINTER(P)], C.c_int),
    'lya_ctx_destroy': ([P], C.c_int),
    'lya_last_error': ([P], C.c_char_p),
    'lya_version': ([], C.c_int),
    'lya_set_bins': ([P, C.c_double, C.c_double, C.c_int32, C.c_int32], C.c_int),
    'lya_upload_forests': ([P, C.c_int64, P, P, P, P, P, P, P, P, P, P, P, P, P, C.c_int32, P, P], C.c_int),
    'lya_upload_deltas': ([P, C.c_int64, P, P, P, P, P, P, P, P, P, P, P, P, P, C.c_int32, C.c_int32], C.c_int),
    'lya_get_projection': ([P, P, P, P, P], C.c_int),
    'lya_build_pairs': ([P, C.c_double, C.c_double, C.POINTER(C.c_int64)], C.c_int),
    'lya_set_pairs': ([P, C.c_int64, P, P], C.c_int),
    'lya_get_pairs': ([P, P, P], C.c_int),
    'lya_select_slots': ([P, P], C.c_int),
    'lya_debug_fail_alloc': ([C.c_int64], C.c_int),
    'lya_debug_inject': ([P, C.c_int32], C.c_int),
    'lya_probe_smem_atomics': ([C.c_int, P], C.c_int),
    'lya_corr_run': ([P, P], C.c_int),
    'lya_corr_get': ([P, C.c_int32, C.c_int32, P, P], C.c_int),
    'lya_corr_adjoint': ([P, P, P, P, C.c_int32], C.c_int),
    'lya_update_weights': ([P, P, P, C.c_int32], C.c_int),
    'lya_corr_totals': ([P, P, P, C.c_int32], C.c_int),
    'lya_stats': ([P, P], C.c_int),
    'lya_timer': ([P, C.c_int32, C.POINTER(C.c_double)], C.c_int),
    'lya_dist_run': ([P, P, P], C.c_int),
    'lya_dist_config': ([P, C.c_int32, C.c_int64], C.c_int),
    'lya_sync': ([P], C.c_int),
    'lya_covariance': ([P, C.c_int64, P, P, P, P], C.c_int),
    'lya_covariance_smooth': ([P, P, P, C.POINTER(C.c_int32)], C.c_int),
    'lya_corr_pixel_noalloc': ([C.c_int, P, P, P, P, P, P, P, P, P, P, C.c_int64, C.c_double, C.c_double,
                                C.c_int32, C.c_int32, P, P, P], C.c_int),
}


class LyaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f'lya2pcf error {code} ({ERROR_NAMES.get(code, "?")}): {msg}')
        self.code = code


class CorrOpts(C.Structure):
    _fields_ = [('kernel', C.c_int32), ('guard', C.c_double), ('warps_per_block', C.c_int32),
                ('blocks_per_sm', C.c_int32), ('slot_begin', C.c_int32), ('slot_end', C.c_int32),
                ('variant', C.c_int32), ('run_cap', C.c_int32)]


class Stats(C.Structure):
    _fields_ = [('ref_pairs', C.c_double), ('evaluated_pairs', C.c_double), ('guard_rechecks', C.c_double),
                ('runs_flushed', C.c_double), ('in_range_pairs', C.c_double), ('kernel_ms', C.c_double),
                ('build_ms', C.c_double), ('n_pairs', C.c_int64), ('n_slots', C.c_int32), ('n_forests', C.c_int32),
                ('guard_bound', C.c_double), ('run_ms', C.c_double), ('run_ref_pairs', C.c_double),
                ('launches', C.c_int64), ('ref_pixels', C.c_double), ('adjoint_ms', C.c_double),
                ('dist_mma_flops', C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load(path=None):
    """Load the native library (once).  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise LyaError(-1, f'native library not found at {path}; build it with python -m lya2pcf_b200.build')
    lib = C.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def check(rc, ctx=None):
    if rc != LYA_OK:
        msg = load().lya_last_error(ctx)
        raise LyaError(rc, msg.decode() if msg else '')
