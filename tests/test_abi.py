"""The C-ABI library: loads, exports every entry point of include/lya2pcf.h,
and reports errors (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

from lya2pcf_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, 'include', 'lya2pcf.h')).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(lya_[a-z0-9_]+)\s*\(', text)))


def test_library_exports_every_declared_symbol():
    lib = N.load()
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(N.SIGNATURES), set(syms) - set(N.SIGNATURES)


def test_version_and_null_errors():
    lib = N.load()
    assert lib.lya_version() >= 10000
    # NULL context arguments are rejected with a message, never a crash
    assert lib.lya_set_bins(None, 200.0, 200.0, 50, 50) == 1
    assert b'ctx is NULL' in lib.lya_last_error(None)
    assert lib.lya_corr_run(None, None) == 1
    assert lib.lya_ctx_create(0, None) == 1


def test_no_silent_fallback_without_gpu():
    """Without a usable device the context cannot be created: the library
    fails loudly instead of falling back to a CPU path."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip('a GPU is present')
    except ImportError:
        pass
    lib = N.load()
    ctx = C.c_void_p()
    rc = lib.lya_ctx_create(0, C.byref(ctx))
    assert rc == 2
    assert b'no CUDA device' in lib.lya_last_error(None)
    with pytest.raises(N.LyaError):
        from lya2pcf_b200.engine import PairEngine
        PairEngine()
