"""The ctypes binding against include/lya2pcf.h (no GPU needed): every
prototype's parameter and return types match the ctypes signature used to call
it, and the option and statistics structs have the C compiler's size and field
offsets.  A mismatch here would pass garbage through the C ABI silently."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

from lya2pcf_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'lya2pcf.h')

SCALARS = {'int': C.c_int, 'int32_t': C.c_int32, 'int64_t': C.c_int64, 'double': C.c_double}


def prototypes():
    """{name: (return type text, [parameter texts])} of every entry point."""
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    text = re.sub(r'//[^\n]*', '', text)
    out = {}
    for ret, name, params in re.findall(r'(int|const char\s*\*)\s+(lya_[a-z0-9_]+)\s*\(([^)]*)\)\s*;', text):
        params = ' '.join(params.split())
        plist = [] if params in ('', 'void') else [p.strip() for p in params.split(',')]
        out[name] = (ret.replace(' ', ''), plist)
    return out


def _is_pointer_ctype(t):
    return t in (C.c_void_p, C.c_char_p) or (isinstance(t, type) and issubclass(t, C._Pointer))


def _check_param(name, k, text, ct):
    if '*' in text:
        assert _is_pointer_ctype(ct), f'{name} argument {k} ({text}) is a pointer, ctypes has {ct}'
        return
    base = text.replace('const ', '').split()[0]
    assert base in SCALARS, f'{name} argument {k}: unexpected C type {text}'
    want = SCALARS[base]
    assert not _is_pointer_ctype(ct), f'{name} argument {k} ({text}) is a scalar, ctypes has a pointer'
    assert C.sizeof(ct) == C.sizeof(want), f'{name} argument {k} ({text}): size {C.sizeof(ct)} != {C.sizeof(want)}'
    assert (want is C.c_double) == (ct is C.c_double), f'{name} argument {k} ({text}): float/integer mismatch'


def test_prototypes_match_ctypes_signatures():
    protos = prototypes()
    assert set(protos) == set(N.SIGNATURES), set(protos) ^ set(N.SIGNATURES)
    for name, (ret, params) in protos.items():
        args, res = N.SIGNATURES[name]
        assert len(params) == len(args), f'{name}: {len(params)} C parameters, {len(args)} ctypes arguments'
        for k, (text, ct) in enumerate(zip(params, args)):
            _check_param(name, k, text, ct)
        assert res is (C.c_char_p if ret == 'constchar*' else C.c_int), f'{name}: return type {ret} vs {res}'


@pytest.mark.skipif(shutil.which('gcc') is None, reason='gcc not installed')
@pytest.mark.parametrize('cname, cls', [('lya_corr_opts', N.CorrOpts), ('lya_stats_t', N.Stats)])
def test_struct_layout_matches_c(tmp_path, cname, cls):
    fields = [f for f, _ in cls._fields_]
    src = tmp_path / 'layout.c'
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "lya2pcf.h"', 'int main(void) {',
             f'  printf("%zu\\n", sizeof({cname}));']
    lines += [f'  printf("%zu %zu\\n", offsetof({cname}, {f}), sizeof((({cname}*)0)->{f}));' for f in fields]
    lines += ['  return 0;', '}']
    src.write_text('\n'.join(lines) + '\n')
    exe = tmp_path / 'layout'
    subprocess.run(['gcc', '-std=c99', '-I', os.path.join(ROOT, 'include'), str(src), '-o', str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split('\n')
    assert int(out[0]) == C.sizeof(cls), f'sizeof({cname}) {out[0]} != ctypes {C.sizeof(cls)}'
    for k, (f, ct) in enumerate(cls._fields_):
        off, size = (int(x) for x in out[1 + k].split())
        assert off == getattr(cls, f).offset, f'{cname}.{f}: offset {off} != ctypes {getattr(cls, f).offset}'
        assert size == C.sizeof(ct), f'{cname}.{f}: size {size} != ctypes {C.sizeof(ct)}'
