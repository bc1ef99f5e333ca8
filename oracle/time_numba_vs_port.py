"""Single-thread rate of the reference's numba pair_correlation against the
oracle port on the same forest pairs.  TEST INFRASTRUCTURE ONLY (it backs the
statement about the CPU baseline; the benchmark's CPU legs time the port).

Run where the lya2pcf reference tree is available, named by the required
LYA2PCF_REFERENCE environment variable:

    LYA2PCF_REFERENCE=<reference tree> python oracle/time_numba_vs_port.py

Workload: a seeded sample of 400 neighbouring forest pairs of the
configuration-1 catalogue at scale 0.01 (the bench's catalogue shape), each
pair through the reference's numba kernel (correlation_procedures_cpu.py:46-84,
JIT warmed up first) and through the oracle with one thread, in both of its
modes (the numba kernel's CPU formula, and the GPU kernel's formula the
benchmark used to time), and through the W/DW-only port the benchmark's CPU
legs time (orc_corr_wdw).  Prints one JSON line of pixel pairs per second.
"""
import json
import os
import sys
import time

import numpy as np

REF = os.environ.get('LYA2PCF_REFERENCE', '')
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def main():
    if not REF:
        raise SystemExit('set LYA2PCF_REFERENCE to the lya2pcf reference tree')
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:] = [x for x in sys.path if os.path.abspath(x or '.') != here]   # the package, not oracle.py
    sys.path.insert(0, ROOT)
    from lya2pcf_b200 import synthetic
    from oracle import oracle as O
    sys.path.insert(0, REF)
    import correlation_procedures_cpu as cpu   # the reference module, read-only
    fs = synthetic.make(1, scale=0.01)
    am = synthetic.angmax_for(fs)
    cpu.init({}, None, (50, 50), am)
    off, nbr = O.neighbours(fs, am)
    f1, f2, _, _ = O.items_from_csr(fs, off, nbr)
    sel = np.random.default_rng(3).choice(len(f1), 400, replace=False)
    a, b = f1[sel], f2[sel]
    L = fs.lengths
    pairs = float(np.sum(L[a] * L[b]))
    seg = lambda f, x: x[fs.start[f]:fs.start[f + 1]]   # noqa: E731
    args = [(am, float(fs.ra[p]), float(fs.dec[p]), seg(p, fs.w), seg(p, fs.dw), 0, seg(p, fs.dc), 0,
             float(fs.ra[q]), float(fs.dec[q]), seg(q, fs.w), seg(q, fs.dw), 0, seg(q, fs.dc), 0) for p, q in zip(a, b)]
    cpu.pair_correlation(*args[0])            # JIT
    t = time.perf_counter()
    for x in args:
        cpu.pair_correlation(*x)
    t_numba = time.perf_counter() - t
    cat = O.Catalog(fs)
    res = {'pixel_pairs': pairs, 'forest_pairs': len(a), 'numba_pairs_per_s': pairs / t_numba}
    for name, mode in (('port_cpu_formula', O.CPU_FORMULA), ('port_gpu_formula', O.GPU_FORMULA)):
        t = time.perf_counter()
        O.corr(fs, a, b, [0, len(a)], mode=mode, angmax=am, nthreads=1, cat=cat)
        res[f'{name}_pairs_per_s'] = pairs / (time.perf_counter() - t)
    t = time.perf_counter()
    O.corr_wdw(fs, a, b, [0, len(a)], nthreads=1, cat=cat)
    res['port_wdw_pairs_per_s'] = pairs / (time.perf_counter() - t)
    res['port_gpu_formula_over_numba'] = res['port_gpu_formula_pairs_per_s'] / res['numba_pairs_per_s']
    res['port_wdw_over_numba'] = res['port_wdw_pairs_per_s'] / res['numba_pairs_per_s']
    print(json.dumps(res))


if __name__ == '__main__':
    main()
