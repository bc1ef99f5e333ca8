"""Golden vectors of the reference's delta projection, quasar.fill_dw
(forest_class.py:48-68).

Run where the lya2pcf reference tree is available, named by the required
LYA2PCF_REFERENCE environment variable.  ``forest_class.py`` imports healpy at module level, which is
not installed here, so the script compiles only the ``fill_dw`` method of the
``quasar`` class from that file's syntax tree and calls it on a stand-in
object holding the weights.  Writes ``tests/golden/fill_dw_golden.npz``:
forests of seeded random lengths (including length 1, whose slope term is
0/0 = NaN in the reference), weights, deltas and log-lambda grids, and the
reference's dw, delta_lambda, omega and omega_delta_lambda2 for project=True
and dw for project=False.
"""
import ast
import os
import types

import numpy as np

REF = os.environ.get('LYA2PCF_REFERENCE', '')
if __name__ == '__main__' and not REF:
    raise SystemExit('set LYA2PCF_REFERENCE to the lya2pcf reference tree')
HERE = os.path.dirname(os.path.abspath(__file__))


def reference_fill_dw():
    path = os.path.join(REF, 'forest_class.py')
    tree = ast.parse(open(path).read())
    cls = next(n for n in tree.body if isinstance(n, ast.ClassDef) and n.name == 'quasar')
    fn = next(n for n in cls.body if isinstance(n, ast.FunctionDef) and n.name == 'fill_dw')
    ns = {'np': np}
    exec(compile(ast.Module(body=[fn], type_ignores=[]), path, 'exec'), ns)
    return ns['fill_dw']


def main():
    fill_dw = reference_fill_dw()
    rng = np.random.default_rng(11)
    lengths = np.array([1, 2, 3, 17, 150, 400, 614, 75, 300, 5])
    start = np.zeros(len(lengths) + 1, dtype=np.int64)
    np.cumsum(lengths, out=start[1:])
    n = start[-1]
    we = np.empty(n); de = np.empty(n); loglam = np.empty(n)
    dw_p = np.empty(n); dl_p = np.empty(n); dw_np = np.empty(n)
    omega = np.empty(len(lengths)); odl2 = np.empty(len(lengths))
    for f, L in enumerate(lengths):
        a, b = start[f], start[f + 1]
        k0 = int(rng.integers(0, 600))
        loglam[a:b] = 3.5563 + 3e-4 * (k0 + np.arange(L))
        we[a:b] = rng.uniform(0.2, 5.0, L)
        de[a:b] = rng.normal(0, 0.25, L)
        q = types.SimpleNamespace(we=we[a:b].copy())
        with np.errstate(all='ignore'):
            fill_dw(q, de[a:b], loglam[a:b], True)
        dw_p[a:b] = q.dw
        dl_p[a:b] = q.delta_lambda
        omega[f] = q.omega
        odl2[f] = q.omega_delta_lambda2
        q2 = types.SimpleNamespace(we=we[a:b].copy())
        fill_dw(q2, de[a:b], loglam[a:b], False)
        dw_np[a:b] = q2.dw
    np.savez(os.path.join(HERE, 'fill_dw_golden.npz'), start=start, we=we, delta=de, loglam=loglam, dw=dw_p,
             delta_lambda=dl_p, omega=omega, odl2=odl2, dw_noproject=dw_np)
    print('wrote', os.path.join(HERE, 'fill_dw_golden.npz'), int(n), 'pixels')


if __name__ == '__main__':
    main()
