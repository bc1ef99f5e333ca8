"""Golden vectors of the reference's covariance post-processing.

Run where the lya2pcf reference tree is available, named by the required
LYA2PCF_REFERENCE environment variable.  ``post_processing.py`` imports fitsio at module level,
which is not installed here, so the script compiles only the definitions of
``bin_coordinates``, ``cov`` (numba), ``cov_smooth`` and ``diag_error``
(post_processing.py:13-109) taken verbatim from that file's syntax tree, runs
them on seeded inputs and writes the inputs and outputs to
``tests/golden/cov_golden.npz``:

* case a: 40 owner pixels x (5 x 5) bins, random xi and weights;
* case b: 12 owner pixels x (4 x 4) bins, one bin with xi = 0 in every
  pixel (variance 0): cov_smooth returns the unsmoothed matrix;
* case c: 30 owner pixels x (6 x 6) bins for diag_error;
* case d: a bin whose weights are all 0: the reference's cov raises
  ZeroDivisionError (numba, Python error model); recorded as d_raises.
"""
import ast
import os
import sys

import numpy as np

REF = os.environ.get('LYA2PCF_REFERENCE', '')
if __name__ == '__main__' and not REF:
    raise SystemExit('set LYA2PCF_REFERENCE to the lya2pcf reference tree')
HERE = os.path.dirname(os.path.abspath(__file__))


def reference_functions():
    src = open(os.path.join(REF, 'post_processing.py')).read()
    tree = ast.parse(src)
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef)
            and n.name in ('bin_coordinates', 'cov', 'cov_smooth', 'diag_error')]
    mod = ast.Module(body=keep, type_ignores=[])
    from numba.core.decorators import jit
    ns = {'np': np, 'jit': jit}
    exec(compile(mod, os.path.join(REF, 'post_processing.py'), 'exec'), ns)
    return ns


def main():
    f = reference_functions()
    rng = np.random.default_rng(7)
    out = {}
    # case a
    n, np_, nt = 40, 5, 5
    xi = rng.normal(0, 1, (n, np_ * nt))
    we = rng.uniform(0.5, 2.0, (n, np_ * nt))
    c, m = f['cov'](xi, we)
    rp, rt = f['bin_coordinates'](np_, nt)
    cs = f['cov_smooth'](xi, we, rp, rt, c)
    out.update(a_xi=xi, a_we=we, a_cov=c, a_mean=m, a_rp=rp, a_rt=rt, a_cov_smooth=cs)
    # case b: an empty bin
    n, np_, nt = 12, 4, 4
    xi = rng.normal(0, 1, (n, np_ * nt))
    we = rng.uniform(0.5, 2.0, (n, np_ * nt))
    xi[:, 5] = 0.0
    c, m = f['cov'](xi, we)
    rp, rt = f['bin_coordinates'](np_, nt)
    cs = f['cov_smooth'](xi, we, rp, rt, c)
    out.update(b_xi=xi, b_we=we, b_cov=c, b_mean=m, b_cov_smooth=cs)
    # case c: diagonal errors
    n, np_, nt = 30, 6, 6
    xi = rng.normal(0, 1, (n, np_ * nt))
    we = rng.uniform(0.5, 2.0, (n, np_ * nt))
    err, mda = f['diag_error'](xi, we)
    out.update(c_xi=xi, c_we=we, c_error=err, c_mean=mda)
    # case d: a zero-weight bin
    xi = rng.normal(0, 1, (8, 9))
    we = rng.uniform(0.5, 2.0, (8, 9))
    we[:, 4] = 0.0
    try:
        f['cov'](xi, we)
        raises = False
    except ZeroDivisionError:
        raises = True
    out.update(d_xi=xi, d_we=we, d_raises=np.array(raises))
    np.savez(os.path.join(HERE, 'cov_golden.npz'), **out)
    print('wrote', os.path.join(HERE, 'cov_golden.npz'), {k: v.shape for k, v in out.items()})


if __name__ == '__main__':
    sys.exit(main())
