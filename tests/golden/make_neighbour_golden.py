"""Golden neighbour lists of the reference's own quasar.neighborhood
(forest_class.py:78-98).

Run where the lya2pcf reference tree is available, named by the required
LYA2PCF_REFERENCE environment variable.  healpy is not installed here, so the
script puts a stand-in ``healpy`` module in ``sys.modules`` before importing
the reference's ``forest_class``: its ``query_disc`` returns every healpix
pixel in ascending order, a superset of the disc, which the reference's own
loop then filters with its exact test (mu > cos(angmax), different name,
ra < ra2).  The neighbour *set* is therefore the reference's; the order is
that of ascending pixels, then list position, which is the order healpy's
sorted pixel list gives.  The forests are built without ``quasar.__init__``
(which calls ``healpy.ang2pix``) and given the attributes ``neighborhood``
reads.  Writes ``tests/golden/neighbour_golden.npz``: two catalogues (a seeded
400-forest patch with same-name twins, and the hand-built edge catalogue of
``tests/edge_cases.py`` with equal ra, coincident lines of sight and pairs
across ra = 0 / 2 pi), each with its angmax and the CSR neighbour lists.

    LYA2PCF_REFERENCE=<reference tree> python tests/golden/make_neighbour_golden.py
"""
import os
import sys
import types

import numpy as np

REF = os.environ.get('LYA2PCF_REFERENCE', '')
if __name__ == '__main__' and not REF:
    raise SystemExit('set LYA2PCF_REFERENCE to the lya2pcf reference tree')
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def reference_forest_class():
    stub = types.ModuleType('healpy')
    stub.query_disc = lambda nside, vec, radius, inclusive=False: np.arange(12 * 64 * 64)
    stub.ang2pix = lambda nside, theta, phi: 0
    sys.modules['healpy'] = stub
    sys.path.insert(0, REF)
    import forest_class   # the reference module, read-only
    assert os.path.dirname(os.path.abspath(forest_class.__file__)) == os.path.abspath(REF)
    return forest_class


def reference_lists(fc, fs, angmax):
    data = {}
    objs = []
    for f in range(fs.n):
        q = fc.quasar.__new__(fc.quasar)
        q.ra = float(fs.ra[f]); q.dec = float(fs.dec[f]); q.name = int(fs.name[f])
        q.x = float(fs.ux[f]); q.y = float(fs.uy[f]); q.z = float(fs.uz[f])
        q.pix = int(fs.pix[f])
        q.index = f
        data.setdefault(q.pix, []).append(q)
        objs.append(q)
    data = {p: data[p] for p in sorted(data)}
    off = [0]
    nbr = []
    for q in objs:
        nbr += [o.index for o in q.neighborhood(data, angmax)]
        off.append(len(nbr))
    return np.array(off, dtype=np.int64), np.array(nbr, dtype=np.int32)


def main():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, 'tests'))
    from lya2pcf_b200 import synthetic
    import edge_cases as E
    fc = reference_forest_class()
    payload = {}
    for tag, fs, am in (('cat0', synthetic.make(0, n=400), None), ('edge', E.edge_catalog(), 0.05)):
        am = synthetic.angmax_for(fs) if am is None else am
        order = np.lexsort((np.arange(fs.n), fs.pix))   # forests grouped by ascending pixel
        assert np.array_equal(order, np.arange(fs.n))
        off, nbr = reference_lists(fc, fs, am)
        payload[f'{tag}_angmax'] = am
        payload[f'{tag}_off'] = off
        payload[f'{tag}_nbr'] = nbr
        payload[f'{tag}_n'] = fs.n
        print(tag, fs.n, 'forests', len(nbr), 'neighbour pairs')
    np.savez_compressed(os.path.join(HERE, 'neighbour_golden.npz'), **payload)


if __name__ == '__main__':
    main()
