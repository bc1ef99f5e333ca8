"""Neighbour enumeration: the oracle and the drop-in quasar.neighborhood follow
forest_class.py:78-98 (mu > cos(angmax), different name, ra < ra2)."""
import numpy as np

import edge_cases as E
from lya2pcf_b200 import synthetic
from oracle import oracle as O


def _brute(fs, angmax):
    mumin = np.cos(angmax)
    key = O.reference_order_key(fs)
    out = []
    for f in range(fs.n):
        mu = (fs.ux[f] * fs.ux + fs.uy[f] * fs.uy) + fs.uz[f] * fs.uz
        m = (mu > mumin) & (fs.name != fs.name[f]) & (fs.ra[f] < fs.ra)
        idx = np.nonzero(m)[0]
        out.append(idx[np.argsort(key[idx], kind='stable')])
    return out


def test_oracle_neighbours_match_bruteforce():
    for fs in (synthetic.make(0).subset(np.arange(0, 2000, 3)), E.edge_catalog()):
        am = synthetic.angmax_for(fs) if fs.n > 100 else 0.05
        off, nbr = O.neighbours(fs, am)
        ref = _brute(fs, am)
        for f in range(fs.n):
            assert np.array_equal(nbr[off[f]:off[f + 1]], ref[f]), f


def test_edge_catalog_exclusions():
    fs = E.edge_catalog()
    off, nbr = O.neighbours(fs, 0.05)
    pairs = {(int(a), int(b)) for a in range(fs.n) for b in nbr[off[a]:off[a + 1]]}
    names = fs.name
    # same name never pairs, equal ra never pairs
    for a, b in pairs:
        assert names[a] != names[b]
        assert fs.ra[a] < fs.ra[b]
    # the ra = 0 / 2 pi neighbours pair (the one at ra ~ 2 pi is the second forest)
    i600, i601 = int(np.nonzero(names == 600)[0][0]), int(np.nonzero(names == 601)[0][0])
    assert (i601, i600) in pairs


def test_dropin_neighborhood_same_as_oracle():
    fs = synthetic.make(4, n=120)
    am = synthetic.angmax_for(fs)
    data = fs.to_quasar_dict()
    flat = [q for p in data for q in data[p]]
    index = {id(q): k for k, q in enumerate(flat)}
    off, nbr = O.neighbours(fs, am)
    for k, q in enumerate(flat):
        got = [index[id(o)] for o in q.neighborhood(data, am)]
        assert got == nbr[off[k]:off[k + 1]].tolist(), k


def _golden_neighbours():
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'neighbour_golden.npz'))
    return [(synthetic.make(0, n=400), 'cat0', g), (E.edge_catalog(), 'edge', g)]


def test_oracle_neighbours_equal_reference_neighborhood():
    """The oracle's neighbour lists equal the reference's own
    quasar.neighborhood (forest_class.py:78-98, run under a healpy stand-in
    whose query_disc returns every pixel: tests/golden/make_neighbour_golden.py),
    forest by forest, in the same order."""
    for fs, tag, g in _golden_neighbours():
        assert int(g[f'{tag}_n']) == fs.n
        off, nbr = O.neighbours(fs, float(g[f'{tag}_angmax']))
        assert np.array_equal(off, g[f'{tag}_off']), tag
        assert np.array_equal(nbr, g[f'{tag}_nbr']), tag
