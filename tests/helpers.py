"""Shared test helpers: build small ForestSets from explicit arrays."""
import numpy as np

from lya2pcf_b200.forests import ForestSet


def forestset(forests, names=None, pix=None):
    """``forests``: list of dicts with ra, dec (radians), dc, w, dw and optional z, dl."""
    n = len(forests)
    lens = np.array([len(f['dc']) for f in forests], dtype=np.int64)
    start = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=start[1:])
    cat = lambda k, default=None: np.concatenate(  # noqa: E731
        [np.asarray(f[k] if k in f else default(f), dtype=np.float64) for f in forests]) if n else np.zeros(0)
    ra = np.array([f['ra'] for f in forests], dtype=np.float64)
    dec = np.array([f['dec'] for f in forests], dtype=np.float64)
    ux = np.cos(ra) * np.cos(dec)
    uy = np.sin(ra) * np.cos(dec)
    uz = np.sin(dec)
    for f in forests:
        if 'ux' in f:
            pass
    ux = np.array([f.get('ux', u) for f, u in zip(forests, ux)], dtype=np.float64)
    uy = np.array([f.get('uy', u) for f, u in zip(forests, uy)], dtype=np.float64)
    uz = np.array([f.get('uz', u) for f, u in zip(forests, uz)], dtype=np.float64)
    w = cat('w')
    dl = cat('dl', lambda f: np.linspace(-0.05, 0.05, len(f['dc'])))
    om = np.array([np.sum(f['w']) for f in forests], dtype=np.float64)
    odl2 = np.array([np.sum(np.asarray(f['w']) * np.asarray(f.get('dl', np.linspace(-0.05, 0.05, len(f['dc'])))) ** 2)
                     for f in forests], dtype=np.float64)
    return ForestSet(start=start, dc=cat('dc'), w=w, dw=cat('dw'), z=cat('z', lambda f: np.full(len(f['dc']), 2.5)),
                     dl=dl, ra=ra, dec=dec, ux=ux, uy=uy, uz=uz,
                     name=np.asarray(names if names is not None else np.arange(n), dtype=np.int64),
                     pix=np.asarray(pix if pix is not None else np.zeros(n), dtype=np.int64), omega=om, odl2=odl2)
