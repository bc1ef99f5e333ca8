"""Flat (CSR) forest catalogue: the host-side layout everything else consumes.

The reference keeps forests as Python ``quasar`` objects grouped by healpix pixel
(``forest_class.py:9-46``) and, at ``init``, packs them into padded
``[n_forest x max_lenght]`` arrays (``correlation_procedures_pycuda.py:56-87``).
This module packs the same per-pixel data unpadded: forest ``f`` owns pixels
``start[f]:start[f+1]`` of the flat arrays.  Forest order is the reference's
``forest.index`` order: the iteration order of the pixel dict, then list order.
"""
from dataclasses import dataclass, field

import numpy as np

from . import parameters as P


@dataclass
class ForestSet:
    start: np.ndarray          # int64 [n+1], CSR offsets into the pixel arrays
    dc: np.ndarray             # float64 [npix] comoving distance, Mpc/h
    w: np.ndarray              # float64 [npix] weight
    dw: np.ndarray             # float64 [npix] weight * projected delta
    z: np.ndarray              # float64 [npix] redshift of the absorber
    dl: np.ndarray             # float64 [npix] log10(lambda) - weighted mean (projection)
    ra: np.ndarray             # float64 [n] radians
    dec: np.ndarray            # float64 [n] radians
    ux: np.ndarray             # float64 [n] unit vector of the line of sight
    uy: np.ndarray
    uz: np.ndarray
    name: np.ndarray           # int64 [n] quasar identity (same name => same quasar)
    pix: np.ndarray            # int64 [n] healpix pixel (the owner pixel of f1 pairs)
    omega: np.ndarray          # float64 [n] sum of weights
    odl2: np.ndarray           # float64 [n] sum of w * dl^2
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return int(self.start.shape[0] - 1)

    @property
    def lengths(self):
        return np.diff(self.start).astype(np.int64)

    @property
    def npix_total(self):
        return int(self.start[-1])

    def forest(self, f):
        a, b = int(self.start[f]), int(self.start[f + 1])
        return dict(dc=self.dc[a:b], w=self.w[a:b], dw=self.dw[a:b], z=self.z[a:b], dl=self.dl[a:b])

    def subset(self, idx):
        """A new ForestSet holding forests ``idx`` (in that order)."""
        idx = np.asarray(idx, dtype=np.int64)
        lens = self.lengths[idx]
        start = np.zeros(len(idx) + 1, dtype=np.int64)
        np.cumsum(lens, out=start[1:])
        gather = np.concatenate([np.arange(self.start[f], self.start[f + 1]) for f in idx]) \
            if len(idx) else np.zeros(0, dtype=np.int64)
        take = lambda a: a[gather].copy()  # noqa: E731
        return ForestSet(start=start, dc=take(self.dc), w=take(self.w), dw=take(self.dw), z=take(self.z),
                         dl=take(self.dl), ra=self.ra[idx].copy(), dec=self.dec[idx].copy(),
                         ux=self.ux[idx].copy(), uy=self.uy[idx].copy(), uz=self.uz[idx].copy(),
                         name=self.name[idx].copy(), pix=self.pix[idx].copy(), omega=self.omega[idx].copy(),
                         odl2=self.odl2[idx].copy(), meta=dict(self.meta))

    def pixel_groups(self):
        """Dict healpix pixel -> forest indices, keyed in first-appearance order."""
        groups = {}
        for f, p in enumerate(self.pix.tolist()):
            groups.setdefault(p, []).append(f)
        return groups

    # ------------------------------------------------------------------ columnar cache
    _COLUMNS = ('start', 'dc', 'w', 'dw', 'z', 'dl', 'ra', 'dec', 'ux', 'uy', 'uz', 'name', 'pix', 'omega', 'odl2')

    def save(self, path):
        """Write the catalogue as one ``.npz`` of columns: a cache that later
        runs load in place of unpickling ``data#.npy`` quasar objects."""
        np.savez(path, **{k: getattr(self, k) for k in self._COLUMNS},
                 meta_keys=np.array(list(self.meta.keys()), dtype=object),
                 meta_values=np.array([str(v) for v in self.meta.values()], dtype=object))

    @classmethod
    def load(cls, path):
        """Read a catalogue written by :meth:`save`."""
        with np.load(path, allow_pickle=True) as z:
            cols = {k: z[k] for k in cls._COLUMNS}
            meta = dict(zip(z['meta_keys'].tolist(), z['meta_values'].tolist())) if 'meta_keys' in z else {}
        return cls(meta=meta, **cols)

    # ------------------------------------------------------------------ dict form
    def to_quasar_dict(self):
        """The reference's ``data`` object: dict pixel -> list of ``forest_class.quasar``."""
        from .dropin_path import quasar_class
        quasar = quasar_class()
        data = {}
        for f in range(self.n):
            a, b = int(self.start[f]), int(self.start[f + 1])
            q = quasar.__new__(quasar)
            q.ra = float(self.ra[f]); q.dec = float(self.dec[f])
            q.fib = int(self.name[f]); q.pl = 0; q.name = int(self.name[f])
            q.lenght = b - a
            q.pix = int(self.pix[f])
            q.we = self.w[a:b].copy(); q.dw = self.dw[a:b].copy(); q.dc = self.dc[a:b].copy()
            q.x = float(self.ux[f]); q.y = float(self.uy[f]); q.z = float(self.uz[f])
            q.rx = q.x * q.dc; q.ry = q.y * q.dc; q.rz = q.z * q.dc
            loglam = np.log10((1.0 + self.z[a:b]) * P.lambdaa)
            q.delta_lambda = self.dl[a:b].copy()
            q.lambda_average = float(np.mean(loglam - q.delta_lambda)) if b > a else 0.0
            q.omega_delta_lambda2 = float(self.odl2[f]); q.omega = float(self.omega[f])
            data.setdefault(q.pix, []).append(q)
        return data


def from_quasar_dict(data, pixel_list=None):
    """Pack ``data`` (dict pixel -> list of quasar) into a :class:`ForestSet`.

    Forest order is ``pixel_list`` order (default: dict order), then list order,
    the order in which the reference assigns ``forest.index``
    (``correlation_procedures_pycuda.py:73-87``).  Returns ``(ForestSet, forests)``
    where ``forests`` is the flat list of quasar objects in that order.
    """
    from .cosmology import default as cosmo
    if not pixel_list:
        pixel_list = list(data.keys())
    forests = [q for p in pixel_list for q in data[p]]
    n = len(forests)
    lens = np.array([len(q.dc) for q in forests], dtype=np.int64)
    start = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=start[1:])
    cat = lambda attr: (np.concatenate([np.asarray(getattr(q, attr), dtype=np.float64) for q in forests])  # noqa: E731
                        if n else np.zeros(0))
    dc, w, dw = cat('dc'), cat('we'), cat('dw')
    dl_parts, z_parts = [], []
    for q in forests:
        m = len(q.dc)
        dl = np.asarray(getattr(q, 'delta_lambda', np.zeros(m)), dtype=np.float64)
        if dl.shape[0] != m:
            dl = np.zeros(m)
        lam_avg = float(getattr(q, 'lambda_average', 0.0) or 0.0)
        if lam_avg != 0.0:
            z = 10.0 ** (dl + lam_avg) / P.lambdaa - 1.0
        else:
            z = cosmo().z_of_dc(np.asarray(q.dc, dtype=np.float64))
        dl_parts.append(dl)
        z_parts.append(np.asarray(z, dtype=np.float64))
    dl = np.concatenate(dl_parts) if n else np.zeros(0)
    z = np.concatenate(z_parts) if n else np.zeros(0)
    names = [q.name for q in forests]
    try:
        name_arr = np.asarray(names, dtype=np.int64)
    except (TypeError, ValueError, OverflowError):
        _, name_arr = np.unique(np.asarray([str(x) for x in names]), return_inverse=True)
        name_arr = name_arr.astype(np.int64)
    fs = ForestSet(
        start=start, dc=dc, w=w, dw=dw, z=z, dl=dl,
        ra=np.array([q.ra for q in forests], dtype=np.float64),
        dec=np.array([q.dec for q in forests], dtype=np.float64),
        ux=np.array([q.x for q in forests], dtype=np.float64),
        uy=np.array([q.y for q in forests], dtype=np.float64),
        uz=np.array([q.z for q in forests], dtype=np.float64),
        name=name_arr,
        pix=np.array([q.pix for q in forests], dtype=np.int64),
        omega=np.array([float(getattr(q, 'omega', 0.0) or 0.0) for q in forests], dtype=np.float64),
        odl2=np.array([float(getattr(q, 'omega_delta_lambda2', 0.0) or 0.0) for q in forests], dtype=np.float64),
    )
    return fs, forests
