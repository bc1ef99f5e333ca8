"""Forest data model, importable as the top-level module ``forest_class``.

The reference's ``data#.npy`` files are pickles of ``dict[healpix pixel ->
list[forest_class.quasar]]`` (``delta_reader.py:139-144``), so this module keeps
the module name ``forest_class`` and the class name ``quasar`` with the same
attributes (``forest_class.py:9-46``).  Differences from the reference:

* no healpy: the pixel index comes from :mod:`lya2pcf_b200.healpix`;
* :meth:`quasar.neighborhood` scans the pixels present in ``data`` in ascending
  order (a superset of the reference's ``query_disc`` pre-filter) and applies the
  reference's own membership test, so it returns the same forests in the same
  order.  The GPU backends never call it per forest: they build the neighbour
  lists on the device in one pass.
"""
import os
import sys

import numpy as np

_here = os.path.dirname(os.path.abspath(__file__))
_root = os.path.dirname(os.path.dirname(_here))
if _root not in sys.path:
    sys.path.insert(0, _root)

from lya2pcf_b200 import parameters as _P          # noqa: E402
from lya2pcf_b200.healpix import ang2pix_ring       # noqa: E402


class quasar(object):
    """One Lyman-alpha forest: per-pixel arrays and the quasar's sky position."""

    def __init__(self, fib, pl, name, ra, dec, lenght):
        self.ra = ra
        self.fib = fib
        self.pl = pl
        self.name = name
        self.dec = dec
        self.lenght = lenght
        self.pix = int(ang2pix_ring(_P.nside, _P.halfpi - dec, ra))

        self.dw = np.zeros(lenght, dtype=np.float64)
        self.we = np.zeros(lenght, dtype=np.float64)
        self.dc = np.zeros(lenght, dtype=np.float64)

        # unit vector of the line of sight
        self.x = np.cos(ra) * np.cos(dec)
        self.y = np.sin(ra) * np.cos(dec)
        self.z = np.sin(dec)

        self.rx = np.zeros(lenght, dtype=np.float64)
        self.ry = np.zeros(lenght, dtype=np.float64)
        self.rz = np.zeros(lenght, dtype=np.float64)

        self.lambda_average = 0
        self.delta_lambda = np.zeros(lenght, dtype=np.float64)
        self.omega_delta_lambda2 = 0
        self.omega = 0

    def fill_dw(self, de, loglam, project):
        """Set ``dw = w * delta``, after removing the weighted mean and the weighted
        linear trend in log-lambda when ``project`` is true (the projection of
        ``forest_class.py:48-68``).  Also stores the moments the distortion uses."""
        we = np.asarray(self.we, dtype=np.float64)
        de = np.asarray(de, dtype=np.float64)
        if not project:
            self.dw = de * we
            return
        sw = we.sum()
        mean_delta = (de * we).sum() / sw
        self.lambda_average = (np.asarray(loglam, dtype=np.float64) * we).sum() / sw
        self.delta_lambda = loglam - self.lambda_average
        dl = self.delta_lambda
        self.omega_delta_lambda2 = np.sum(dl * dl * we)
        slope_num = (dl * de * we).sum() / sw
        slope_den = (dl * dl * we).sum() / sw
        self.dw = we * (de - mean_delta - dl * slope_num / slope_den)
        self.omega = sw

    def dot_product(self, other):
        """cos of the angle between two lines of sight, in the reference's order of
        operations (``forest_class.py:70-76``)."""
        return self.x * other.x + self.y * other.y + self.z * other.z

    def neighborhood(self, data, angmax):
        """Forests of ``data`` within ``angmax`` of this one, each unordered pair
        once (``ra < ra2``), same quasar excluded (``forest_class.py:78-98``)."""
        mumin = np.cos(angmax)
        neighs = []
        for pix2 in sorted(data.keys()):
            for forest2 in data[pix2]:
                mu = self.dot_product(forest2)
                if mu > mumin and self.name != forest2.name and self.ra < forest2.ra:
                    neighs.append(forest2)
        return neighs

    def neighborhood_names(self, data, angmax):
        """Names and pixels of :meth:`neighborhood`'s forests (``forest_class.py:100-122``)."""
        neighs = self.neighborhood(data, angmax)
        return [[f.name for f in neighs], [f.pix for f in neighs]]
