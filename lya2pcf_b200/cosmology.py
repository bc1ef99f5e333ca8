"""Line-of-sight comoving distance d_c(z) in Mpc/h for flat LambdaCDM.

Same physics as lya2pcf ``cosmology.py:9-34`` (``d_c(z) = (c/100) * int_0^z dz'/E(z')``
with ``E(z) = sqrt(Om (1+z)^3 + 1 - Om)``, ``Om = 0.3153`` from ``parameters.py:44``),
computed here by composite Gauss-Legendre quadrature on a fine z table and a
cubic spline instead of ``scipy.integrate.quad`` per node.  Only the synthetic
generator and the z-recovery of the drop-in API use it; the pair path receives
d_c as input data.
"""
import numpy as np
from scipy.interpolate import CubicSpline

from . import parameters as P


def _inv_e(z, om):
    return 1.0 / np.sqrt(om * (1.0 + z) ** 3 + (1.0 - om))


def _table(om, zmax=10.0, n=20001):
    z = np.linspace(0.0, zmax, n)
    # 8-point Gauss-Legendre per interval: error far below 1e-12 relative.
    x, wq = np.polynomial.legendre.leggauss(8)
    a, b = z[:-1], z[1:]
    mid, half = 0.5 * (a + b), 0.5 * (b - a)
    nodes = mid[:, None] + half[:, None] * x[None, :]
    seg = (half[:, None] * wq[None, :] * _inv_e(nodes, om)).sum(axis=1)
    dc = np.concatenate([[0.0], np.cumsum(seg)]) * P.d_H0
    return z, dc


class Cosmology:
    """d_c(z) and its inverse for a flat LambdaCDM model."""

    def __init__(self, om=P.Omm):
        self.om = float(om)
        z, dc = _table(self.om)
        self._dc = CubicSpline(z, dc)
        self._z = CubicSpline(dc, z)

    def dc(self, z):
        return self._dc(np.asarray(z, dtype=np.float64))

    def z_of_dc(self, dc):
        return self._z(np.asarray(dc, dtype=np.float64))


_default = None


def default():
    global _default
    if _default is None:
        _default = Cosmology()
    return _default


def dc_interpol(z):
    """Comoving distance of redshift ``z`` (Mpc/h), the reference's entry-point name."""
    return default().dc(z)
