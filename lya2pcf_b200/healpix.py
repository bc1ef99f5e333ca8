"""HEALPix RING-scheme pixel index, restated from the published algorithm.

The reference calls ``healpy.ang2pix(nside, theta, phi)`` (``forest_class.py:22-25``)
and ``healpy.query_disc(..., inclusive=True)`` (``forest_class.py:89``).  healpy
(unpinned in the reference's ``requirements.txt``) is not available here, so the
pixel index is computed from the HEALPix definition of Gorski et al. 2005
(ApJ 622, 759), section 4, as implemented by the HEALPix library's
``loc2pix`` for the RING scheme: equatorial belt ``|cos(theta)| <= 2/3`` indexed by
the two families of edge lines, polar caps by the distance to the pole, with the
``sin(theta)`` form of the polar distance near the poles.

``query_disc`` only pre-filters candidate pixels in the reference; the final
neighbour set is decided by the ``mu > cos(angmax)`` test, so any superset of the
disc's pixels yields the same set.  The neighbour *order* of the reference is the
ascending order of the pixel indices that ``query_disc`` returns (a sorted range
set), then list order within each pixel; :func:`neighbour_order_key` reproduces it.
"""
import numpy as np

_HALFPI = 0.5 * np.pi
_INV_HALFPI = 2.0 / np.pi


def ang2pix_ring(nside, theta, phi):
    """RING-scheme pixel of colatitude ``theta`` and longitude ``phi`` (radians).

    Works elementwise on numpy arrays; returns int64.
    """
    theta = np.asarray(theta, dtype=np.float64)
    phi = np.asarray(phi, dtype=np.float64)
    scalar = theta.ndim == 0 and phi.ndim == 0
    theta, phi = np.broadcast_arrays(np.atleast_1d(theta), np.atleast_1d(phi))
    ns = int(nside)
    npix = 12 * ns * ns
    ncap = 2 * ns * (ns - 1)

    z = np.cos(theta)
    za = np.abs(z)
    tt = np.mod(phi * _INV_HALFPI, 4.0)          # in [0, 4)
    out = np.empty(theta.shape, dtype=np.int64)

    eq = za <= 2.0 / 3.0
    if np.any(eq):
        zz = z[eq]
        t = tt[eq]
        temp1 = ns * (0.5 + t)
        temp2 = ns * (zz * 0.75)
        jp = (temp1 - temp2).astype(np.int64)     # ascending edge line index
        jm = (temp1 + temp2).astype(np.int64)     # descending edge line index
        ir = ns + 1 + jp - jm                     # ring index within the belt, 1..2ns+1
        kshift = 1 - (ir & 1)
        ip = (jp + jm - ns + kshift + 1) // 2
        ip = np.mod(ip, 4 * ns)
        out[eq] = ncap + (ir - 1) * 4 * ns + ip

    pol = ~eq
    if np.any(pol):
        zz = z[pol]
        zap = za[pol]
        t = tt[pol]
        th = theta[pol]
        tp = t - np.floor(t)
        near_pole = (th < 0.01) | (th > np.pi - 0.01)
        tmp = np.where(near_pole,
                       ns * np.sin(th) / np.sqrt((1.0 + zap) / 3.0),
                       ns * np.sqrt(3.0 * (1.0 - zap)))
        jp = (tp * tmp).astype(np.int64)
        jm = ((1.0 - tp) * tmp).astype(np.int64)
        ir = jp + jm + 1                          # ring index counted from the nearer pole
        ip = (t * ir).astype(np.int64)
        ip = np.mod(ip, 4 * ir)
        out[pol] = np.where(zz > 0, 2 * ir * (ir - 1) + ip, npix - 2 * ir * (ir + 1) + ip)

    return int(out[0]) if scalar else out


def radec_to_pix(nside, ra, dec):
    """Pixel of a sky position as the reference computes it: theta = pi/2 - dec, phi = ra."""
    return ang2pix_ring(nside, _HALFPI - np.asarray(dec, dtype=np.float64), ra)


def neighbour_order_key(pix, local_index):
    """Sort key that orders candidate neighbours the way the reference visits them:
    ascending healpix pixel, then position inside that pixel's forest list."""
    pix = np.asarray(pix, dtype=np.int64)
    local_index = np.asarray(local_index, dtype=np.int64)
    return pix * (1 << 32) + local_index
