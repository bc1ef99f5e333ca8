"""Seeded synthetic forest catalogues with the shapes of the benchmark configurations.

No public data set is used: the workloads are defined synthetically.  Every
catalogue is a deterministic function of (config, scale, seed).

Common to all configurations:

* spectral grid: log10(lambda) = log10(3600) + 3e-4 * k, k = 0..613 (the last
  pixel is 5498.9 A < 5500 A), z = lambda / 1215.67 - 1;
* d_c(z) from flat LambdaCDM with Om = 0.3153 (the reference's
  ``parameters.py:44``; h cancels in Mpc/h);
* delta ~ Normal(mean 0, standard deviation 0.25) per pixel;
* w = ((1+z)/3.25)^1.9 / (0.1 + U[0.01, 0.5]), U drawn per pixel;
* dw from the reference projection ``fill_dw(project=True)``
  (``forest_class.py:48-68``): weighted mean and weighted log-lambda slope removed;
* quasar names unique except for a 0.5% set of "re-observations" that copy an
  existing quasar's name and sit 1 arcsec from it (exercises the same-quasar
  exclusion);
* healpix RING pixel with the configured nside (16 for the benchmark configs).

Configurations (sky patch, forest lengths):

0. 2,000 forests uniform on 100 deg^2 (RA 150-160 deg, Dec -5..5 deg),
   length U[150, 600], window start uniform on the grid.
1. 150,000 forests uniform on 8,000 deg^2 (RA 100-220 deg, sin(Dec) uniform
   from Dec -20 deg to 55.25 deg).  Length U[50, 700] clamped to the 614-pixel
   grid; the red end sits at the quasar's Lyman-alpha line, z_q ~ U[2.1, 3.5],
   shifted blueward only as far as the length requires.
2. Same catalogue as 1 (the guard-band precision form).
3. 30,000 forests on 1,500 deg^2 (RA 20-70 deg, Dec 0-31.6 deg) drawn from a
   log-normal density field exp(G - 1/2), G a unit-variance Gaussian field with a
   2-degree Gaussian correlation length (flat-sky FFT on a 0.25-degree grid);
   lengths as configuration 1.
4. 500 forests uniform on 10 deg^2 (RA 150-153.162 deg, Dec -1.58..1.58 deg),
   length U[100, 300].

``scale`` < 1 keeps the sky density and shrinks the forest count and the patch
area together (the shape of a full-size run at a size the CPU oracle finishes).
"""
import numpy as np

from . import parameters as P
from .cosmology import default as _cosmo
from .forests import ForestSet
from .healpix import radec_to_pix

NGRID = 614
LOGLAM0 = np.log10(3600.0)
DLOGLAM = 3e-4
SIGMA_DELTA = 0.25

_DEG = np.pi / 180.0

CONFIGS = {
    0: dict(n=2000, ra=(150.0, 160.0), dec=(-5.0, 5.0), length=(150, 600), window='uniform', field=False),
    1: dict(n=150000, ra=(100.0, 220.0), dec=(-20.0, 55.25), length=(50, 700), window='zq', field=False),
    2: dict(n=150000, ra=(100.0, 220.0), dec=(-20.0, 55.25), length=(50, 700), window='zq', field=False),
    3: dict(n=30000, ra=(20.0, 70.0), dec=(0.0, 31.6), length=(50, 700), window='zq', field=True),
    4: dict(n=500, ra=(150.0, 153.162), dec=(-1.58, 1.58), length=(100, 300), window='uniform', field=False),
}
SEEDS = {0: 20240, 1: 20241, 2: 20241, 3: 20243, 4: 20244}


def _patch(cfg, scale):
    """Shrink the RA range by ``scale`` (area scales linearly, density kept)."""
    ra0, ra1 = cfg['ra']
    return (ra0, ra0 + (ra1 - ra0) * scale), cfg['dec']


def _uniform_positions(rng, n, ra_rng, dec_rng):
    ra = rng.uniform(ra_rng[0], ra_rng[1], n) * _DEG
    s0, s1 = np.sin(dec_rng[0] * _DEG), np.sin(dec_rng[1] * _DEG)
    dec = np.arcsin(rng.uniform(s0, s1, n))
    return ra, dec


def _lognormal_positions(rng, n, ra_rng, dec_rng, corr_deg=2.0, sigma_ln=1.0, cell_deg=0.25):
    dec_mid = 0.5 * (dec_rng[0] + dec_rng[1])
    width = (ra_rng[1] - ra_rng[0]) * np.cos(dec_mid * _DEG)       # flat-sky extent, deg
    height = dec_rng[1] - dec_rng[0]
    pad = 4.0 * corr_deg
    nx = int(np.ceil((width + 2 * pad) / cell_deg))
    ny = int(np.ceil((height + 2 * pad) / cell_deg))
    white = rng.standard_normal((ny, nx))
    kx = np.fft.fftfreq(nx, d=cell_deg) * 2 * np.pi
    ky = np.fft.fftfreq(ny, d=cell_deg) * 2 * np.pi
    k2 = ky[:, None] ** 2 + kx[None, :] ** 2
    g = np.real(np.fft.ifft2(np.fft.fft2(white) * np.exp(-0.25 * k2 * corr_deg ** 2)))
    ipad = int(round(pad / cell_deg))
    mx = int(np.ceil(width / cell_deg)); my = int(np.ceil(height / cell_deg))
    g = g[ipad:ipad + my, ipad:ipad + mx]
    g = (g - g.mean()) / g.std()
    rho = np.exp(sigma_ln * g - 0.5 * sigma_ln ** 2)
    # cells of equal flat-sky area; multinomial draw then uniform inside the cell
    p = (rho / rho.sum()).ravel()
    cell = rng.choice(p.size, size=n, p=p)
    cy, cx = np.divmod(cell, mx)
    fx = (cx + rng.uniform(0, 1, n)) * cell_deg / width
    fy = (cy + rng.uniform(0, 1, n)) * cell_deg / height
    fx = np.clip(fx, 0.0, 1.0); fy = np.clip(fy, 0.0, 1.0)
    ra = (ra_rng[0] + fx * (ra_rng[1] - ra_rng[0])) * _DEG
    s0, s1 = np.sin(dec_rng[0] * _DEG), np.sin(dec_rng[1] * _DEG)
    dec = np.arcsin(s0 + fy * (s1 - s0))
    return ra, dec


def _windows(rng, n, cfg, length=None):
    lo, hi = cfg['length'] if length is None else length
    length = rng.integers(lo, hi + 1, n)
    length = np.minimum(length, NGRID)
    if cfg['window'] == 'uniform':
        start = (rng.uniform(0, 1, n) * (NGRID - length + 1)).astype(np.int64)
    else:
        zq = rng.uniform(2.1, 3.5, n)
        lam_end = P.lambdaa * (1.0 + zq)
        idx_end = np.floor(np.log10(lam_end / 3600.0) / DLOGLAM).astype(np.int64)
        idx_end = np.clip(idx_end, length - 1, NGRID - 1)
        start = idx_end - length + 1
    return start.astype(np.int64), length.astype(np.int64)


def _project(w, delta, loglam):
    """Weighted mean-and-slope removal of ``forest_class.fill_dw(project=True)``."""
    sw = w.sum()
    mean_delta = (delta * w).sum() / sw
    lam_avg = (loglam * w).sum() / sw
    dl = loglam - lam_avg
    odl2 = (dl * dl * w).sum()
    slope_num = (dl * delta * w).sum() / sw
    slope_den = (dl * dl * w).sum() / sw
    dw = w * (delta - mean_delta - dl * slope_num / slope_den)
    return dw, dl, sw, odl2


def make(config, scale=1.0, seed=None, nside=16, n=None, length=None):
    """Build the synthetic catalogue of benchmark configuration ``config``;
    ``length=(lo, hi)`` replaces the configuration's forest-length range."""
    cfg = CONFIGS[int(config)]
    rng = np.random.default_rng(SEEDS[int(config)] if seed is None else seed)
    n_forest = int(n) if n is not None else max(2, int(round(cfg['n'] * scale)))
    area_scale = n_forest / cfg['n']
    ra_rng, dec_rng = _patch(cfg, area_scale)
    if cfg['field']:
        ra, dec = _lognormal_positions(rng, n_forest, ra_rng, dec_rng)
    else:
        ra, dec = _uniform_positions(rng, n_forest, ra_rng, dec_rng)
    name = np.arange(n_forest, dtype=np.int64) + 10_000_000
    # re-observations: same quasar name, 1 arcsec away
    n_twin = n_forest // 200
    if n_twin:
        src = rng.choice(n_forest - n_twin, size=n_twin, replace=False)
        dst = np.arange(n_forest - n_twin, n_forest)
        off = (1.0 / 3600.0) * _DEG
        ra[dst] = ra[src] + off
        dec[dst] = dec[src]
        name[dst] = name[src]
    start_idx, length = _windows(rng, n_forest, cfg, length)

    grid_loglam = LOGLAM0 + DLOGLAM * np.arange(NGRID)
    grid_z = 10.0 ** grid_loglam / P.lambdaa - 1.0
    grid_dc = _cosmo().dc(grid_z)

    starts = np.zeros(n_forest + 1, dtype=np.int64)
    np.cumsum(length, out=starts[1:])
    tot = int(starts[-1])
    dc = np.empty(tot); w = np.empty(tot); dw = np.empty(tot); z = np.empty(tot); dl = np.empty(tot)
    omega = np.empty(n_forest); odl2 = np.empty(n_forest)
    delta_all = rng.normal(0.0, SIGMA_DELTA, tot)
    u_all = rng.uniform(0.01, 0.5, tot)
    for f in range(n_forest):
        a, b = starts[f], starts[f + 1]
        k = np.arange(start_idx[f], start_idx[f] + length[f])
        zz = grid_z[k]
        ww = ((1.0 + zz) / (1.0 + P.z_ref)) ** P.gammaovertwo / (0.1 + u_all[a:b])
        dww, dll, om, o2 = _project(ww, delta_all[a:b], grid_loglam[k])
        dc[a:b] = grid_dc[k]; w[a:b] = ww; dw[a:b] = dww; z[a:b] = zz; dl[a:b] = dll
        omega[f] = om; odl2[f] = o2
    ux = np.cos(ra) * np.cos(dec)
    uy = np.sin(ra) * np.cos(dec)
    uz = np.sin(dec)
    pix = radec_to_pix(nside, ra, dec)
    # forest order: grouped by healpix pixel (ascending), as a pixel dict would list them
    order = np.lexsort((np.arange(n_forest), pix))
    fs = ForestSet(start=starts, dc=dc, w=w, dw=dw, z=z, dl=dl, ra=ra, dec=dec, ux=ux, uy=uy, uz=uz,
                   name=name, pix=pix, omega=omega, odl2=odl2,
                   meta=dict(config=int(config), scale=float(scale), nside=int(nside),
                             seed=int(SEEDS[int(config)] if seed is None else seed)))
    fs = fs.subset(order)
    fs.meta.update(dict(config=int(config), scale=float(scale), nside=int(nside)))
    return fs


def angmax_for(fs, rtmax=P.rtmax):
    """Largest pair angle that can reach ``rtmax``: ``2 asin(rtmax / (2 dmin))`` with
    dmin the smallest first-pixel distance (``2pla.py:64-73``)."""
    first = fs.dc[fs.start[:-1][fs.lengths > 0]]
    dmin = float(np.min(first))
    return 2.0 * np.arcsin(0.5 * rtmax / dmin)
