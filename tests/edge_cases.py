"""Adversarial and edge-case catalogues shared by the CPU and GPU tests."""
import numpy as np

from helpers import forestset


def _unit(ra, dec):
    return np.array([np.cos(ra) * np.cos(dec), np.sin(ra) * np.cos(dec), np.sin(dec)])


def cos_variant_cases(n_cases=192, seed=3):
    """1-pixel forest pairs whose rt lies within a few ulps of an rt bin edge,
    chosen so that the three FMA contractions of cos12 (see the oracle's
    orc_cos12) put the pair in different rt bins.  Returns (ForestSet, f1, f2,
    variant_bins[n_cases, 3]) with variant_bins the flat bin (or -1) of each
    contraction under the reference FP64 formula."""
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    forests, f1, f2, vb = [], [], [], []
    tries = 0
    while len(f1) < n_cases and tries < 200000:
        tries += 1
        ra1, dec1 = rng.uniform(0.5, 1.0), rng.uniform(-0.3, 0.3)
        sep, pa = rng.uniform(0.003, 0.05), rng.uniform(0, 2 * np.pi)
        ra2 = ra1 + abs(sep * np.sin(pa) / np.cos(dec1)) + 1e-9
        dec2 = dec1 + sep * np.cos(pa)
        u1, u2 = _unit(ra1, dec1), _unit(ra2, dec2)
        cs = [O.cos12(u1, u2, v) for v in range(3)]
        if len(set(cs)) == 1:
            continue
        shs = [np.sqrt(0.5 * (1.0 - c)) for c in cs]
        chs = [np.sqrt(0.5 * (1.0 + c)) for c in cs]
        k = int(rng.integers(5, 49))
        s = 4.0 * k / shs[0]
        found = None
        for d in range(0, 200):
            for sgn in (1, -1):
                t = s
                for _ in range(d):
                    t = np.nextafter(t, np.inf if sgn > 0 else -np.inf)
                dc1 = float(np.float64(t) / 2.0)
                dc2 = float(t - dc1)
                if dc1 + dc2 != t:
                    continue
                bins = []
                for ch, sh in zip(chs, shs):
                    rp = abs(dc1 - dc2) * ch
                    rt = (dc1 + dc2) * sh
                    bp, bt = np.floor(rp * 0.25), np.floor(rt * 0.25)
                    bins.append(int(bp) * 50 + int(bt) if (bp < 50 and bt < 50) else -1)
                if len(set(bins)) > 1:
                    found = (dc1, dc2, bins)
                    break
            if found:
                break
        if not found:
            continue
        dc1, dc2, bins = found
        i = len(forests)
        forests.append(dict(ra=ra1, dec=dec1, dc=[dc1], w=[1.0], dw=[1.0], z=[2.0], ux=u1[0], uy=u1[1], uz=u1[2]))
        forests.append(dict(ra=ra2, dec=dec2, dc=[dc2], w=[1.0], dw=[1.0], z=[2.0], ux=u2[0], uy=u2[1], uz=u2[2]))
        f1.append(i)
        f2.append(i + 1)
        vb.append(bins)
    n = len(forests)
    pix = np.repeat(np.arange(n // 2), 2)      # one owner slot per case
    fs = forestset(forests, names=np.arange(n), pix=pix)
    return fs, np.array(f1, dtype=np.int32), np.array(f2, dtype=np.int32), np.array(vb, dtype=np.int64)


def same_grid_forest(ra, dec, start, length, rng, name=None):
    """A forest on the synthetic log-lambda grid (sorted dc)."""
    from lya2pcf_b200 import synthetic as S
    from lya2pcf_b200.cosmology import dc_interpol
    k = start + np.arange(length)
    loglam = S.LOGLAM0 + S.DLOGLAM * k
    z = 10 ** loglam / 1215.67 - 1
    w = ((1 + z) / 3.25) ** 1.9 / (0.1 + rng.uniform(0.01, 0.5, length))
    delta = rng.normal(0, 0.25, length)
    return dict(ra=ra, dec=dec, dc=np.asarray(dc_interpol(z)), w=w, dw=w * delta, z=z)


def edge_catalog(seed=11):
    """Hand-built catalogue exercising the reference's edge cases:
    length-1 and empty forests, an unsorted forest, same-name twins, equal ra,
    coincident lines of sight with different names (rt = 0), pairs across
    ra = 0 / 2 pi, and exact bin edges in rp (|dc1-dc2| = 4k on one line of
    sight)."""
    rng = np.random.default_rng(seed)
    deg = np.pi / 180
    F = []
    names = []
    pix = []
    # pixel 0: ordinary forests around (ra, dec) = (30, 10) deg
    for q in range(6):
        F.append(same_grid_forest(30 * deg + rng.uniform(0, 1) * deg, 10 * deg + rng.uniform(0, 1) * deg,
                                  int(rng.integers(0, 300)), int(rng.integers(40, 200)), rng))
        names.append(100 + q); pix.append(0)
    # length-1 forest and an empty forest
    F.append(same_grid_forest(30.4 * deg, 10.4 * deg, 200, 1, rng)); names.append(200); pix.append(0)
    F.append(dict(ra=30.45 * deg, dec=10.45 * deg, dc=np.zeros(0), w=np.zeros(0), dw=np.zeros(0), z=np.zeros(0)))
    names.append(201); pix.append(0)
    # unsorted forest (dc reversed)
    g = same_grid_forest(30.5 * deg, 10.5 * deg, 100, 150, rng)
    F.append({k: (v[::-1].copy() if isinstance(v, np.ndarray) else v) for k, v in g.items()}); names.append(202); pix.append(0)
    # same-name twin 1 arcsec away: excluded from pairs
    g = same_grid_forest(30.6 * deg, 10.6 * deg, 50, 120, rng)
    F.append(g); names.append(300); pix.append(0)
    g2 = same_grid_forest(30.6 * deg + 1 / 3600 * deg, 10.6 * deg, 60, 120, rng)
    F.append(g2); names.append(300); pix.append(0)
    # equal ra: the ra < ra2 rule excludes the pair in both directions
    F.append(same_grid_forest(30.7 * deg, 10.2 * deg, 0, 100, rng)); names.append(400); pix.append(0)
    F.append(same_grid_forest(30.7 * deg, 10.3 * deg, 0, 100, rng)); names.append(401); pix.append(0)
    # pixel 1: coincident lines of sight, different names (rt = 0), exact rp edges
    base = dict(ra=31.0 * deg, dec=11.0 * deg)
    d1 = 4000.0 + 4.0 * np.arange(40)                    # |d1 - d2| multiples of 4 exactly
    d2 = 4000.0 + 4.0 * np.arange(40) + 0.0
    F.append(dict(base, dc=d1, w=np.ones(40), dw=np.linspace(-1, 1, 40), z=np.full(40, 2.3)))
    names.append(500); pix.append(1)
    F.append(dict(ra=31.0 * deg + 1e-12, dec=11.0 * deg, dc=d2 + 2.0, w=np.ones(40), dw=np.linspace(1, -1, 40),
                  z=np.full(40, 2.4)))
    names.append(501); pix.append(1)
    # pixel 2: pairs across ra = 0 / 2 pi
    F.append(same_grid_forest(2 * np.pi - 0.2 * deg, 0.5 * deg, 100, 200, rng)); names.append(600); pix.append(2)
    F.append(same_grid_forest(0.1 * deg, 0.6 * deg, 120, 200, rng)); names.append(601); pix.append(2)
    F.append(same_grid_forest(0.3 * deg, 0.2 * deg, 80, 150, rng)); names.append(602); pix.append(2)
    return forestset(F, names=np.array(names), pix=np.array(pix))
