"""Generate the golden fixtures in this directory from the reference itself.

Runs where the lya2pcf reference tree is available, named by the required
``LYA2PCF_REFERENCE`` environment variable: it imports the
reference's numba CPU kernel ``correlation_procedures_cpu.pair_correlation``
(``correlation_procedures_cpu.py:46-84``) and its ``two_point_per_pixel`` driver
(``:19-43``), feeds them seeded synthetic forests, and stores inputs and outputs
as ``.npz`` (``numba_pairs``: hand-placed pairs; ``numba_sweep``: seeded random
pairs over the whole sky; ``numba_pixel``: one pixel through the driver).  The GPU test machine has no reference tree; it only reads the
committed ``.npz`` files.

    LYA2PCF_REFERENCE=<reference tree> python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

REF = os.environ.get('LYA2PCF_REFERENCE', '')
if __name__ == '__main__' and not REF:
    raise SystemExit('set LYA2PCF_REFERENCE to the lya2pcf reference tree')
OUT = os.path.dirname(os.path.abspath(__file__))


def _forest(rng, n, lam_start_idx, ra, dec):
    sys.path.insert(0, os.path.dirname(os.path.dirname(OUT)))
    from lya2pcf_b200.cosmology import dc_interpol
    k = lam_start_idx + np.arange(n)
    loglam = np.log10(3600.0) + 3e-4 * k
    z = 10 ** loglam / 1215.67 - 1
    dc = dc_interpol(z)
    w = ((1 + z) / 3.25) ** 1.9 / (0.1 + rng.uniform(0.01, 0.5, n))
    delta = rng.normal(0, 0.25, n)
    dw = w * (delta - np.average(delta, weights=w))
    return dict(ra=float(ra), dec=float(dec), dc=np.asarray(dc, dtype=np.float64), w=w, dw=dw, z=z)


def main():
    sys.path.insert(0, REF)
    import correlation_procedures_cpu as cpu   # the reference module, read-only
    import parameters as refpar
    shape = (refpar.numpix_rp, refpar.numpix_rt)
    rng = np.random.default_rng(7)
    deg = np.pi / 180
    angmax = 2 * np.arcsin(0.5 * refpar.rtmax / 3540.0)
    cpu.init({}, None, shape, angmax)

    # ---- single forest pairs: numba pair_correlation, bit-level reference
    cases = []
    specs = [
        # (len1, len2, start1, start2, separation deg, position angle deg)
        (40, 60, 0, 10, 0.5, 30.0),
        (120, 90, 100, 130, 1.2, 75.0),
        (200, 150, 50, 0, 2.9, 10.0),
        (64, 64, 300, 300, 0.05, 45.0),
        (1, 80, 40, 20, 0.8, 200.0),       # length-1 forest
        (97, 33, 500, 560, 3.1, 300.0),
        (150, 150, 0, 0, 0.0004, 0.0),     # 1.4 arcsec: the small-angle branch
    ]
    for (l1, l2, s1, s2, sep, pa) in specs:
        ra1, dec1 = 150.0 * deg, 2.0 * deg
        dra = sep * np.sin(pa * deg) / np.cos(dec1)
        ddec = sep * np.cos(pa * deg)
        ra2, dec2 = ra1 + dra * deg, dec1 + ddec * deg
        a = _forest(rng, l1, s1, ra1, dec1)
        b = _forest(rng, l2, s2, ra2, dec2)
        wh, dwh = cpu.pair_correlation(angmax, a['ra'], a['dec'], a['w'], a['dw'], 0, a['dc'], 0,
                                       b['ra'], b['dec'], b['w'], b['dw'], 0, b['dc'], 0)
        cases.append((a, b, wh, dwh))

    payload = {'angmax': angmax, 'n_cases': len(cases), 'rpmax': float(refpar.rpmax), 'rtmax': float(refpar.rtmax),
               'np': int(refpar.numpix_rp), 'nt': int(refpar.numpix_rt)}
    for c, (a, b, wh, dwh) in enumerate(cases):
        for tag, f in (('a', a), ('b', b)):
            for k, v in f.items():
                payload[f'c{c}_{tag}_{k}'] = np.asarray(v)
        payload[f'c{c}_w_hist'] = wh
        payload[f'c{c}_dw_hist'] = dwh
    np.savez_compressed(os.path.join(OUT, 'numba_pairs.npz'), **payload)
    print('wrote numba_pairs.npz with', len(cases), 'forest pairs')

    # ---- a whole pixel through the reference CPU backend (two_point_per_pixel)
    class Q:   # minimal stand-in with the attributes the CPU backend reads
        pass
    data = {}
    forests = []
    for f in range(12):
        q = Q()
        fr = _forest(rng, int(rng.integers(20, 90)), int(rng.integers(0, 400)),
                     150.0 * deg + rng.uniform(0, 1.5) * deg, 2.0 * deg + rng.uniform(0, 1.5) * deg)
        q.ra, q.dec, q.dc, q.we, q.dw = fr['ra'], fr['dec'], fr['dc'], fr['w'], fr['dw']
        q.pl = 0; q.fib = 0; q.name = 1000 + f
        q.z_pix = fr['z']
        forests.append(q)
    # neighbour lists are supplied explicitly (healpy is absent): every later
    # forest with larger ra is a neighbour, in list order
    order = sorted(range(len(forests)), key=lambda i: forests[i].ra)
    for q in forests:
        q.neigh = [o for o in forests if o.ra > q.ra]
        q.neighborhood = (lambda qq: (lambda data_, angmax_: qq.neigh))(q)
    data[7] = forests
    cpu.init(data, None, shape, angmax)
    wh, dwh = cpu.two_point_per_pixel(7)
    payload = {'angmax': angmax, 'n': len(forests)}
    for f, q in enumerate(forests):
        payload[f'f{f}_ra'] = q.ra; payload[f'f{f}_dec'] = q.dec; payload[f'f{f}_dc'] = q.dc
        payload[f'f{f}_w'] = q.we; payload[f'f{f}_dw'] = q.dw; payload[f'f{f}_z'] = q.z_pix
        payload[f'f{f}_nbr'] = np.array([forests.index(o) for o in q.neigh], dtype=np.int64)
    payload['w_hist'] = wh
    payload['dw_hist'] = dwh
    del order
    np.savez_compressed(os.path.join(OUT, 'numba_pixel.npz'), **payload)
    print('wrote numba_pixel.npz')
    sweep(cpu, refpar, angmax)


def _offset(ra1, dec1, sep, pa):
    """The point at angular distance sep and position angle pa from (ra1, dec1)."""
    dec2 = np.arcsin(np.sin(dec1) * np.cos(sep) + np.cos(dec1) * np.sin(sep) * np.cos(pa))
    ra2 = ra1 + np.arctan2(np.sin(pa) * np.sin(sep) * np.cos(dec1), np.cos(sep) - np.sin(dec1) * np.sin(dec2))
    return float(np.mod(ra2, 2 * np.pi)), float(dec2)


def sweep(cpu, refpar, angmax, n_cases=32):
    """numba_sweep.npz: seeded random forest pairs over the whole sky through
    the reference numba pair_correlation, same layout as numba_pairs.npz.
    Declinations up to +-80 deg, a quarter of the pairs straddling ra = 0 / 2 pi,
    separations up to 1.05 angmax (the reference's angle cut, ``:69``, drops
    the farthest), lengths 1..250 anywhere on the 614-pixel grid."""
    rng = np.random.default_rng(11)
    deg = np.pi / 180
    cases = []
    for c in range(n_cases):
        dec1 = rng.uniform(-80.0, 80.0) * deg
        ra1 = rng.uniform(0.0, 2 * np.pi) if c % 4 else float(np.mod(rng.uniform(-0.5, 0.5) * deg, 2 * np.pi))
        sep = angmax * rng.uniform(0.0, 1.05)
        ra2, dec2 = _offset(ra1, dec1, sep, rng.uniform(0.0, 2 * np.pi))
        l1, l2 = (int(x) for x in rng.integers(1, 251, 2))
        s1, s2 = (int(x) for x in rng.integers(0, 614 - 250, 2))
        a = _forest(rng, l1, s1, ra1, dec1)
        b = _forest(rng, l2, s2, ra2, dec2)
        wh, dwh = cpu.pair_correlation(angmax, a['ra'], a['dec'], a['w'], a['dw'], 0, a['dc'], 0,
                                       b['ra'], b['dec'], b['w'], b['dw'], 0, b['dc'], 0)
        cases.append((a, b, wh, dwh))
    payload = {'angmax': angmax, 'n_cases': len(cases), 'rpmax': float(refpar.rpmax), 'rtmax': float(refpar.rtmax),
               'np': int(refpar.numpix_rp), 'nt': int(refpar.numpix_rt)}
    for c, (a, b, wh, dwh) in enumerate(cases):
        for tag, f in (('a', a), ('b', b)):
            for k, v in f.items():
                payload[f'c{c}_{tag}_{k}'] = np.asarray(v)
        payload[f'c{c}_w_hist'] = wh
        payload[f'c{c}_dw_hist'] = dwh
    np.savez_compressed(os.path.join(OUT, 'numba_sweep.npz'), **payload)
    nonzero = sum(int(np.count_nonzero(wh) > 0) for _, _, wh, _ in cases)
    print('wrote numba_sweep.npz with', len(cases), 'forest pairs,', nonzero, 'with pairs in range')


if __name__ == '__main__':
    main()
