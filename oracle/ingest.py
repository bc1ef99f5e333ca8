"""CPU restatement of the reference's delta projection -- test infrastructure
(the checker of lya_upload_deltas), never part of the product path.

Follows lya2pcf ``forest_class.py:48-68`` (quasar.fill_dw): with weights w,
deltas de and log10(lambda) loglam of one forest and project=True,
    deltaprom = average(de, w), lambda_average = average(loglam, w)
    delta_lambda = loglam - lambda_average
    omega_delta_lambda2 = sum(delta_lambda^2 w)
    Ldprom = average(delta_lambda de, w), LLprom = average(delta_lambda^2, w)
    dw = w (de - deltaprom - delta_lambda Ldprom / LLprom),  omega = sum(w)
(LLprom = 0, e.g. a one-pixel forest, gives NaN as in numpy); project=False
gives dw = de w only.  Pinned against golden vectors from the reference's own
method (tests/golden/make_fill_dw_golden.py).
"""
import numpy as np


def fill_dw(we, de, loglam, project=True):
    """Returns (dw, delta_lambda, omega, omega_delta_lambda2) of one forest."""
    we = np.asarray(we, dtype=np.float64)
    de = np.asarray(de, dtype=np.float64)
    loglam = np.asarray(loglam, dtype=np.float64)
    if not project:
        return de * we, np.zeros_like(de), 0.0, 0.0
    with np.errstate(all='ignore'):
        deltaprom = np.average(de, weights=we)
        lam = np.average(loglam, weights=we)
        dl = loglam - lam
        odl2 = np.sum(dl ** 2 * we)
        ld = np.average(dl * de, weights=we)
        ll = np.average(dl * dl, weights=we)
        dw = we * (de - deltaprom - dl * ld / ll)
    return dw, dl, float(np.sum(we)), float(odl2)


def fill_dw_all(start, we, de, loglam, project=True):
    """fill_dw of every forest of a CSR catalogue (forest f owns start[f]..start[f+1]-1)."""
    n = len(start) - 1
    dw = np.empty_like(np.asarray(de, dtype=np.float64))
    dl = np.empty_like(dw)
    om = np.empty(n)
    o2 = np.empty(n)
    for f in range(n):
        a, b = start[f], start[f + 1]
        dw[a:b], dl[a:b], om[f], o2[f] = fill_dw(we[a:b], de[a:b], loglam[a:b], project)
    return dw, dl, om, o2
