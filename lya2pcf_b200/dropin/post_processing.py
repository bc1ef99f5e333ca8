"""Post-processing driver with the CLI and outputs of lya2pcf's ``post_processing.py``.

    python post_processing.py [--write-coordinates] [--diagonal-error]

Reads every ``corr_dir/2d_histogram_pixel_*`` file (w_hist, dw_hist of one
owner pixel), forms xi = dw/w per pixel (0 where w = 0), and writes
``covariance.npy``, ``covariance_not_smooth.npy``, ``correlation_2d.npy``,
``error_2d.npy`` (and ``rp.npy``, ``rt.npy`` with --write-coordinates), then
the FITS table ``correlation.out.gz`` with the distortion matrix when
``distortion.npy`` exists (post_processing.py:111-218).  The covariance and its
smoothing (post_processing.py:30-91) run on the GPU through
:mod:`lya2pcf_b200.covariance`; fitsio is imported only for the FITS table.
"""
import argparse
import glob
import os
import sys
import warnings

import numpy as np

_here = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, _here)
sys.path.insert(1, os.path.dirname(os.path.dirname(_here)))

from parameters import *   # noqa: E402,F401,F403
from parameters import corr_dir, numpix_rp, numpix_rt, rpmax, rtmax, Omm   # noqa: E402
from lya2pcf_b200.covariance import bin_coordinates, cov, cov_smooth, diag_error   # noqa: E402,F401


def read_histograms(corr_dir_, shape_hist):
    """(da, we): per-pixel xi = dw/w and w, flattened, one row per file of
    ``2d_histogram_pixel_*`` (post_processing.py:128-149)."""
    histogram_files = glob.glob(corr_dir_ + '2d_histogram_pixel_*')
    print('In total ' + str(len(histogram_files)) + ' files were found.')
    we_list, cor_list = [], []
    for file in histogram_files:
        w_hist, dw_hist = np.load(file)
        w_hist = w_hist.flatten()
        dw_hist = dw_hist.flatten()
        we_list.append(w_hist)
        cor_list.append(np.divide(dw_hist, w_hist, out=np.zeros_like(dw_hist), where=w_hist != 0))
    return np.array(cor_list), np.array(we_list)


def main(argv=None):
    parser = argparse.ArgumentParser(formatter_class=argparse.ArgumentDefaultsHelpFormatter,
                                     description='Correlation, covariance and errors from the histogram files of 2pla.py.')
    parser.add_argument('--write-coordinates', action='store_true', required=False)
    parser.add_argument('--diagonal-error', action='store_true', required=False)
    parser.add_argument('--corr-dir', default=corr_dir)
    args = parser.parse_args(argv)
    cdir = args.corr_dir
    shape = (numpix_rp, numpix_rt)
    print('Looking for histogram files in ' + cdir)
    da, we = read_histograms(cdir, shape)
    if args.diagonal_error:
        print('We are computing diagonal error, not the full covariance.')
        error, correlation = diag_error(da, we)
    else:
        covariance_not_smooth, correlation = cov(da, we, numpix=shape)
        bin_r_p, bin_r_t = bin_coordinates(numpix_rp, numpix_rt)
        covariance = cov_smooth(da, we, bin_r_p, bin_r_t, covariance_not_smooth, numpix=shape)
        error = np.sqrt(np.diagonal(covariance))
        np.save(cdir + 'covariance', covariance)
        np.save(cdir + 'covariance_not_smooth', covariance_not_smooth)
    correlation = np.reshape(correlation, shape)
    error = np.reshape(error, shape)
    np.save(cdir + 'correlation_2d', correlation)
    np.save(cdir + 'error_2d', error)
    rp = np.repeat(((np.arange(numpix_rp) + 0.5) * rpmax / numpix_rp)[:, None], numpix_rt, axis=1)
    rt = np.repeat(((np.arange(numpix_rt) + 0.5) * rtmax / numpix_rt)[None, :], numpix_rp, axis=0)
    if args.write_coordinates:
        np.save(cdir + 'rp', rp)
        np.save(cdir + 'rt', rt)
    if not os.path.exists(cdir + 'distortion.npy') or args.diagonal_error:
        warnings.warn('No distortion.npy found. Compute it first if you want to obtain a fits.gz file with all the outputs.')
        return 0
    import fitsio   # only the FITS table needs it
    distortion = np.load(cdir + 'distortion.npy')
    n_rows = numpix_rp * numpix_rt
    matrix_type = str(int(n_rows)) + 'D'
    dtype = [('DA', 'f8'), ('RP', 'f8'), ('RT', 'f8'), ('CO', matrix_type), ('DM', matrix_type)]
    table = np.zeros(n_rows, dtype=dtype)
    table['DA'] = correlation.flatten()
    table['RP'] = rp.flatten()
    table['RT'] = rt.flatten()
    table['CO'] = covariance
    table['DM'] = distortion
    header = {'RPMIN': 0, 'RPMAX': rpmax, 'RTMAX': rtmax, 'NP': numpix_rp, 'NT': numpix_rt, 'OMEGAM': Omm,
              'OMEGAR': 0, 'OMEGAK': 0, 'WL': -1}
    f = fitsio.FITS(cdir + 'correlation.out.gz', 'rw')
    f.write(table, extname='COR', header=header)
    f.close()
    return 0


if __name__ == '__main__':
    sys.exit(main())
