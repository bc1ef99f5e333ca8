"""Two-point driver over several data files, with the CLI of lya2pcf's
``2pla_multiple_data.py``.

    python 2pla_multiple_data.py (--cpu | --gpu) [--verbose] [--per-file]
                                  [--data-dir DIR] [--corr-dir DIR]

The reference (``2pla_multiple_data.py:47-119``) splits the ``data*.npy`` files
over the ranks and ``init``-s and bins each file alone, so pairs of forests
that sit in different files are never counted.  By default this driver merges
every file into one catalogue and one device work queue (angmax from the
smallest first-pixel distance of all files), so an owner pixel's histograms
include its partners from every file; ``--per-file`` reproduces the
reference's per-file computation (its own angmax per file).  Either way one
``2d_histogram_pixel_<pixel>.npy`` = (w_hist, dw_hist) is written per owner
pixel, which ``post_processing.py`` reads unchanged; with ``--gpu`` also
``pairs_2d_pixel_<pixel>.npz`` (counts and weighted mean r_par, r_perp, z).
A pixel present in several files is one owner pixel in the merged catalogue;
with ``--per-file`` the last file's histogram of it is kept, as the reference
overwrites it.
"""
import argparse
import glob
import os
import sys

import numpy as np

_here = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, _here)
sys.path.insert(1, os.path.dirname(os.path.dirname(_here)))

from parameters import *   # noqa: E402,F401,F403
import parameters as _P   # noqa: E402
from forest_class import quasar   # noqa: E402,F401  (unpickling needs it)
from lya2pcf_b200.ranks import Ranks   # noqa: E402




def _angmax(data):
    dmin = min(float(f.dc[0]) for p in data for f in data[p] if len(f.dc))
    return 2 * np.arcsin(0.5 * _P.rtmax / dmin)


def _bin_file(correlations, data, corr_dir, log_file, gpu, pixels, verbose):
    correlations.init(data, log_file, (_P.numpix_rp, _P.numpix_rt), _angmax(data))
    for count, pixel in enumerate(pixels):
        log_file.write(f'\nComputing pixel {pixel}, completed {int(count / max(len(pixels), 1) * 100)}%')
        log_file.flush()
        np.save(corr_dir + '2d_histogram_pixel_' + str(pixel), correlations.two_point_per_pixel(pixel))
        if gpu:
            np.savez(corr_dir + 'pairs_2d_pixel_' + str(pixel), **correlations.pixel_extras(pixel))
        if verbose and count + 1 > 1:
            print('Exiting early due to --verbose option.')
            break


def main(argv=None):
    ranks = Ranks()
    rank, size = ranks.rank, ranks.size
    os.environ['CUDA_DEVICE'] = str(int(rank % _P.number_of_cuda_devices + _P.cuda_device_first_number))
    parser = argparse.ArgumentParser(description='Computes the two point correlation histograms of every data*.npy '
                                                 'file of a directory.')
    g = parser.add_mutually_exclusive_group(required=True)
    g.add_argument('--cpu', action='store_true', help='Compute the forest correlation using the cpu.')
    g.add_argument('--gpu', action='store_true', help='Compute the forest correlation with the help of a GPU.')
    parser.add_argument('--verbose', action='store_true', help='Only compute the first two pixels of a file.')
    parser.add_argument('--per-file', action='store_true',
                        help='bin every file alone, as the reference does (pairs across files are not counted)')
    parser.add_argument('--data-dir', default=_P.data_dir)
    parser.add_argument('--corr-dir', default=_P.corr_dir)
    args = parser.parse_args(argv)
    data_dir = os.path.join(args.data_dir, '')
    corr_dir = os.path.join(args.corr_dir, '')
    os.makedirs(corr_dir, exist_ok=True)
    log_file = open(corr_dir + f'thread_{rank}_of_{size}.log', 'w+')
    files = sorted(glob.glob(data_dir + 'data*.npy'))
    if not files:
        raise NameError('Empty data. Did you write correctly the input directory?')
    if args.cpu:
        import correlation_procedures_cpu as correlations   # the reference CPU backend, if importable
    else:
        import correlation_procedures_pycuda as correlations

    if args.per_file:
        for datafile in [str(f) for f in np.array_split(np.array(files), size)[rank]]:
            data = np.load(datafile, allow_pickle=True).item()
            _bin_file(correlations, data, corr_dir, log_file, args.gpu, list(data.keys()), args.verbose)
    else:
        data = {}
        for datafile in files:
            for pixel, forests in np.load(datafile, allow_pickle=True).item().items():
                data.setdefault(pixel, []).extend(forests)
        pixels = list(data.keys())
        mine = [p for p in np.array_split(np.array(pixels, dtype=object), size)[rank]]
        _bin_file(correlations, data, corr_dir, log_file, args.gpu, mine, args.verbose)
    log_file.close()
    ranks.close()
    print('Finished correlation computation.')
    return 0


if __name__ == '__main__':
    sys.exit(main())
