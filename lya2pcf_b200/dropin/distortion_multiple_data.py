"""Distortion-matrix driver over several data files, with the CLI of lya2pcf's
``distortion_multiple_data.py``.

    python distortion_multiple_data.py [--excluded 0.95] [--verbose] [--per-file]
                                       [--data-dir DIR] [--corr-dir DIR]

The reference (``distortion_multiple_data.py:47-125``) splits the
``data*.npy`` files over the ranks and ``init``-s each file alone (its own
angmax), summing ``distortion_per_pixel`` over every pixel of the file, so
pairs of forests that sit in different files never enter the matrix.  By
default this driver merges every file into one catalogue and one device work
queue (angmax from the smallest first-pixel distance of all files) and splits
its owner pixels over the ranks, so an owner pixel's first forests keep their
partners from every file; ``--per-file`` reproduces the reference's per-file
computation, consuming Python's ``random`` stream in the same file, pixel and
forest order.  The ranks' sums are added (mpi4py ``reduce`` when installed, as
the reference at ``:129-130``, else one torch.distributed reduce under
torchrun) and rank 0 saves ``corr_dir/distortion.npy = D / W[:, None]``
(``:136``).
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
import distortion_procedures_pycuda as distortion   # noqa: E402
from lya2pcf_b200.ranks import Ranks   # noqa: E402


def _angmax(data):
    dminlist = [float(f.dc[0]) for p in data for f in data[p] if len(f.dc)]
    if not dminlist:
        raise NameError('Empty data. Did you write correctly the input directory?')
    return 2 * np.arcsin(0.5 * _P.rtmax / min(dminlist))


def _sum_file(data, pixels, log_file, excluded, verbose, disto, weight_A):
    """Adds distortion_per_pixel of ``pixels`` into (disto, weight_A), with
    ``data`` the catalogue ``init`` sees (``distortion_multiple_data.py:67-125``)."""
    shape_hist = (_P.numpix_rp, _P.numpix_rt)
    distortion.init(data, log_file, shape_hist, _angmax(data), excluded)
    for count, pixel in enumerate(pixels):
        log_file.write(f'\nComputing pixel {pixel}, completed {int(count / max(len(pixels), 1) * 100)}%')
        log_file.flush()
        d, w = distortion.distortion_per_pixel(data[pixel])
        disto += d
        weight_A += w
        if verbose and count + 1 > 1:
            print('Exiting early due to --verbose option.')
            break


def main(argv=None):
    ranks = Ranks()
    rank, size = ranks.rank, ranks.size
    os.environ['CUDA_DEVICE'] = str(int(rank % _P.number_of_cuda_devices + _P.cuda_device_first_number))
    parser = argparse.ArgumentParser(description='Takes the data*.npy files and computes the distortion matrix of the '
                                                 'two point correlation function.')
    parser.add_argument('--excluded', default=0.95, help='Fraction of forests pairs excluded from the computation.')
    parser.add_argument('--verbose', action='store_true', help='Only compute the first two pixels of a file.')
    parser.add_argument('--per-file', action='store_true',
                        help='init and sum every file alone, as the reference does (pairs across files are not used)')
    parser.add_argument('--data-dir', default=_P.data_dir)
    parser.add_argument('--corr-dir', default=_P.corr_dir)
    args = parser.parse_args(argv)
    data_dir = os.path.join(args.data_dir, '')
    corr_dir = os.path.join(args.corr_dir, '')
    os.makedirs(corr_dir, exist_ok=True)
    log_file = open(corr_dir + f'thread_{rank}_of_{size}_distortion.log', 'w+')
    files = sorted(glob.glob(data_dir + 'data*.npy'))
    if not files:
        raise NameError('Empty data. Did you write correctly the input directory?')
    total_bins = int(_P.numpix_rp * _P.numpix_rt)
    disto = np.zeros((total_bins, total_bins))
    weight_A = np.zeros(total_bins)
    excluded = float(args.excluded)

    if args.per_file:
        for datafile in [str(f) for f in np.array_split(np.array(files), size)[rank]]:
            data = np.load(datafile, allow_pickle=True).item()
            _sum_file(data, list(data.keys()), log_file, excluded, args.verbose, disto, weight_A)
            print('Finished data file ' + datafile)
    else:
        data = {}
        for datafile in files:
            for pixel, forests in np.load(datafile, allow_pickle=True).item().items():
                data.setdefault(pixel, []).extend(forests)
        mine = list(np.array_split(np.array(list(data.keys()), dtype=object), size)[rank])
        _sum_file(data, mine, log_file, excluded, args.verbose, disto, weight_A)

    disto, weight_A = ranks.reduce_sum(disto, weight_A)
    if rank == 0:
        with np.errstate(divide='ignore', invalid='ignore'):
            np.save(corr_dir + 'distortion', disto / weight_A[:, None])
    log_file.close()
    ranks.close()
    print('Finished distortion computation.')
    return 0


if __name__ == '__main__':
    sys.exit(main())
