"""Distortion-matrix driver with the CLI of lya2pcf's ``distortion.py``.

    python distortion.py [--excluded 0.95] [--verbose] [--data-dir DIR] [--corr-dir DIR]

Loads ``data_dir/data1.npy``, computes angmax from the smallest first-pixel
distance, sums ``distortion_per_pixel`` over this rank's pixels
(``distortion.py:101-108``), adds the ranks' sums (mpi4py ``reduce`` when
installed, as the reference at ``:118-119``, else one torch.distributed
reduce when started by torchrun) and saves
``corr_dir/distortion.npy = D / W[:, None]`` (``:125``).
"""
import argparse
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


def main():
    ranks = Ranks()
    rank, size = ranks.rank, ranks.size
    os.environ['CUDA_DEVICE'] = str(int(rank % _P.number_of_cuda_devices + _P.cuda_device_first_number))
    parser = argparse.ArgumentParser(description='Takes the data.npy file and computes the distortion matrix of the '
                                                 'two point correlation function.')
    parser.add_argument('--excluded', default=0.95, help='Fraction of forests pairs excluded from the computation.')
    parser.add_argument('--verbose', action='store_true', help='Only compute the first two pixels.')
    parser.add_argument('--data-dir', default=_P.data_dir)
    parser.add_argument('--corr-dir', default=_P.corr_dir)
    args = parser.parse_args()
    data_dir = os.path.join(args.data_dir, '')
    corr_dir = os.path.join(args.corr_dir, '')
    os.makedirs(corr_dir, exist_ok=True)
    log_file = open(corr_dir + f'thread_{rank}_of_{size}_distortion.log', 'w+')
    data = np.load(data_dir + 'data1.npy', allow_pickle=True).item()
    shape_hist = (_P.numpix_rp, _P.numpix_rt)
    total_bins = int(np.prod(shape_hist))
    disto = np.zeros((total_bins, total_bins))
    weight_A = np.zeros(total_bins)
    pixels_list = np.array_split(np.array(list(data.keys())), size)[rank]
    dmin = min(float(f.dc[0]) for p in data for f in data[p] if len(f.dc))
    angmax = 2 * np.arcsin(0.5 * _P.rtmax / dmin)
    distortion.init(data, log_file, shape_hist, angmax, float(args.excluded))
    for count, pixel in enumerate(pixels_list):
        log_file.write(f'\nComputing pixel {pixel}, completed {int(count / max(len(pixels_list), 1) * 100)}%')
        log_file.flush()
        d, w = distortion.distortion_per_pixel(data[pixel])
        disto += d
        weight_A += w
        if args.verbose and count + 1 > 1:
            print('Exiting early due to --verbose option.')
            break
    disto, weight_A = ranks.reduce_sum(disto, weight_A)
    if rank == 0:
        with np.errstate(divide='ignore', invalid='ignore'):
            np.save(corr_dir + 'distortion', disto / weight_A[:, None])
    ranks.close()
    print('Finished distortion computation.')


if __name__ == '__main__':
    main()
