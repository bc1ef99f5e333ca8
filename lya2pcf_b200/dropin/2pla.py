"""Two-point correlation driver with the CLI of lya2pcf's ``2pla.py``.

    python 2pla.py (--cpu | --gpu) [--verbose] [--data-dir DIR] [--corr-dir DIR]

Loads ``data_dir/data1.npy`` (pickled dict pixel -> list of
``forest_class.quasar``), computes angmax = 2 asin(rtmax / (2 dmin)) from the
smallest first-pixel distance (``2pla.py:64-73``), splits the pixels over the
ranks and writes ``corr_dir/2d_histogram_pixel_<pixel>.npy`` = (w_hist,
dw_hist) per pixel (``2pla.py:129-136``), which ``post_processing.py`` reads
unchanged.  With ``--gpu`` it also writes ``corr_dir/pairs_2d_pixel_<pixel>.npz``
(pair counts, weighted mean r_par / r_perp / z), whose names do not match the
``2d_histogram_pixel_*`` glob of ``post_processing.py``.

Ranks: mpi4py when installed (as the reference), else torchrun's torch.distributed
environment, else a single process (lya2pcf_b200.ranks).  The
GPU of a rank is ``rank % number_of_cuda_devices + cuda_device_first_number``
(``2pla.py:21``).  Pixels are split into contiguous runs balanced by pair
count instead of ``np.array_split`` by pixel count.
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
from lya2pcf_b200.ranks import Ranks   # noqa: E402




def main():
    ranks = Ranks()
    rank, size = ranks.rank, ranks.size
    os.environ['CUDA_DEVICE'] = str(int(rank % _P.number_of_cuda_devices + _P.cuda_device_first_number))
    parser = argparse.ArgumentParser(description='Takes the data.npy file and computes the two point correlation '
                                                 'function histograms.')
    g = parser.add_mutually_exclusive_group(required=True)
    g.add_argument('--cpu', action='store_true', help='Compute the forest correlation using the cpu.')
    g.add_argument('--gpu', action='store_true', help='Compute the forest correlation with the help of a GPU.')
    parser.add_argument('--verbose', action='store_true', help='Only compute the first two pixels.')
    parser.add_argument('--data-dir', default=_P.data_dir)
    parser.add_argument('--corr-dir', default=_P.corr_dir)
    args = parser.parse_args()
    data_dir = os.path.join(args.data_dir, '')
    corr_dir = os.path.join(args.corr_dir, '')
    os.makedirs(corr_dir, exist_ok=True)
    log_file = open(corr_dir + f'thread_{rank}_of_{size}.log', 'w+')

    data = np.load(data_dir + 'data1.npy', allow_pickle=True).item()
    dmin = min(float(f.dc[0]) for p in data for f in data[p] if len(f.dc))
    angmax = 2 * np.arcsin(0.5 * _P.rtmax / dmin)
    shape_hist = (_P.numpix_rp, _P.numpix_rt)
    pixels_total = list(data.keys())

    if args.cpu:
        import correlation_procedures_cpu as correlations   # the reference CPU backend, if importable
    else:
        import correlation_procedures_pycuda as correlations
    correlations.init(data, log_file, shape_hist, angmax)

    if args.gpu and size > 1:
        from lya2pcf_b200.sharding import shard_slots
        eng = correlations._engine
        f1, f2 = eng.get_pairs()
        L = eng.fs.lengths
        costs = np.bincount(eng.slot_of_forest[f1], weights=L[f1] * L[f2], minlength=len(eng.slot_pixels))
        lo, hi = shard_slots(costs, size)[rank]
        mine = [int(p) for p in eng.slot_pixels[lo:hi]]
        correlations.restrict_pixels(mine)
    else:
        mine = [int(p) for p in np.array_split(np.array(pixels_total), size)[rank]]

    log_file.write(f'\nThis process computes {len(mine)} pixels')
    for count, pixel in enumerate(mine):
        log_file.write(f'\nComputing pixel {pixel}, completed {int(count / max(len(mine), 1) * 100)}%')
        log_file.flush()
        histo = correlations.two_point_per_pixel(pixel)
        np.save(corr_dir + '2d_histogram_pixel_' + str(pixel), histo)
        if args.gpu:
            np.savez(corr_dir + 'pairs_2d_pixel_' + str(pixel), **correlations.pixel_extras(pixel))
        if args.verbose and count + 1 > 1:
            print('Exiting early due to --verbose option.')
            break
    log_file.close()
    ranks.close()
    print('Finished correlation computation.')


if __name__ == '__main__':
    main()
