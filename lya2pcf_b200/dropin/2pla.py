"""Two-point correlation driver with the CLI of lya2pcf's ``2pla.py``.

    python 2pla.py (--cpu | --gpu) [--verbose] [--data-dir DIR] [--corr-dir DIR] [--resume]
                   [--stale-after S]

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
(``2pla.py:21``).  With ``--gpu`` the owner pixels are shared by LPT on their
pair count instead of ``np.array_split`` by pixel count.

Additions the reference lacks (lya2pcf_b200.requeue): ``--resume`` computes
only the pixels whose output file is missing; with several ranks every rank
keeps a heartbeat file in corr_dir, and rank 0, after its own share, waits on
the host (no collective) until every other rank has finished or has not
beaten for ``--stale-after`` seconds, then computes the pixels a dead rank
left unfinished.
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
from lya2pcf_b200.requeue import ShareTracker, pending   # noqa: E402




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
    parser.add_argument('--resume', action='store_true', help='skip pixels whose output file exists')
    parser.add_argument('--stale-after', type=float, default=120.0,
                        help='seconds without a heartbeat after which rank 0 re-queues a rank\'s pixels')
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

    todo = pending(corr_dir, pixels_total) if args.resume else pixels_total
    if args.gpu and size > 1:
        from lya2pcf_b200.sharding import shard_slots
        eng = correlations._engine
        f1, f2 = eng.get_pairs()
        L = eng.fs.lengths
        costs = np.bincount(eng.slot_of_forest[f1], weights=L[f1] * L[f2], minlength=len(eng.slot_pixels))
        wanted = set(int(p) for p in todo)
        costs[[int(p) not in wanted for p in eng.slot_pixels.tolist()]] = 0.0
        share = set(int(p) for p in eng.slot_pixels[shard_slots(costs, size)[rank]])
        mine = [int(p) for p in todo if int(p) in share]
        correlations.restrict_pixels(mine)
    else:
        mine = [int(p) for p in np.array_split(np.array(todo, dtype=np.int64), size)[rank]]

    tracker = ShareTracker(corr_dir, rank, size, stale_after=args.stale_after) if size > 1 else None
    if tracker:
        tracker.start()

    def compute(pixels):
        log_file.write(f'\nThis process computes {len(pixels)} pixels')
        for count, pixel in enumerate(pixels):
            log_file.write(f'\nComputing pixel {pixel}, completed {int(count / max(len(pixels), 1) * 100)}%')
            log_file.flush()
            histo = correlations.two_point_per_pixel(pixel)
            np.save(corr_dir + '2d_histogram_pixel_' + str(pixel), histo)
            if args.gpu:
                np.savez(corr_dir + 'pairs_2d_pixel_' + str(pixel), **correlations.pixel_extras(pixel))
            if tracker:
                tracker.beat()
            if args.verbose and count + 1 > 1:
                print('Exiting early due to --verbose option.')
                return False
        return True

    complete = compute(mine)
    if tracker:
        tracker.finish()
        if rank == 0 and complete:
            left = tracker.missing([int(p) for p in todo])
            if left:
                log_file.write(f'\nRe-queued {len(left)} pixels of ranks that stopped')
                if args.gpu:
                    correlations.restrict_pixels(left)
                compute(left)
    log_file.close()
    ranks.close()
    print('Finished correlation computation.')


if __name__ == '__main__':
    main()
