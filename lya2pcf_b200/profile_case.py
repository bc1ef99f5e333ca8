"""One pass of a hot kernel over a synthetic catalogue, for profilers.

    python -m lya2pcf_b200.profile_case --config 1 --scale 0.1 --kernel 0
    python -m lya2pcf_b200.profile_case --config 3 --scale 0.03 --distortion

Builds the catalogue, uploads it, builds the work queue, runs the chosen pair
kernel (or the distortion matrix) once -- a warm-up run first when --warm is
given -- and prints the library's statistics.  Used to capture one kernel
under ncu on a case whose inputs exceed L2 while holding a few GB at most.
"""
import argparse
import json

from . import synthetic
from .engine import PairEngine


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--config', type=int, default=1)
    ap.add_argument('--scale', type=float, default=0.1)
    ap.add_argument('--kernel', type=int, default=0)
    ap.add_argument('--variant', type=int, default=0)
    ap.add_argument('--distortion', action='store_true', help='distortion matrix instead of the histograms')
    ap.add_argument('--warm', action='store_true')
    args = ap.parse_args()
    fs = synthetic.make(args.config, scale=args.scale)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(synthetic.angmax_for(fs))
        if args.distortion:
            if args.warm:
                eng.distortion()
            eng.distortion()
            st = eng.stats()
        else:
            if args.warm:
                eng.run(kernel=args.kernel, variant=args.variant)
            st = eng.run(kernel=args.kernel, variant=args.variant)
        st['npix_total'] = fs.npix_total
        print(json.dumps(st))


if __name__ == '__main__':
    main()
