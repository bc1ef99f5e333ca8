"""Split owner pixels across ranks (one process per GPU).

The reference scatters healpix pixels over MPI ranks with
``np.array_split(pixels, mpi_size)`` (``2pla.py:87,102``), which balances pixel
counts, not work.  Here each rank gets a contiguous range of owner slots with
about the same reference pair count (sum of len1*len2 of the forest pairs it
owns).  Per-slot histograms are disjoint, so the correlation needs no
collective: every rank writes its own pixels.
"""
import numpy as np


def slot_costs(lengths, f1, f2, slot_of_forest, n_slots):
    """Reference pair count of every owner slot of a forest-pair list."""
    lengths = np.asarray(lengths, dtype=np.float64)
    f1 = np.asarray(f1); f2 = np.asarray(f2)
    return np.bincount(np.asarray(slot_of_forest)[f1], weights=lengths[f1] * lengths[f2], minlength=n_slots)


def shard_slots(costs, world):
    """Contiguous slot ranges [(lo, hi)] * world with near-equal total cost
    (each boundary at the cost quantile r/world)."""
    costs = np.asarray(costs, dtype=np.float64)
    n = len(costs)
    if world <= 1:
        return [(0, n)]
    cum = np.concatenate([[0.0], np.cumsum(costs)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        b = int(np.searchsorted(cum, total * r / world, side='left'))
        bounds.append(min(max(b, bounds[-1]), n))
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]
