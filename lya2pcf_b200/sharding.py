"""Split owner pixels across ranks (one process per GPU).

The reference scatters healpix pixels over MPI ranks with
``np.array_split(pixels, mpi_size)`` (``2pla.py:87,102``), which balances pixel
counts, not work.  Here the owner slots (healpix pixels) go to ranks by
longest-processing-time-first (LPT) on their reference pair count (sum of
len1*len2 of the forest pairs they own): slots in decreasing cost order, each
to the rank with the least cost so far.  A rank's share is any subset of the
slots; the library keeps only that subset's pairs (``lya_select_slots``).
Per-slot histograms are disjoint, so the correlation needs no collective:
every rank writes its own pixels.
"""
import numpy as np


def slot_costs(lengths, f1, f2, slot_of_forest, n_slots):
    """Reference pair count of every owner slot of a forest-pair list."""
    lengths = np.asarray(lengths, dtype=np.float64)
    f1 = np.asarray(f1); f2 = np.asarray(f2)
    return np.bincount(np.asarray(slot_of_forest)[f1], weights=lengths[f1] * lengths[f2], minlength=n_slots)


def shard_slots(costs, world):
    """LPT shares: a list of ``world`` sorted int64 arrays of slot indices that
    partition ``range(len(costs))``.  The largest share exceeds the average by
    at most the largest single slot cost.  Ties go to the lowest rank, so every
    rank computes the same split from the same costs."""
    costs = np.asarray(costs, dtype=np.float64)
    n = len(costs)
    if world <= 1:
        return [np.arange(n, dtype=np.int64)]
    order = np.lexsort((np.arange(n), -costs))    # decreasing cost, then slot index
    load = np.zeros(world)
    owner = np.zeros(n, dtype=np.int64)
    for s in order:
        r = int(np.argmin(load))
        owner[s] = r
        load[r] += costs[s]
    return [np.nonzero(owner == r)[0].astype(np.int64) for r in range(world)]


def share_loads(costs, shares):
    """Total cost of every share."""
    costs = np.asarray(costs, dtype=np.float64)
    return np.array([costs[s].sum() for s in shares])
