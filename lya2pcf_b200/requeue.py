"""Resume and re-queue of owner pixels for the drivers' ranks.

The reference writes one output file per owner pixel as soon as the pixel is
done (``2d_histogram_pixel_<p>.npy``, ``2pla.py:136``) and never looks at
them again: a rank that dies loses its remaining pixels, and a rerun starts
from scratch.  Here the output files are the record of what is done:

* ``pending(out_dir, pixels)``: the pixels whose output file does not exist
  (a rerun with ``--resume`` computes only those);
* every rank refreshes a heartbeat file while it works and writes a ``done``
  file when its share is finished (:class:`ShareTracker`);
* after its own share, rank 0 waits -- on the host, with a deadline, through
  files only (no collective that a dead rank could hang) -- until every other
  rank has either finished or stopped refreshing its heartbeat, then computes
  whatever pixels are still missing (:meth:`ShareTracker.missing`).

The output directory must be shared by the ranks, as the reference's drivers
already assume (every rank writes its pixels there).
"""
import os
import time

HIST_PREFIX = '2d_histogram_pixel_'


def hist_path(out_dir, pixel):
    """Output file of one owner pixel, as the reference driver names it."""
    return os.path.join(out_dir, f'{HIST_PREFIX}{int(pixel)}.npy')


def pending(out_dir, pixels):
    """The pixels (in the given order) whose output file does not exist."""
    return [p for p in pixels if not os.path.exists(hist_path(out_dir, p))]


class ShareTracker:
    """Heartbeat, completion and re-queue of the ranks' pixel shares."""

    def __init__(self, out_dir, rank, world, stale_after=30.0):
        self.dir = out_dir
        self.rank, self.world = int(rank), int(world)
        self.stale_after = float(stale_after)

    def _alive(self, r):
        return os.path.join(self.dir, f'.lya2pcf_rank{r}.alive')

    def _done(self, r):
        return os.path.join(self.dir, f'.lya2pcf_rank{r}.done')

    def start(self):
        """Clear this rank's marks of an earlier run and beat once."""
        if os.path.exists(self._done(self.rank)):
            os.remove(self._done(self.rank))
        self.beat()

    def beat(self):
        """Refresh this rank's heartbeat (call after every pixel)."""
        with open(self._alive(self.rank), 'w') as f:
            f.write(f'{time.time():.3f}\n')

    def finish(self):
        """Mark this rank's share as done."""
        with open(self._done(self.rank), 'w') as f:
            f.write(f'{time.time():.3f}\n')

    def rank_state(self, r, now=None):
        """'done', 'alive' or 'dead' (no heartbeat for stale_after seconds)."""
        if os.path.exists(self._done(r)):
            return 'done'
        now = time.time() if now is None else now
        try:
            age = now - os.path.getmtime(self._alive(r))
        except OSError:
            return 'dead' if now - self._t0 > self.stale_after else 'alive'
        return 'alive' if age <= self.stale_after else 'dead'

    def missing(self, all_pixels, deadline=600.0, poll=0.5):
        """Rank 0, after its own share: wait until every other rank is done or
        dead (at most ``deadline`` seconds, then every unfinished rank counts as
        dead), and return the pixels of ``all_pixels`` that still have no output
        file -- the dead ranks' unfinished pixels, to be computed here."""
        self._t0 = time.time()
        while True:
            states = [self.rank_state(r) for r in range(self.world) if r != self.rank]
            if all(s != 'alive' for s in states) or time.time() - self._t0 > deadline:
                break
            time.sleep(poll)
        return pending(self.dir, all_pixels)

    _t0 = 0.0
