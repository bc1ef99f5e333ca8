"""Resume and re-queue of owner pixels (lya2pcf_b200.requeue) on CPU.

A rank that dies is made on the host: rank 1 of two gloo ranks writes one
pixel and then leaves with os._exit, without finishing or cleaning up.  Rank
0, after its own share, waits on the host through the heartbeat files (no
collective) and computes the pixels rank 1 left.  The per-pixel compute is the
CPU oracle; the union of the files must equal the single-process result."""
import os
import socket
import time

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from lya2pcf_b200.requeue import ShareTracker, hist_path, pending


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _catalogue():
    from lya2pcf_b200 import synthetic
    from oracle import oracle as O
    fs = synthetic.make(0, scale=0.05)
    am = synthetic.angmax_for(fs)
    off, nbr = O.neighbours(fs, am, nthreads=1)
    return fs, O.items_from_csr(fs, off, nbr)


def _pixel_hist(fs, items, s):
    from oracle import oracle as O
    f1, f2, sis, _ = items
    h, _ = O.corr(fs, f1[sis[s]:sis[s + 1]], f2[sis[s]:sis[s + 1]], [0, sis[s + 1] - sis[s]], nthreads=1)
    return np.stack([h[0, O.Q_W], h[0, O.Q_DW]])


def _worker(rank, world, port, out_dir, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    fs, items = _catalogue()
    pixels = [int(p) for p in items[3]]
    shares = [pixels[r::world] for r in range(world)]
    tr = ShareTracker(out_dir, rank, world, stale_after=2.0)
    tr.start()
    for k, p in enumerate(shares[rank]):
        np.save(hist_path(out_dir, p), _pixel_hist(fs, items, pixels.index(p)))
        tr.beat()
        if rank == 1 and k == 0:
            os._exit(3)      # dies without finishing, cleaning up or leaving the group
    tr.finish()
    left = tr.missing(pixels, deadline=60.0, poll=0.2)
    for p in left:
        np.save(hist_path(out_dir, p), _pixel_hist(fs, items, pixels.index(p)))
    q.put((len(left), len(shares[1]) - 1, pending(out_dir, pixels)))
    q.close()
    q.join_thread()          # the result reaches the parent before the process ends
    os._exit(0)              # the peer is gone: leave without a group teardown


def test_rank_that_dies_is_requeued(tmp_path):
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = []
    for r in range(2):
        p = ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path), q))
        p.start()
        procs.append(p)
    left, expected, still = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
    assert procs[1].exitcode == 3
    assert left == expected > 0 and still == []
    fs, items = _catalogue()
    for s, p in enumerate(items[3].tolist()):
        assert np.array_equal(np.load(hist_path(str(tmp_path), p)), _pixel_hist(fs, items, s))


def test_resume_lists_only_missing_pixels(tmp_path):
    pix = [5, 9, 12, 40]
    np.save(hist_path(str(tmp_path), 9), np.zeros(2))
    np.save(hist_path(str(tmp_path), 40), np.zeros(2))
    assert pending(str(tmp_path), pix) == [5, 12]


def test_tracker_states(tmp_path):
    a = ShareTracker(str(tmp_path), 0, 3, stale_after=0.5)
    b = ShareTracker(str(tmp_path), 1, 3, stale_after=0.5)
    a._t0 = b._t0 = time.time()
    b.start()
    assert a.rank_state(1) == 'alive'
    assert a.rank_state(2) == 'alive'            # not started yet, within the grace period
    b.finish()
    assert a.rank_state(1) == 'done'
    assert a.rank_state(2, now=time.time() + 1.0) == 'dead'
