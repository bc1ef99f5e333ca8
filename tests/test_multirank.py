"""The multi-rank path on CPU: two gloo ranks split the owner pixels of one
catalogue (sharding.shard_slots), each computes only its pixels, and the
union equals the single-process result.  The per-rank compute here is the
CPU oracle (the GPU library is exercised by the gpu tests); what is under test
is the ownership split and the absence of any data-path collective: results
are only gathered at the end to check them."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch
    from lya2pcf_b200 import synthetic
    from lya2pcf_b200.engine import owner_slots
    from lya2pcf_b200.sharding import shard_slots, slot_costs
    from oracle import oracle as O
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        fs = synthetic.make(0, scale=0.1)
        am = synthetic.angmax_for(fs)
        off, nbr = O.neighbours(fs, am, nthreads=2)
        f1, f2, sis, pixels = O.items_from_csr(fs, off, nbr)
        slot, _ = owner_slots(fs.pix)
        costs = slot_costs(fs.lengths, f1, f2, slot, len(pixels))
        lo, hi = shard_slots(costs, world)[rank]
        mine, cnt = O.corr(fs, f1[sis[lo]:sis[hi]], f2[sis[lo]:sis[hi]], sis[lo:hi + 1] - sis[lo], nthreads=2)
        full = np.zeros((len(pixels), O.NQ, 2500))
        full[lo:hi] = mine
        t = torch.from_numpy(full)
        gathered = [torch.zeros_like(t) for _ in range(world)]
        dist.all_gather(gathered, t)
        if rank == 0:
            union = sum(g.numpy() for g in gathered)
            ref, _ = O.corr(fs, f1, f2, sis, nthreads=2)
            q.put((bool(np.array_equal(union, ref)), float(costs[lo:hi].sum()), float(costs.sum())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_cover_every_pixel_once():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, q), nprocs=2, join=True, start_method='spawn')
    ok, mine, total = q.get(timeout=60)
    assert ok
    assert 0.3 * total < mine < 0.7 * total


def _reduce_worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from lya2pcf_b200.ranks import Ranks
    r = Ranks()
    try:
        rng = np.random.default_rng(rank)
        d, w = rng.normal(size=(50, 50)), rng.uniform(size=50)
        sd, sw = r.reduce_sum(d, w)
        if r.rank == 0:
            r1 = np.random.default_rng(1)
            d1 = r1.normal(size=(50, 50))
            w1 = r1.uniform(size=50)
            q.put((bool(np.allclose(sd, d + d1, rtol=0, atol=1e-14)), bool(np.allclose(sw, w + w1, rtol=0, atol=1e-14)),
                   r.size))
    finally:
        r.close()


def test_distortion_reduction_over_torch_ranks():
    """The drivers' rank helper without mpi4py: two torchrun-style gloo ranks;
    rank 0 receives the sum of the ranks' distortion numerators and weights
    (the single collective of the distortion driver)."""
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    mp.start_processes(_reduce_worker, args=(2, port, q), nprocs=2, join=True, start_method='spawn')
    okd, okw, size = q.get(timeout=60)
    assert okd and okw and size == 2
