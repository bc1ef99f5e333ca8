"""The multi-rank path on CPU: two gloo ranks split the owner pixels of one
catalogue (sharding.shard_slots, LPT on the reference pair count), each
computes only its pixels, and the union equals the single-process result.  The
per-rank compute here is the CPU oracle (the GPU library's share path is
exercised by the gpu tests); what is under test is the ownership split and the
absence of any data-path collective: results are only gathered at the end to
check them.  The adjoint's gradient reduction is checked the same way."""
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
        share = shard_slots(costs, world)[rank]
        full = np.zeros((len(pixels), O.NQ, 2500))
        for s in share:
            h, _ = O.corr(fs, f1[sis[s]:sis[s + 1]], f2[sis[s]:sis[s + 1]], [0, sis[s + 1] - sis[s]], nthreads=2)
            full[s] = h[0]
        t = torch.from_numpy(full)
        gathered = [torch.zeros_like(t) for _ in range(world)]
        dist.all_gather(gathered, t)
        if rank == 0:
            union = sum(g.numpy() for g in gathered)
            ref, _ = O.corr(fs, f1, f2, sis, nthreads=2)
            q.put((bool(np.array_equal(union, ref)), float(costs[share].sum()), float(costs.sum())))
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
    # gloo even where a GPU is visible: the test runs both ranks on one machine
    os.environ.update(LYA2PCF_DIST_BACKEND='gloo', MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port),
                      WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank))
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


def test_lpt_shares_partition_and_balance():
    from lya2pcf_b200.sharding import share_loads, shard_slots
    rng = np.random.default_rng(3)
    costs = rng.lognormal(0.0, 1.5, 500)
    costs[10:14] = costs.max() * 3          # a few heavy pixels next to each other
    for world in (2, 3, 8):
        shares = shard_slots(costs, world)
        allslots = np.sort(np.concatenate(shares))
        assert np.array_equal(allslots, np.arange(len(costs)))
        loads = share_loads(costs, shares)
        assert loads.max() - costs.sum() / world <= costs.max() + 1e-9
        assert shard_slots(costs, world)[0].tolist() == shares[0].tolist()   # deterministic


def _adjoint_worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    # gloo even where a GPU is visible: the test runs both ranks on one machine
    os.environ.update(LYA2PCF_DIST_BACKEND='gloo', MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port),
                      WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank))
    from lya2pcf_b200 import synthetic
    from lya2pcf_b200.engine import owner_slots
    from lya2pcf_b200.ranks import Ranks
    from lya2pcf_b200.sharding import shard_slots, slot_costs
    from oracle import oracle as O
    r = Ranks()
    try:
        fs = synthetic.make(4, n=80)
        am = synthetic.angmax_for(fs)
        off, nbr = O.neighbours(fs, am, nthreads=2)
        f1, f2, sis, pixels = O.items_from_csr(fs, off, nbr)
        slot, _ = owner_slots(fs.pix)
        costs = slot_costs(fs.lengths, f1, f2, slot, len(pixels))
        share = shard_slots(costs, r.size)[r.rank]
        items = np.concatenate([np.arange(sis[s], sis[s + 1]) for s in share]) if len(share) else np.zeros(0, int)
        # forward: this rank's W and DW totals, summed over the ranks (2 x nb values)
        h, _ = O.corr(fs, f1[items], f2[items], [0, len(items)], nthreads=2)
        W, DW = r.allreduce_sum(h[0, O.Q_W], h[0, O.Q_DW])
        g = np.random.default_rng(11).normal(size=2500)
        xi = np.divide(DW, W, out=np.zeros_like(W), where=W != 0)
        cdw = np.divide(g, W, out=np.zeros_like(W), where=W != 0)
        # backward: this rank's pairs scatter into both forests; the sum over ranks is the gradient
        gdw, gw = O.adjoint(fs, f1[items], f2[items], cdw, -cdw * xi)
        gdw, gw = r.allreduce_sum(gdw, gw)
        if r.rank == 0:
            ho, _ = O.corr(fs, f1, f2, [0, len(f1)], nthreads=2)
            W1, DW1 = ho[0, O.Q_W], ho[0, O.Q_DW]
            xi1 = np.divide(DW1, W1, out=np.zeros_like(W1), where=W1 != 0)
            c1 = np.divide(g, W1, out=np.zeros_like(W1), where=W1 != 0)
            rdw, rw = O.adjoint(fs, f1, f2, c1, -c1 * xi1)
            sc = max(np.abs(rdw).max(), 1e-300)
            q.put((float(np.abs(gdw - rdw).max() / sc), float(np.abs(gw - rw).max() / max(np.abs(rw).max(), 1e-300)),
                   len(share)))
    finally:
        r.close()


def test_sharded_adjoint_gradient_reduction():
    """The adjoint over owner-pixel shares: each rank all-reduces its W and DW
    totals (2 x nb values) to form xi, scatters the gradient of its own pairs
    into both forests of each pair, and the all-reduced gradient vectors equal
    the single-process gradient (to FP64 rounding of the reordered sums)."""
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    mp.start_processes(_adjoint_worker, args=(2, port, q), nprocs=2, join=True, start_method='spawn')
    edw, ew, nshare = q.get(timeout=120)
    assert edw < 1e-12 and ew < 1e-12 and nshare > 0


def test_collective_backend_choice(monkeypatch):
    """NCCL only for a rank whose GPU exists; gloo when asked or when the rank's
    index is beyond the visible GPUs (two ranks on a one-GPU machine)."""
    import torch
    from lya2pcf_b200.ranks import use_nccl
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: True)
    monkeypatch.setattr(torch.cuda, 'device_count', lambda: 1)
    assert use_nccl({'LOCAL_RANK': '0'}) == (True, 0)
    assert use_nccl({'LOCAL_RANK': '1'}) == (False, 1)
    assert use_nccl({'LOCAL_RANK': '0', 'LYA2PCF_DIST_BACKEND': 'gloo'}) == (False, 0)
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: False)
    assert use_nccl({'LOCAL_RANK': '0'}) == (False, 0)
