"""Ranks of the drop-in drivers: mpi4py when it is installed (as the
reference, ``2pla.py:13-22``), else ``torch.distributed`` when the process was
started by torchrun (``WORLD_SIZE`` > 1 in the environment; NCCL when the rank's
GPU exists, gloo otherwise or when ``LYA2PCF_DIST_BACKEND=gloo``), else one process.

The correlation needs no collective (owner pixels are disjoint; each rank
writes its own files).  The distortion needs one: :meth:`Ranks.reduce_sum`
adds the ranks' D (np*nt squared) and W_A to rank 0, which replaces
``comm.reduce`` of ``distortion.py:118-119``.  The adjoint over sharded owner
pixels needs two: :meth:`Ranks.allreduce_sum` of the W and DW totals (to form
xi on every rank) and of the per-pixel gradient vectors (a rank's pairs
scatter into forests of any pixel).
"""
import datetime
import os

import numpy as np


def use_nccl(env=None):
    """``(nccl, local_rank)`` for a torchrun rank: NCCL when the rank has a GPU
    of its own (``LOCAL_RANK`` below the visible GPU count); gloo (host memory)
    when it does not, or when ``LYA2PCF_DIST_BACKEND=gloo`` asks for it."""
    import torch
    env = os.environ if env is None else env
    local = int(env.get('LOCAL_RANK', '0'))
    nccl = (env.get('LYA2PCF_DIST_BACKEND', '') != 'gloo' and torch.cuda.is_available()
            and local < torch.cuda.device_count())
    return nccl, local


class Ranks:
    def __init__(self):
        self.comm, self.rank, self.size, self.torch_pg = None, 0, 1, False
        try:
            from mpi4py import MPI
            self.comm = MPI.COMM_WORLD
            self.rank, self.size = self.comm.Get_rank(), self.comm.Get_size()
            return
        except ImportError:
            pass
        if int(os.environ.get('WORLD_SIZE', '1')) > 1:
            import torch
            import torch.distributed as dist
            self.cuda, local = use_nccl()
            if self.cuda:
                torch.cuda.set_device(local)
            dist.init_process_group('nccl' if self.cuda else 'gloo', timeout=datetime.timedelta(seconds=300))
            self.rank, self.size, self.torch_pg = dist.get_rank(), dist.get_world_size(), True

    def reduce_sum(self, *arrays):
        """The element-wise sums of ``arrays`` over the ranks, on rank 0 (the
        other ranks get their own arrays back)."""
        if self.size == 1:
            return arrays
        if self.comm is not None:
            return tuple(self.comm.reduce(a) if self.rank == 0 else (self.comm.reduce(a), a)[1] for a in arrays)
        import torch
        import torch.distributed as dist
        out = []
        for a in arrays:
            t = torch.tensor(np.asarray(a, dtype=np.float64))   # a copy: the caller's array is not touched
            if self.cuda:
                t = t.cuda()
            dist.reduce(t, dst=0, op=dist.ReduceOp.SUM)
            out.append(t.cpu().numpy() if self.rank == 0 else a)
        return tuple(out)

    def allreduce_sum(self, *arrays):
        """The element-wise sums of ``arrays`` over the ranks, on every rank
        (float64 numpy arrays; the callers' arrays are not modified)."""
        if self.size == 1:
            return tuple(np.array(a, dtype=np.float64) for a in arrays)
        if self.comm is not None:
            return tuple(np.asarray(self.comm.allreduce(np.asarray(a, dtype=np.float64))) for a in arrays)
        import torch
        import torch.distributed as dist
        out = []
        for a in arrays:
            t = torch.tensor(np.asarray(a, dtype=np.float64))
            if self.cuda:
                t = t.cuda()
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            out.append(t.cpu().numpy())
        return tuple(out)

    def close(self):
        if self.torch_pg:
            import torch.distributed as dist
            dist.destroy_process_group()
            self.torch_pg = False
