"""Multi-process ensembles: the reference's parfor over ensemble blocks
(Simulator/xsim.m:50-57) as one process per GPU.

Blocks are independent (each has its own Philox key), so they are split into
contiguous ranges, one per rank, with no data exchange during integration.
The only collective is the sum of the per-rank FP64 moment accumulators,
addcell of Simulator/xsim.m:217-228, done as one all-reduce.
"""
import numpy as np


def world():
    """(rank, world size, group) of an initialised torch.distributed job, else (0, 1, None)."""
    try:
        import torch.distributed as dist
    except Exception:
        return 0, 1, None
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1, None
    return dist.get_rank(), dist.get_world_size(), dist.group.WORLD


def shard(nblocks, rank, size):
    """Contiguous block range [b0, b1) of `rank` among `size` ranks."""
    per, extra = divmod(nblocks, size)
    b0 = rank * per + min(rank, extra)
    return b0, b0 + per + (1 if rank < extra else 0)


def allreduce_sum(arrays, group=None, device=None):
    """Sum lists of FP64 arrays over the ranks in one all-reduce (in place)."""
    import torch
    import torch.distributed as dist
    flat = np.concatenate([np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in arrays])
    t = torch.from_numpy(flat)
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    flat = t.cpu().numpy()
    out, pos = [], 0
    for a in arrays:
        n = a.size
        out.append(flat[pos:pos + n].reshape(a.shape))
        pos += n
    return out
