"""Multi-rank ensembles on CPU (gloo, world size 2): each rank integrates its
share of the blocks and the moment accumulators are summed with one
all-reduce.  The device path is replaced by a fake whose block means depend
only on the global block index, so the reduced moments must equal a
single-process run exactly."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from xspde_matlab_b200.dist import shard


class FakePath:
    """Stands in for GpuPath: av of block b is a fixed function of b."""

    def __init__(self, p):
        self.p = p
        self.obs = [(1, True)]
        self.per_block = 2 * p.points[0] * p.nspace
        self.calls = []

    def av_shapes(self):
        return [(1, self.p.points[0]) + tuple(self.p.space)]

    def run_path(self, first, nblocks, nc, a_in=None, a_out=False):
        self.calls.append((first, nblocks, nc))
        out = []
        for b in range(first, first + nblocks):
            shp = self.av_shapes()[0]
            base = np.arange(np.prod(shp)).reshape(shp) * 0.001
            out.append([base * (b + 1) + 0.5 * nc + 0j])
        return out, None


def _inputs():
    from xspde_matlab_b200.xsim import xpreferences
    p = dict(dimensions=2, points=[5, 8], ensembles=[4, 6, 1], checks=1, order=1,
             deriv="@(a,w,p) 0*a", observe=["@(a,p) a.*conj(a)"])
    inp = xpreferences([p])
    q = inp[0]
    q.gpoints = [[1, q.points[0], q.space[0], max(3, 1 + q.nchk)]]
    return inp


def test_shard_covers_all_blocks():
    for nb in (1, 5, 16, 17):
        for size in (1, 2, 3, 8):
            got = []
            for r in range(size):
                lo, hi = shard(nb, r, size)
                got += list(range(lo, hi))
            assert got == list(range(nb))


def _worker(rank, size, port, out):
    import torch.distributed as dist
    from xspde_matlab_b200.dist import allreduce_sum
    from xspde_matlab_b200.xsim import _ensembles
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        inp = _inputs()
        data = _ensembles(inp, [FakePath(inp[0])], rank, size, reduce=lambda a: allreduce_sum(a))
        if rank == 0:
            out.put(data[0][0])
    finally:
        dist.destroy_process_group()


def test_two_ranks_match_single_process():
    from xspde_matlab_b200.xsim import _ensembles
    inp = _inputs()
    ref = _ensembles(inp, [FakePath(inp[0])])[0][0]
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = q.get(timeout=120)
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    assert np.allclose(got, ref, rtol=0, atol=1e-12)


def test_compensated_moment_sums():
    """The moment accumulation over blocks keeps terms that a plain FP64 sum loses."""
    import numpy as np
    from xspde_matlab_b200.xsim import _kadd
    s = np.zeros(3)
    c = np.zeros(3)
    for x in (1e16, 1.0, -1e16, 1.0, 3.0, -3.0):
        _kadd(s, c, np.full(3, x))
    assert np.all(s + c == 2.0)
    plain = 0.0
    for x in (1e16, 1.0, -1e16, 1.0, 3.0, -3.0):
        plain += x
    assert plain != 2.0
