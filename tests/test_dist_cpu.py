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


def _xsim_inputs():
    """A stochastic NLS on 8 points, 4 blocks of 3 trajectories, both check passes."""
    base = dict(dimensions=2, points=[4, 8], ranges=[0.5, 6.0], steps=2, ensembles=[3, 4, 1], noises=2,
                method="MP", checks=1, order=1)
    g = dict(base, deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.05*(w(1,:)+1i*w(2,:))",
             initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2", observe=["@(a,p) a.*conj(a)"])
    o = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.05 * (w[0:1] + 1j * w[1:2]),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2,
             observe=[lambda a, p: a * np.conj(a)])
    return g, o


def _xsim_worker(rank, size, port, out):
    import importlib

    import torch.distributed as dist
    from tests.test_host_mirror_cpu import OraclePath
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        M = importlib.import_module("xspde_matlab_b200.xsim")
        g, o = _xsim_inputs()
        M.GpuPath = lambda p, path_kind=0, runtime_params=False: OraclePath(p, o)
        e, d, _ = M.xsim(g)
        if rank == 0:
            out.put((np.asarray(e), [np.asarray(x) for x in d[0]]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_xsim_with_oracle_blocks_matches_oracle_xsim():
    """The whole host xsim on two gloo ranks, each integrating its half of the
    blocks through the oracle's own p.path (Simulator/xpath.m) and one
    all-reduce of the moment sums (xsim.m:50-57, addcell): the error vector and
    data columns equal the oracle's single-process xsim (1e-10; the mirror's
    sums are compensated, the oracle's plain)."""
    import warnings

    from oracle import xspde_ref as X
    g, o = _xsim_inputs()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        eo, do, _ = X.xsim(o)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_xsim_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    eg, dg = q.get(timeout=300)
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    eo = np.asarray(eo)
    keep = [i for i in range(len(eo)) if i != 5]  # error(6) is the run time
    assert np.allclose(eg[keep], eo[keep], rtol=1e-10, atol=1e-15), (eg, eo)
    for a, b in zip(dg, do[0]):
        assert np.allclose(a, np.asarray(b), rtol=1e-10, atol=1e-13)


class FailingPath(FakePath):
    """A device path whose call fails on this rank, as a C-ABI error status raised
    by the host library does."""

    def run_path(self, first, nblocks, nc, a_in=None, a_out=False):
        raise RuntimeError("injected failure at block %d" % first)


def _fail_worker(rank, size, port, mode, out):
    import datetime
    import time

    import torch.distributed as dist
    from xspde_matlab_b200.dist import allreduce_sum
    from xspde_matlab_b200.xsim import _ensembles
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=20))
    inp = _inputs()
    if rank == 1 and mode == "exit":
        os._exit(3)  # leaves without reaching the reduction
    path = FailingPath(inp[0]) if rank == 1 else FakePath(inp[0])
    t0 = time.monotonic()
    try:
        _ensembles(inp, [path], rank, size, reduce=lambda a: allreduce_sum(a))
        out.put((rank, "ok", "", time.monotonic() - t0))
    except Exception as ex:
        out.put((rank, type(ex).__name__, str(ex), time.monotonic() - t0))
    if mode != "exit":
        dist.destroy_process_group()


def _run_failure(mode, nres):
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_fail_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    try:
        res = {}
        for _ in range(nres):
            r, kind, msg, dt = q.get(timeout=120)
            res[r] = (kind, msg, dt)
    finally:
        for pr in procs:
            pr.join(timeout=60)
            if pr.is_alive():
                pr.kill()
    return res, [pr.exitcode for pr in procs]


def test_failing_rank_is_reported_on_every_rank():
    """A rank whose device path raises still joins the moment reduction with a failure
    count: it re-raises its own error and its peer raises at the reduction, at once,
    instead of waiting there for the process-group timeout."""
    res, codes = _run_failure("raise", 2)
    assert res[1][0] == "RuntimeError" and "injected failure" in res[1][1]
    assert res[0][0] == "RuntimeError" and "1 of 2 ranks failed" in res[0][1]
    assert res[0][2] < 15
    assert codes == [0, 0]


def test_rank_that_leaves_ends_peers_reduction_with_error():
    """A rank that exits before the reduction: its peer's all-reduce ends with an
    error (closed connection or the short process-group timeout), not a hang."""
    res, codes = _run_failure("exit", 1)
    assert res[0][0] != "ok"
    assert res[0][2] < 60
    assert codes[1] == 3
