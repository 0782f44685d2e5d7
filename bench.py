"""Benchmark: ensemble integration of the 2D stochastic GPE / CGL on one B200.

Workload (the reference's second configuration): 256x256 periodic lattice over
[-10,10]^2, da/dt = (i+0.1) lap a + (1-|a|^2) a - 0.5i |a|^2 a + 0.05 xi,
a0 = 1 + 0.1 complex Gaussian, 4096 trajectories (16 blocks of 256), MP with 4
iterations, 51 output points x 10 steps (509 integration steps, the xSPDE
path's own count), observable <|a|^2>(x, y, t).  FP32 fields and transforms,
FP64 propagator tables and moments.  Synthetic inputs: the initial field and
all noise come from the counter-based Philox stream (seed 0).

One "step" of this benchmark is one full p.path call over all 4096
trajectories.  value = trajectory-steps/s with everything resident in HBM
(field 2.1 GB > L2 every pass); e2e = the same through the host C ABI call
xs_run_path with a pinned FP64 initial field copied in and the block means
copied out inside the timed region.  The line also carries the same problem
in plain FP64 (`fp64`: value, e2e and roofline, the reference's own
precision), the oracle timed on the host (`cpu_baseline`), and each
observable's error against the FP64 oracle on identical noise over the whole
path at 256x256 (`precision_vs_oracle`).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) every rank integrates its own 16
blocks (global block ids rank*16 .. rank*16+15: weak scaling); the FP64 block
moments are summed over ranks with one NCCL all-reduce inside the timed
region.  --impl reference times the CPU restatement of the reference path
(the oracle; MATLAB itself is not available) on the host cores.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "traj-steps/s (2D 256x256 stochastic GPE, MP, 4096 trajectories)"
HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (read + write) per trajectory of the two streaming kernels in FP32
# (keyed by kernel kind and bytes per complex value), from one ncu --set full
# capture of a 512-trajectory case of this problem; a launch's traffic grows
# in proportion to the trajectories it processes, so bench lines scale these
# by the trajectory count.
NCU_TRAFFIC_PER_TRAJ = {("x_step", 8): (268598272 + 209662208) / 512.0, ("y_pass", 8): (268474880 + 213282816) / 512.0}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def _bf16_peak():
    """Dense BF16 tensor-core peak (TFLOP/s) for a kernel timed on its own: the burst figure."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                for nm, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _config(ntraj, world, method="MP"):
    return {"workload": "gpe_2d: 256x256 periodic, %d trajectories per GPU (%d blocks x 256), 51 points x 10 steps"
                        " = 509 %s steps, observable <|a|^2>(x,y,t)" % (ntraj, ntraj // 256, method),
            "global_batch": world * ntraj, "l2": "field 2.1 GB per pass > 126 MB L2 (no flush needed)",
            "parallelism": "dp%d (blocks per rank)" % world}


def _problem(ntraj=4096, method="MP"):
    from xspde_matlab_b200.problems import GPE_2D
    p = dict(GPE_2D, method=method)
    p["ensembles"] = [256, max(1, ntraj // 256), 1]
    return p


def _oracle_gpe(npoints, ntraj, observables):
    """The oracle's (FP64 NumPy restatement of the reference path) input for the
    256x256 problem with `npoints` output times, 10 steps between them, one
    block of `ntraj` trajectories; observables chosen by name."""
    import numpy as np
    obs = {"abs2": lambda a, q: abs(a) ** 2, "re": lambda a, q: np.real(a)}
    return dict(dimensions=3, points=[npoints, 256, 256], ranges=[0.1 * (npoints - 1), 20.0, 20.0], steps=10,
                ensembles=[ntraj, 1, 1], noises=2, method="MP", checks=0,
                deriv=lambda a, w, q: (1 - abs(a) ** 2) * a - 0.5j * abs(a) ** 2 * a
                + 0.05 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
                initial=lambda v, q: 1 + 0.1 * (v[0:1] + 1j * v[1:2]) / np.sqrt(2),
                linear=lambda q: (1j + 0.1) * (q.Dx ** 2 + q.Dy ** 2), observe=[obs[k] for k in observables])


def _oracle_path(o, block=0):
    """One p.path call of the oracle (Simulator/xpath.m:16-107 restated): the
    initial field, every MP step with its Philox noise and the observables at
    every output time.  Returns (seconds, trajectory-steps, av)."""
    import warnings

    import numpy as np
    from oracle import xspde_ref as X
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        q = X.xpreferences([o])[0].copy()
        t0 = time.perf_counter()
        q.block, q.seq = block, 0
        q.dtr = q.dt / q.steps[0]
        q.propagator, q.da = q.propfactor(q)
        v = q.randomgen(q)
        q.t = q.origins[0]
        a = X.fit(np.asarray(X.call_cells(q.initial, None, v, q), dtype=complex), q.ca)
        _, av, _ = q.path(a, 1, q)
        el = time.perf_counter() - t0
    steps = q.points[0] * q.steps[0] - 1
    return el, steps * q.ensembles[0], av


def _precision_vs_oracle(npoints=51, ntraj=2):
    """cpu_baseline and the FP64-oracle error of each observable.

    The oracle integrates `ntraj` trajectories of the benchmark problem over
    the whole path (509 MP steps, observables <|a|^2> and <Re a> at all 51
    output times) on one host core; that run is timed as the CPU baseline.
    The same trajectories (same Philox noise) run through the streaming
    kernels in FP32 (the benchmark's mode) and FP64, and each observable is
    compared with the oracle: max |GPU - oracle| / max |oracle| and the rms
    ratio, over all sites and times."""
    import numpy as np
    from xspde_matlab_b200 import GpuPath, xpreferences
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    secs, tsteps, av_o = _oracle_path(_oracle_gpe(npoints, ntraj, ("abs2", "re")))
    g = dict(_problem(ntraj), ensembles=[ntraj, 1, 1], points=[npoints, 256, 256],
             ranges=[0.1 * (npoints - 1), 20.0, 20.0], observe=["@(a,p) abs(a).^2", "@(a,p) real(a)"])
    errs = {}
    for prec in ("fp32", "fp64"):
        av_g, _ = GpuPath(xpreferences([dict(g, precision=prec)])[0], path_kind=2).run_path(0, 1, 1)
        for k, name in enumerate(("<|a|^2>(x,y,t)", "<Re a>(x,y,t)")):
            x, y = np.asarray(av_g[0][k]).ravel(), np.asarray(av_o[k]).ravel()
            d = np.abs(x - y)
            errs.setdefault(prec, {})[name] = {
                "max_rel": float(d.max() / np.abs(y).max()),
                "rms_rel": float(np.sqrt(np.mean(d ** 2)) / np.sqrt(np.mean(np.abs(y) ** 2)))}
    cpu = {"value": tsteps / secs, "unit": "traj-steps/s", "cores": 1, "kind": "port",
           "sample": "%d trajectories x %d MP steps of the 256x256 problem with <|a|^2> and <Re a> at %d output "
                     "times (FP64 NumPy oracle, 1 core, %.1f s)" % (ntraj, tsteps // ntraj, npoints, secs)}
    prec = {"reference": "FP64 oracle (CPU restatement of the reference path) on the same Philox noise",
            "trajectories": ntraj, "output_times": npoints, "steps": tsteps // ntraj,
            "bound_fp32": 1e-5, "fp32": errs["fp32"], "fp64": errs["fp64"]}
    return cpu, prec


def _reference_worker(args):
    npoints, ntraj = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    secs, tsteps, _ = _oracle_path(_oracle_gpe(npoints, ntraj, ("abs2",)))
    return tsteps, secs


def run_reference(args, rank, world):
    """--impl reference: the CPU restatement of the reference path on all host
    cores.  Each step every core runs one p.path of its own trajectories (the
    benchmark's problem, observables included) over a bounded stretch of the
    path; the step's value is the sum over cores of trajectory-steps per
    second of integration (process-pool dispatch excluded)."""
    import multiprocessing as mp
    if rank != 0:
        print("reference arm: rank %d has no work (rank 0 times the CPU reference)" % rank, file=sys.stderr)
        return
    cores = os.cpu_count() or 1
    npoints, ntraj = 4, 2  # 39 MP steps and 4 observations per trajectory, as the benchmark's 509 and 51
    per_step = []
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = pool.map(_reference_worker, [(npoints, ntraj)] * cores)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                per_step.append((sum(r[0] / r[1] for r in res), dt))
    value = statistics.mean(r for r, _ in per_step)
    ms = 1000 * statistics.mean(d for _, d in per_step)
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "traj-steps/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": dict(_config(4096, 1), parallelism="host processes (bounded sample per step)"),
        "same_config": False,
        "same_config_note": "same problem, lattice, step and observable; each core integrates %d trajectories over "
                            "%d output times (%d MP steps, observables at every output time as the GPU arm) instead "
                            "of 4096 trajectories over 51, so one step ends in seconds" % (
                                ntraj, npoints, npoints * 10 - 1),
        "cpu_baseline": {"value": value, "unit": "traj-steps/s", "cores": cores, "kind": "port",
                         "sample": "per core and step: one oracle p.path of %d trajectories x %d MP steps with "
                                   "<|a|^2> at %d output times of the 256x256 problem; MATLAB reference "
                                   "unavailable on this box (no MATLAB/Octave)" % (ntraj, npoints * 10 - 1, npoints)},
        "e2e": {"value": value, "unit": "traj-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _measure(p, args, rank, world, local_rank, steps, warmup, cxbytes):
    """Device-timed and end-to-end throughput of one precision mode.

    value: `steps` p.path calls over all of this rank's blocks through
    xs_run_path_device with the field resident in HBM, each followed by the
    device-side block moments (xs_block_moments, xensemble.m:98-101) and, with
    several ranks, their all-reduce; CUDA events on the launching stream,
    max over ranks.  e2e: the same calls through xs_run_path with a pinned
    FP64 host initial field copied in and the block means copied out."""
    import torch
    from xspde_matlab_b200 import GpuPath, _lib
    dist = None
    if world > 1:
        import torch.distributed as dist
    nb = p.ensembles[1] * p.ensembles[2]
    ntraj = nb * p.ensembles[0]
    steps_per_traj = p.points[0] * p.steps[0] - 1
    path = GpuPath(p)
    L = _lib.lib()
    n = p.points[0] * p.nspace  # complex means per block (one site observable)
    av = torch.zeros((nb, n, 2), dtype=torch.float64, device="cuda")
    moments = torch.zeros((2, n), dtype=torch.float64, device="cuda")
    first = rank * nb
    stream = torch.cuda.current_stream()
    st = ctypes.c_void_p(stream.cuda_stream)

    def one_step():
        _lib.check(L.xs_run_path_device(path.h, first, nb, 1, None, ctypes.c_void_p(av.data_ptr()), None, st))
        _lib.check(L.xs_block_moments(ctypes.c_void_p(av.data_ptr()), nb, n, 1.0 / (nb * world),
                                      ctypes.c_void_p(moments.data_ptr()), 0, st))
        if dist is not None:
            dist.all_reduce(moments)

    for _ in range(warmup):
        one_step()
    torch.cuda.synchronize()
    _lib.check(L.xs_sync(path.h))
    L.xs_set_kernel_timing(path.h, 1)
    L.xs_kernel_stats(path.h, 1, None, None)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local_rank) as clk:
        ev0.record(stream)
        for _ in range(steps):
            one_step()
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = ev0.elapsed_time(ev1) / steps
    nk = len(_lib.KERNEL_KINDS)
    kms = (ctypes.c_double * nk)()
    kl = (ctypes.c_longlong * nk)()
    _lib.check(L.xs_kernel_stats(path.h, 1, kms, kl))
    L.xs_set_kernel_timing(path.h, 0)
    _lib.check(L.xs_sync(path.h))
    clocks = clk.summary()
    t_max = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_max = float(t_max.item())
    value = world * ntraj * steps_per_traj / (ms_max / 1000.0)
    kinds = _lib.KERNEL_KINDS
    stats = {kinds[i]: {"launches": int(kl[i]), "ms": float(kms[i])} for i in range(nk) if kl[i]}
    # the block-moment kernel runs once per step, outside the handle's counters
    launches = sum(int(kl[i]) for i in range(nk)) + steps
    out = {"value": value, "ms_per_step": ms_max, "steps": steps, "warmup": warmup, "kernels": stats,
           "gpu_launches": launches, "clocks": clocks}
    if args.quick:
        return out
    # end to end through the host C ABI (pinned host buffers, copies inside the timed region)
    a_in = torch.empty((ntraj * p.nspace * 2,), dtype=torch.float64, pin_memory=True)
    g = torch.Generator().manual_seed(1)
    a_in.normal_(0.0, 0.1 / math.sqrt(2), generator=g)
    a_in[0::2] += 1.0
    av_host = torch.empty((nb * path.per_block,), dtype=torch.float64, pin_memory=True)
    e2e_steps = max(1, min(steps, 3))
    _lib.check(L.xs_run_path(path.h, first, nb, 1, ctypes.c_void_p(a_in.data_ptr()),
                             ctypes.c_void_p(av_host.data_ptr()), None))
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        _lib.check(L.xs_run_path(path.h, first, nb, 1, ctypes.c_void_p(a_in.data_ptr()),
                                 ctypes.c_void_p(av_host.data_ptr()), None))
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1000 / e2e_steps
    te = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    out["e2e"] = {"value": world * ntraj * steps_per_traj / (float(te.item()) / 1000.0), "unit": "traj-steps/s",
                  "h2d_bytes_per_step": int(a_in.numel() * 8), "d2h_bytes_per_step": int(av_host.numel() * 8),
                  "steps": e2e_steps}
    # roofline of the dominant kernel and of the whole step
    rk4 = p.method == "RK4"
    dom = max(("x_step", "y_pass", "rc_pass"), key=lambda k: stats.get(k, {"ms": 0})["ms"])
    if rk4:
        dom = "y_pass"  # RK4 row passes move two to four field passes each; the column pass two
    per_launch_ms = stats[dom]["ms"] / stats[dom]["launches"]
    if dom == "rc_pass":
        # one fused launch: the row pass of one half of the trajectories and the column pass of the
        # other half, each one read and one write of its half's field
        traj_per_launch = ntraj / 2.0
        alg_bytes = 2.0 * 2.0 * traj_per_launch * p.fields * p.nspace * cxbytes
    elif rk4:
        traj_per_launch = float(ntraj)  # every column pass covers all trajectories of one of the two fields
        alg_bytes = 2.0 * traj_per_launch * p.fields * p.nspace * cxbytes
    else:
        launches_per_pass = max(1, round(stats[dom]["launches"] / float(steps * steps_per_traj)))
        traj_per_launch = ntraj / launches_per_pass
        alg_bytes = 2.0 * traj_per_launch * p.fields * p.nspace * cxbytes  # read + write of the complex field
    achieved = alg_bytes / (per_launch_ms / 1000.0) / 1e9
    peak, kind = _peaks()
    tr = NCU_TRAFFIC_PER_TRAJ.get((dom, cxbytes))
    bstep = (16.0 if rk4 else 4.0) * p.fields * p.nspace * cxbytes
    out["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": achieved / peak, "peak_kind": kind, "traffic": (tr * traj_per_launch if tr else None),
                       "algorithmic_bytes_per_launch": alg_bytes, "trajectories_per_launch": traj_per_launch}
    out["step_roofline"] = {"bound": "hbm", "unit": "GB/s", "peak": peak,
                            "achieved": value / world * bstep / 1e9, "frac": value / world * bstep / 1e9 / peak,
                            "bytes_per_traj_step": bstep,
                            "note": ("whole RK4 step: four passes over two fields, each one read and one write"
                                     if rk4 else "whole MP step: two passes, each one read and one write of the field")}
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    from xspde_matlab_b200 import xpreferences
    torch.cuda.set_device(local_rank)
    p32 = xpreferences([_problem(args.ntraj, args.method)])[0]
    ntraj = p32.ensembles[0] * p32.ensembles[1] * p32.ensembles[2]
    m32 = _measure(p32, args, rank, world, local_rank, args.steps, args.warmup, 8)
    if args.quick or args.method != "MP":
        if rank == 0:
            out = {"quick": args.quick, "method": args.method, "value": m32["value"], "unit": "traj-steps/s",
                   "ms_per_step": m32["ms_per_step"], "kernels": m32["kernels"], "clocks": m32["clocks"],
                   "config": _config(ntraj, world, args.method)}
            for k in ("e2e", "roofline", "step_roofline"):
                if k in m32:
                    out[k] = m32[k]
            print(json.dumps(out))
        return
    torch.cuda.empty_cache()
    # plain FP64 (the reference's own precision, c128), fewer steps: one step takes ~4 s
    p64 = xpreferences([dict(_problem(args.ntraj), precision="fp64")])[0]
    m64 = _measure(p64, args, rank, world, local_rank, max(3, min(args.steps, 5)), max(3, min(args.warmup, 3)), 16)
    torch.cuda.empty_cache()
    if rank != 0:
        return
    cpu, prec = _precision_vs_oracle()
    fp64 = {k: m64[k] for k in ("value", "ms_per_step", "steps", "warmup", "e2e", "roofline", "step_roofline",
                                "kernels", "clocks")}
    fp64.update(unit="traj-steps/s", dtype="c128",
                note="plain FP64 fields, transforms, drift, tables and moments (the reference's precision)")
    line = {
        "metric": METRIC,
        "value": m32["value"], "unit": "traj-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": m32["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64", "precision_mode": "FP32 fields, transforms and drift; FP64 propagator tables and moments",
        "data": "synthetic (Philox initial field and noise, seed 0)",
        "config": _config(ntraj, world),
        "e2e": m32["e2e"],
        "gpu_launches": m32["gpu_launches"],
        "kernels": m32["kernels"],
        "roofline": m32["roofline"],
        "step_roofline": m32["step_roofline"],
        "cpu_baseline": cpu,
        "clocks": m32["clocks"],
        "fp64": fp64,
        "precision_vs_oracle": prec,
    }
    print(json.dumps(line))


# ---- second headline: time to 1e-3 relative sampling error on <|a|^2> ----------
CV_OBSERVE = "@(a,p) Int(abs(a).^2, p.dx, [0 0; -1.2 1.25; -1.2 1.25], p)"  # central 32x32 sites at t = 5
# Control-variate inputs: (region {i1lo, i2lo, bw, bh, nbx, nby}, steps per window,
# windows, steps between the window end and the observed step).  The 64x64
# sites around the centre: 8x8 blocks over the last 30 steps, then 4x4 blocks
# over four windows of 30 steps before that; 2 noise components each.
CV_SETS = (((96, 96, 8, 8, 8, 8), 30, 1, 0), ((96, 96, 16, 16, 4, 4), 30, 4, 30))
CV_FEATURES = sum(2 * nt * r[4] * r[5] for r, dw, nt, gap in CV_SETS)


def _cv_path(prec, nb):
    from xspde_matlab_b200 import GpuPath, xpreferences
    from xspde_matlab_b200.problems import GPE_2D
    p = dict(GPE_2D, precision=prec, ensembles=[1, nb, 1], observe=[CV_OBSERVE])
    return GpuPath(xpreferences([p])[0])


def _cv_solve(path, first, nb, feats=False):
    """Per-trajectory observable at the last output time (blocks of one
    trajectory) and, optionally, the noise features of the same trajectories."""
    import torch
    from xspde_matlab_b200 import _lib
    L = _lib.lib()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    av = torch.zeros((nb, path.p.points[0], 1, 2), dtype=torch.float64, device="cuda")
    _lib.check(L.xs_run_path_device(path.h, first, nb, 1, None, ctypes.c_void_p(av.data_ptr()), None, st))
    X = None
    if feats:
        X = torch.empty((nb, CV_FEATURES), dtype=torch.float32, device="cuda")
        last = (path.p.points[0] - 1) * path.p.steps[0]  # draw of the step observed at the last output
        col = 0
        for reg, dw, nt, gap in CV_SETS:
            nf = 2 * nt * reg[4] * reg[5]
            part = torch.empty((nb, nf), dtype=torch.float32, device="cuda")
            r = (ctypes.c_int * 6)(*reg)
            _lib.check(L.xs_noise_features(path.h, first, nb, r, last - gap - dw * nt + 1, dw, nt, 0.0,
                                           ctypes.c_void_p(part.data_ptr()), st))
            X[:, col:col + nf] = part
            col += nf
    _lib.check(L.xs_sync(path.h))  # surfaces device-side status (non-finite values, refused launches)
    return av[:, -1, 0, 0], X


def run_cv(args):
    """Second headline (cfg5): the learned control variate on the 256x256 GPE.

    Training: 2^16 + 8192 (noise features, observable) pairs generated by the FP32
    solver.  The control variate g is the best, on the 8192 held-out pairs, of linear
    least squares on the features, least squares on the features and their squares,
    and that plus the BF16 MLP (tcgen05 forward, trained by the project's kernels) on
    the residual.  Estimators, each timed on fresh trajectories:
      cfg5   N = 512 FP32 solves and M = 2^20 network evaluations on fresh inputs,
             mean_N(f - g) + mean_M(g), against the plain FP64 estimator with the
             trajectories that give it the same sampling error;
      1e-3   both at the trajectory counts their pilot variances need for 1e-3
             relative sampling error (xsim.m:95 block estimate).
    Times are reported with and without generating the training pairs and fitting."""
    import numpy as np
    import torch
    global CV_SETS, CV_FEATURES
    if args.cv_sets:
        CV_SETS = tuple((tuple(r), dw, nt, gap) for r, dw, nt, gap in json.loads(args.cv_sets))
        CV_FEATURES = sum(2 * nt * r[4] * r[5] for r, dw, nt, gap in CV_SETS)
    from xspde_matlab_b200.cv import ControlVariateNet, block_sampling_error, fresh_moments, two_level
    target = 1e-3
    nblk = 16
    ntrain, nval, chunk = args.cv_train, 8192, 8192
    p32 = _cv_path("fp32", chunk)
    t0 = time.perf_counter()
    fs, Xs = [], []
    for b0 in range(0, ntrain + nval, chunk):
        f, X = _cv_solve(p32, b0, chunk, feats=True)
        fs.append(f)
        Xs.append(X)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    f_all, X_all = torch.cat(fs), torch.cat(Xs)
    f_tr, X_tr, f_va, X_va = f_all[:ntrain], X_all[:ntrain], f_all[ntrain:], X_all[ntrain:]
    t0 = time.perf_counter()

    def lsq(feat):
        A = torch.cat([feat(X_tr).double(), torch.ones(ntrain, 1, dtype=torch.float64, device="cuda")], 1)
        c = torch.linalg.solve(A.T @ A, A.T @ f_tr.double().unsqueeze(1))[:, 0]
        w, b = c[:-1].float(), float(c[-1])
        return lambda X: (feat(X) @ w).double() + b  # FP32 dot, FP64 sum: same for solver and fresh inputs
    lin = lsq(lambda X: X)
    quad = lsq(lambda X: torch.cat([X, X * X], 1))
    var_plain = float(f_va.double().var())
    var_lin = float((f_va.double() - lin(X_va)).var())
    var_quad = float((f_va.double() - quad(X_va)).var())
    base, var_base = (quad, var_quad) if var_quad < var_lin else (lin, var_lin)
    net = ControlVariateNet(CV_FEATURES, 256, seed=0)
    r_tr = (f_tr.double() - base(X_tr)).float()
    r_va = f_va.double() - base(X_va)
    best = (var_base, None)
    for ep in range(20):
        net.fit(X_tr, r_tr, epochs=1, batch=1024, lr=3e-4 if ep > 9 else 1e-3, seed=ep, weight_decay=1e-2)
        v = float((r_va - net.predict(X_va)).var())
        if v < best[0]:
            best = (v, net.params.clone(), net.mean, net.scale)
    use_mlp = best[1] is not None
    if use_mlp:
        net.params.copy_(best[1])
        net.mean, net.scale = best[2], best[3]
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t0

    def g(X):
        return base(X) + (net.predict(X) if use_mlp else 0.0)
    var_cv = float((f_va.double() - g(X_va)).var())
    mu = float(f_va.double().mean())
    print("cv pilot: mean %.6g var_plain %.4g lin %.4g quad %.4g cv %.4g mlp %s" % (
        mu, var_plain, var_lin, var_quad, var_cv, use_mlp), file=sys.stderr)

    def time_cv(n, m, first):
        """N fresh FP32 solves with features + M fresh network inputs; returns (s, est, err, phases)."""
        pcv = _cv_path("fp32", n)
        _, Xw = _cv_solve(pcv, first + (1 << 22), n, feats=True)  # warm at the timed size
        g(Xw)
        gen = torch.Generator(device="cuda").manual_seed(777)
        fresh_moments(g(torch.randn((m, CV_FEATURES), device="cuda", generator=gen)))
        gen = torch.Generator(device="cuda").manual_seed(12345 + first)
        torch.cuda.synchronize()
        ta = time.perf_counter()
        f32, Xc = _cv_solve(pcv, first, n, feats=True)
        tb = time.perf_counter()
        gx = g(Xc)
        mom = fresh_moments(g(torch.randn((m, CV_FEATURES), device="cuda", generator=gen)))
        tc_ = time.perf_counter()
        est, err = two_level(f32.cpu().numpy(), gx.cpu().numpy(), mom, nblk)
        te = time.perf_counter()
        return te - ta, est, err, {"solve_and_features": tb - ta, "network_and_fresh_inputs": tc_ - tb,
                                   "estimate": te - tc_}, f32

    def time_plain(n, first):
        p64 = _cv_path("fp64", n)
        _cv_solve(p64, first + (1 << 22), n)  # compile and warm at the timed size
        torch.cuda.synchronize()
        ta = time.perf_counter()
        f64, _ = _cv_solve(p64, first, n)
        est, err = block_sampling_error(f64.cpu().numpy(), nblk)
        return time.perf_counter() - ta, est, err, f64

    m_fresh = 1 << 20
    # cfg5: N = 512, M = 2^20; the plain FP64 estimator at the same sampling error
    n5 = 512
    t5, est5, err5, ph5, f5 = time_cv(n5, m_fresh, 1 << 21)
    n5p = nblk * max(2, math.ceil(n5 * var_plain / var_cv / nblk))
    t5p, est5p, err5p, _ = time_plain(n5p, 1 << 20)
    # time to 1e-3 relative sampling error, each at the count its pilot variance needs
    n_plain = nblk * max(2, math.ceil(var_plain / (target * mu) ** 2 / nblk))
    n_cv = nblk * max(2, math.ceil(var_cv / (target * mu) ** 2 / nblk))
    t_plain, est_plain, err_plain, f64p = time_plain(n_plain, (1 << 20) + (1 << 19))
    t_cv, est_cv, err_cv, ph, f32c = time_cv(n_cv, m_fresh, (1 << 21) + (1 << 19))
    # FP32 trajectories against FP64 ones on identical noise
    ncmp = min(256, n_cv)
    f64b, _ = _cv_solve(_cv_path("fp64", ncmp), (1 << 21) + (1 << 19), ncmp)
    d32 = float(((f32c[:ncmp].double() - f64b) / f64b).abs().max())
    train = t_data + t_fit
    line = {
        "metric": "time to 1e-3 relative sampling error on <|a|^2> (central region, t=5)", "value": t_cv,
        "unit": "s", "higher_is_better": False, "n_gpus": 1,
        "plain_fp64": {"seconds": t_plain, "trajectories": n_plain, "estimate": est_plain,
                       "rel_sampling_error": err_plain / est_plain},
        "fp32_cv": {"seconds": t_cv, "seconds_with_training": t_cv + train, "trajectories": n_cv,
                    "fresh_network_inputs": m_fresh, "estimate": est_cv, "rel_sampling_error": err_cv / est_cv,
                    "seconds_by_phase": ph},
        "speedup_vs_plain_fp64": t_plain / t_cv,
        "speedup_with_training": t_plain / (t_cv + train),
        "cfg5_N512_M2p20": {"cv_seconds": t5, "cv_seconds_with_training": t5 + train, "cv_estimate": est5,
                            "cv_rel_sampling_error": err5 / est5, "cv_seconds_by_phase": ph5,
                            "plain_fp64_trajectories_same_error": n5p, "plain_fp64_seconds": t5p,
                            "plain_fp64_estimate": est5p, "plain_fp64_rel_sampling_error": err5p / est5p,
                            "speedup": t5p / t5, "speedup_with_training": t5p / (t5 + train)},
        "variance": {"plain": var_plain, "linear": var_lin, "linear_and_squares": var_quad,
                     "used": var_cv, "mlp_used": use_mlp, "mlp_on_residual_best": best[0],
                     "reduction_used": var_plain / var_cv,
                     "mlp_gain_over_least_squares": var_base / best[0]},
        "estimates_agree_sigma": abs(est_cv - est_plain) / math.sqrt(err_cv ** 2 + err_plain ** 2),
        "fp32_vs_fp64_traj_max_rel": d32,
        "training": {"pairs": ntrain, "validation_pairs": nval, "data_seconds": t_data, "fit_seconds": t_fit,
                     "features": "%d coarse space-time noise projections: %s" % (CV_FEATURES, CV_SETS)},
        "config": {"workload": "gpe_2d 256x256, 509 MP steps; sampling error from %d blocks (xsim.m:95)" % nblk},
    }
    print(json.dumps(line))


def run_mlp(args):
    """The control-variate network's inference on M fresh inputs (cfg5's M = 2^20 network
    evaluations): 256 inputs -> 256 x 3 (GELU) -> 1, hidden layers on the tcgen05 tensor
    cores with BF16 operands and FP32 accumulation.  One step = one xs_mlp_forward over
    all M rows (FP32 inputs resident in HBM)."""
    import numpy as np
    import torch
    from oracle import mlp_ref
    from xspde_matlab_b200 import _lib
    from xspde_matlab_b200.cv import ControlVariateNet
    L = _lib.lib()
    n_in, H, B = 256, 256, args.mlp_batch
    net = ControlVariateNet(n_in, H, seed=0)
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn((B, n_in), device="cuda", generator=g)
    work = torch.empty(L.xs_mlp_sizes(n_in, H, B, None), dtype=torch.float32, device="cuda")
    y = torch.empty(B, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    st = ctypes.c_void_p(stream.cuda_stream)

    def fwd():
        _lib.check(L.xs_mlp_forward(B, n_in, H, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(net.params.data_ptr()),
                                    ctypes.c_void_p(work.data_ptr()), ctypes.c_void_p(y.data_ptr()), st))
    for _ in range(max(3, args.warmup)):
        fwd()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(torch.cuda.current_device()) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            fwd()
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    flops = 2.0 * B * (n_in * H + 2 * H * H + H)
    # HBM bytes of the forward per row: FP32 inputs read, their BF16 copy written and read,
    # per hidden layer the BF16 activations read and written, the head's read and the output
    bytes_row = 4 * n_in + 2 * 2 * n_in + 3 * 2 * 2 * H + 2 * H + 4
    tf, tkind = _bf16_peak()
    hbm, hkind = _peaks()
    # CPU baseline: the FP64 NumPy network (oracle/mlp_ref.py) on a sample of rows
    P = net.params.cpu().numpy()
    Xs = X[:8192].cpu().numpy()
    t0 = time.perf_counter()
    ys, _, _ = mlp_ref.forward(Xs, P, n_in, H)
    cpu_s = time.perf_counter() - t0
    err = float(np.max(np.abs(y[:8192].cpu().numpy() - ys)) / np.max(np.abs(ys)))
    line = {"metric": "network evaluations/s, control-variate MLP 256-256x3-1 on fresh inputs", "value": B / (ms * 1e-3),
            "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
            "higher_is_better": True, "dtype": "bf16 operands, f32 accumulation", "data": "synthetic N(0,1) inputs",
            "tflops": flops / (ms * 1e-3) / 1e12,
            "roofline": {"bound": "hbm", "achieved": bytes_row * B / (ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": bytes_row * B / (ms * 1e-3) / 1e9 / hbm, "peak_kind": hkind,
                         "bytes_per_row": bytes_row, "traffic": None},
            "tensor": {"achieved_tflops": flops / (ms * 1e-3) / 1e12, "peak_tflops": tf, "peak_kind": tkind,
                       "frac": flops / (ms * 1e-3) / 1e12 / tf, "flops_per_row": flops / B},
            "max_rel_vs_fp64_oracle": err,
            "cpu_baseline": {"value": 8192 / cpu_s, "unit": "rows/s", "cores": 1, "kind": "port",
                             "sample": "8192 rows through the FP64 NumPy network (oracle/mlp_ref.py)"},
            "clocks": clk.summary(),
            "config": {"workload": "mlp 256->256x3->1, M=%d rows" % B}}
    print(json.dumps(line))


def run_batch(args):
    """Uneven batch: the instances of batch.uneven_instances (Philox seed 1) in
    one CUDA-graph launch with autotuned tiles.  A step is one launch of the
    whole batch; the metric counts every item's trajectory-steps."""
    import torch
    from xspde_matlab_b200 import batch as B
    inst = B.uneven_instances(args.batch_items, seed=1)
    t0 = time.perf_counter()
    b = B.Batch(inst, skip_unsupported=True)
    t_create = time.perf_counter() - t0
    t0 = time.perf_counter()
    b.tune(1)
    t_tune = time.perf_counter() - t0
    st = torch.cuda.Stream()
    t0 = time.perf_counter()
    b.run(st)
    st.synchronize()
    b.sync()
    t_first = time.perf_counter() - t0
    for _ in range(max(0, args.warmup - 1)):
        b.run(st)
    st.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(torch.cuda.current_device()) as clk:
        e0.record(st)
        for _ in range(args.steps):
            b.run(st)
        e1.record(st)
        e1.synchronize()
    b.sync()
    ms = e0.elapsed_time(e1) / args.steps
    done = [inst[k] for k in b.index]
    ts = sum(B.trajectory_steps(i) for i in done)
    sites = sum(B.trajectory_steps(i) * math.prod(i["points"][1:]) for i in done)
    ts_stream = sum(B.trajectory_steps(i) for i in done if i["points"][1:] == [256, 256])
    summ = b.summary()
    tiles = {}
    for i in range(len(b)):
        inf = b.info(i)
        if inf["path"] == 1:
            tiles[done[i]["name"]] = [inf["G"], inf["threads"], inf["ctas"]]
    line = {
        "metric": "traj-steps/s, uneven batch in one CUDA-graph launch", "value": ts / (ms * 1e-3),
        "unit": "traj-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "dtype": "f32 fields, f64 tables and moments", "data": "synthetic",
        "site_steps_per_s": sites / (ms * 1e-3), "items": summ["items"], "skipped_items": len(b.skipped),
        "skipped_reason": "the library rejected these inputs (xs_batch_create)" if b.skipped else None,
        "variants": summ["variants"], "streaming_items": summ["streaming"], "launches_per_step": summ["launches"],
        "stream_traj_step_share": ts_stream / ts, "tiles": tiles,
        "host_seconds": {"create": t_create, "tune": t_tune, "first_run_with_compile_and_capture": t_first},
        "clocks": clk.summary(),
        "config": {"workload": "uneven_instances(%d, seed=1): 1D N=32..1024 / 2D N=32..256, NLS or Allen-Cahn, "
                               "g~U[0.001,0.1], 50..2000 steps, 64..1024 trajectories, MP, FP32"
                               % args.batch_items},
    }
    print(json.dumps(line))


def _dpo_cpu_sample(seconds=10.0, ntraj=4096):
    """Oracle (FP64 NumPy, one core) on the DPO: `ntraj` trajectories for as
    many MP steps as fit in about `seconds`."""
    import numpy as np
    from oracle import xspde_ref as X
    from xspde_matlab_b200.problems import DPO_0D
    gam, eps, chi = 1.0, 1.25, 1e-3

    def deriv(a, w, q):
        a1, a2 = a[0:1], a[1:2]
        return np.concatenate([
            -gam * a1 + eps * a2 - chi * a1 ** 2 * a2 + 0.5 * chi * a1 + np.sqrt(-chi * a1 ** 2 + 0j) * w[0:1],
            -gam * a2 + eps * a1 - chi * a2 ** 2 * a1 + 0.5 * chi * a2 + np.sqrt(-chi * a2 ** 2 + 0j) * w[1:2]])
    o = {k: v for k, v in DPO_0D.items() if k not in ("deriv", "initial", "observe", "params")}
    o.update(ensembles=[ntraj, 1, 1], deriv=deriv, initial=lambda v, q: np.array([[1.0 + 0j], [1.0 + 0j]]),
             observe=[lambda a, q: np.real(a[0:1] * a[1:2])])
    q = X.xpreferences([o])[0].copy()
    q.block, q.seq = 0, 0
    q.dtr = q.dt / q.steps[0]
    q.propagator, q.da = q.propfactor(q)
    q.t = q.origins[0]
    a = X.fit(np.asarray(q.initial(0, q), dtype=complex), q.ca)
    method = X.METHODS["MP"]
    q.draw = 0
    t0 = time.perf_counter()
    steps = 0
    while time.perf_counter() - t0 < seconds:
        q.draw += 1
        a = method(a, q.noisegen(None, 1, q.nscale, q), q)
        q.t += q.dtr
        steps += 1
    el = time.perf_counter() - t0
    return steps * ntraj / el, "%d DPO trajectories x %d MP steps (FP64 NumPy oracle, 1 core)" % (ntraj, steps)


def run_ac3d(args):
    """3D stochastic Allen-Cahn 64^3 (Dirichlet/Neumann/mixed), FP32, 256
    trajectories, 99 MP steps: one p.path over all blocks per step.  Default:
    the 3D streaming path (plane and z-line passes over the field in HBM);
    --ac3d-path 1: the resident path with per-CTA device-memory slices."""
    import numpy as np
    import torch
    from xspde_matlab_b200 import GpuPath, _lib, xpreferences
    from xspde_matlab_b200.problems import AC_3D
    L = _lib.lib()
    blocks = max(1, args.ac3d_traj // AC_3D["ensembles"][0])
    p = xpreferences([dict(AC_3D, ensembles=[AC_3D["ensembles"][0], blocks, 1])])[0]
    g = GpuPath(p, path_kind=args.ac3d_path)
    nb = p.ensembles[1]
    av = torch.zeros((nb * g.per_block,), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()

    def run():
        _lib.check(L.xs_run_path_device(g.h, 0, nb, 1, None, ctypes.c_void_p(av.data_ptr()), None,
                                        ctypes.c_void_p(st.cuda_stream)))
    for _ in range(max(3, args.warmup)):
        run()
    torch.cuda.synchronize()
    _lib.check(L.xs_sync(g.h))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(torch.cuda.current_device()) as clk:
        e0.record(st)
        for _ in range(args.steps):
            run()
        e1.record(st)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    _lib.check(L.xs_sync(g.h))
    steps = p.points[0] * p.steps[0] - 1
    ntraj = nb * p.ensembles[0]
    # per-pass device times (events around every launch, one more path)
    nk = len(_lib.KERNEL_KINDS)
    kms = (ctypes.c_double * nk)()
    kl = (ctypes.c_longlong * nk)()
    L.xs_set_kernel_timing(g.h, 1)
    L.xs_kernel_stats(g.h, 1, None, None)
    run()
    torch.cuda.synchronize()
    _lib.check(L.xs_kernel_stats(g.h, 1, kms, kl))
    L.xs_set_kernel_timing(g.h, 0)
    kinds = _lib.KERNEL_KINDS
    stats = {kinds[i]: {"launches": int(kl[i]), "ms": float(kms[i])} for i in range(nk) if kl[i]}
    peak, peak_kind = _peaks()
    field_bytes = ntraj * p.nspace * 8  # complex FP32
    roof = None
    if g.kind == 3:
        # plane pass (x_step) and z-line pass (y_pass): each one read and one write of the field
        passes = {}
        for k in ("x_step", "y_pass"):
            per = stats[k]["ms"] / stats[k]["launches"]
            ach = 2.0 * field_bytes / (per * 1e-3) / 1e9
            passes[k] = {"ms_per_launch": per, "achieved": ach, "frac": ach / peak}
        dom = max(passes, key=lambda k: stats[k]["ms"])
        roof = {"bound": "hbm", "kernel": dom, "achieved": passes[dom]["achieved"], "peak": peak, "unit": "GB/s",
                "frac": passes[dom]["frac"], "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes_per_launch": 2.0 * field_bytes, "passes": passes,
                "step": {"bytes_per_traj_step": 4.0 * p.nspace * 8,
                         "achieved": ntraj * steps / (ms * 1e-3) * 4.0 * p.nspace * 8 / 1e9,
                         "frac": ntraj * steps / (ms * 1e-3) * 4.0 * p.nspace * 8 / 1e9 / peak}}
    # oracle sample: one trajectory for a few steps
    from oracle import xspde_ref as X
    o = {k: v for k, v in AC_3D.items() if k not in ("deriv", "initial", "linear", "observe", "precision")}
    o.update(ensembles=[1, 1, 1], deriv=lambda a, w, q: a - a ** 3 + 0.1 * w[0:1], initial=lambda v, q: 0.1 * v[0:1],
             linear=lambda q: 0.05 * (q.Dx ** 2 + q.Dy ** 2 + q.Dz ** 2), observe=[lambda a, q: abs(a) ** 2])
    q = X.xpreferences([o])[0].copy()
    q.block, q.seq = 0, 0
    q.dtr = q.dt / q.steps[0]
    q.propagator, q.da = q.propfactor(q)
    q.t = q.origins[0]
    a = X.fit(np.asarray(q.initial(q.randomgen(q), q), dtype=complex), q.ca)
    q.draw = 0
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < 10.0:
        q.draw += 1
        a = X.METHODS["MP"](a, q.noisegen(None, 1, q.nscale, q), q)
        n += 1
    cpu = n / (time.perf_counter() - t0)
    path = ("streaming 3D: plane passes (dense DST/DCT along x and y, MP step) and z-line passes "
            "(dense DST/DCT along z, FP64 propagator) over the field in HBM" if g.kind == 3 else
            "resident, field in per-CTA device-memory slices (dense DST/DCT matrices)")
    line = {"metric": "traj-steps/s, 3D stochastic Allen-Cahn 64^3 DST/DCT", "value": ntraj * steps / (ms * 1e-3),
            "unit": "traj-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f32 fields, f64 tables and moments", "data": "synthetic",
            "path": path, "kernels": stats, "roofline": roof,
            "cpu_baseline": {"value": cpu, "unit": "traj-steps/s", "cores": 1, "kind": "port",
                             "sample": "1 trajectory x %d MP steps (FP64 NumPy oracle)" % n},
            "clocks": clk.summary(),
            "config": {"workload": "ac_3d: 64^3, x Neumann (DCT-I), y Dirichlet (DST-I), z Neumann-Dirichlet (DCT-III/II), "
                                   "%d trajectories (%d blocks), 6 points x 20 steps = 99 MP steps; field %d MB "
                                   "(larger than L2)" % (ntraj, nb, field_bytes // 2 ** 20)}}
    print(json.dumps(line))


def run_snls(args):
    """1D stochastic NLS (64 points on [-5, 5], RK4, 51 x 4 = 200 steps to t = 1,
    1024 trajectories in 8 blocks, <|a|^2> and <Re a>): one p.path over all
    blocks per step, resident kernel (field and noise in shared memory).  FP64
    (the reference's c128) is the line's value, FP32 a sub-line; e2e through
    xs_run_path with a pinned host initial field; the CPU baseline is the FP64
    oracle's p.path over one block of 128 trajectories."""
    import numpy as np
    import torch
    from xspde_matlab_b200 import GpuPath, _lib, xpreferences
    from xspde_matlab_b200.problems import SNLS_1D
    L = _lib.lib()
    steps = SNLS_1D["points"][0] * SNLS_1D["steps"] - 1
    out = {}
    for prec in ("fp64", "fp32"):
        p = xpreferences([dict(SNLS_1D, precision=prec)])[0]
        g = GpuPath(p)
        nb = p.ensembles[1]
        ntraj = nb * p.ensembles[0]
        av = torch.zeros((nb * g.per_block,), dtype=torch.float64, device="cuda")
        st = torch.cuda.current_stream()

        def run():
            _lib.check(L.xs_run_path_device(g.h, 0, nb, 1, None, ctypes.c_void_p(av.data_ptr()), None,
                                            ctypes.c_void_p(st.cuda_stream)))
        for _ in range(max(3, args.warmup)):
            run()
        torch.cuda.synchronize()
        _lib.check(L.xs_sync(g.h))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        nrep = max(args.steps, 20)  # one path takes about a millisecond
        with Clocks(torch.cuda.current_device()) as clk:
            e0.record(st)
            for _ in range(nrep):
                run()
            e1.record(st)
            e1.synchronize()
        ms = e0.elapsed_time(e1) / nrep
        _lib.check(L.xs_sync(g.h))
        nk = len(_lib.KERNEL_KINDS)
        kms = (ctypes.c_double * nk)()
        kl = (ctypes.c_longlong * nk)()
        L.xs_set_kernel_timing(g.h, 1)
        L.xs_kernel_stats(g.h, 1, None, None)
        run()
        torch.cuda.synchronize()
        _lib.check(L.xs_kernel_stats(g.h, 1, kms, kl))
        L.xs_set_kernel_timing(g.h, 0)
        stats = {_lib.KERNEL_KINDS[i]: {"launches": int(kl[i]), "ms": float(kms[i])} for i in range(nk) if kl[i]}
        # end to end: pinned FP64 host initial field in, block means out, inside the timed region
        x = np.linspace(-5.0, 5.0, 64)
        a_in = torch.empty((ntraj * 64 * 2,), dtype=torch.float64, pin_memory=True)
        a_in.view(ntraj, 64, 2)[:, :, 0] = torch.from_numpy(np.exp(-x ** 2))[None, :]
        a_in.view(ntraj, 64, 2)[:, :, 1] = 0.0
        av_host = torch.empty((nb * g.per_block,), dtype=torch.float64, pin_memory=True)
        for _ in range(2):
            _lib.check(L.xs_run_path(g.h, 0, nb, 1, ctypes.c_void_p(a_in.data_ptr()),
                                     ctypes.c_void_p(av_host.data_ptr()), None))
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(st)
        for _ in range(nrep):
            _lib.check(L.xs_run_path(g.h, 0, nb, 1, ctypes.c_void_p(a_in.data_ptr()),
                                     ctypes.c_void_p(av_host.data_ptr()), None))
        t1.record(st)
        t1.synchronize()
        ems = t0.elapsed_time(t1) / nrep
        cx = 16 if prec == "fp64" else 8
        alg = ntraj * 64 * 16 + nb * g.per_block * 8  # field in (FP64), block means out
        out[prec] = {"value": ntraj * steps / (ms * 1e-3), "ms_per_step": ms, "steps": nrep,
                     "kernels": stats, "clocks": clk.summary(),
                     "e2e": {"value": ntraj * steps / (ems * 1e-3), "unit": "traj-steps/s",
                             "h2d_bytes_per_step": int(a_in.numel() * 8), "d2h_bytes_per_step": int(av_host.numel() * 8)},
                     "roofline": {"bound": "hbm", "kernel": "resident", "unit": "GB/s",
                                  "achieved": alg / (stats["resident"]["ms"] / stats["resident"]["launches"] * 1e-3) / 1e9,
                                  "peak": _peaks()[0], "peak_kind": _peaks()[1],
                                  "note": "the field (%d B per site) and noise stay in shared memory for the whole "
                                          "path: HBM carries only the initial field and the block means, so this "
                                          "kernel is bound by FP%d arithmetic and latency, not by HBM" % (cx, 64 if cx == 16 else 32)}}
        out[prec]["roofline"]["frac"] = out[prec]["roofline"]["achieved"] / out[prec]["roofline"]["peak"]
    # CPU baseline: the oracle's p.path over one block (128 trajectories, FP64 NumPy, one core)
    from oracle import xspde_ref as X
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    o = dict(SNLS_1D)
    o.update(deriv=lambda a, w, q: 1j * a * np.conj(a) * a + 0.01 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, q: np.exp(-q.x ** 2), linear=lambda q: 1j * q.Dx ** 2,
             observe=[lambda a, q: a * np.conj(a), lambda a, q: np.real(a)])
    q = X.xpreferences([o])[0].copy()
    q.block, q.seq = 0, 0
    q.dtr = q.dt / q.steps[0]
    q.propagator, q.da = q.propfactor(q)
    q.t = q.origins[0]
    a = X.fit(np.asarray(X.call_cells(q.initial, None, q.randomgen(q), q), dtype=complex), q.ca)
    t0 = time.perf_counter()
    q.path(a, 1, q)
    secs = time.perf_counter() - t0
    m = out["fp64"]
    line = {"metric": "traj-steps/s, 1D stochastic NLS (64 points, RK4)", "value": m["value"], "unit": "traj-steps/s",
            "n_gpus": 1, "steps": m["steps"], "warmup": max(3, args.warmup), "ms_per_step": m["ms_per_step"],
            "higher_is_better": True, "dtype": "c128", "data": "synthetic (Philox noise, seed 0)",
            "path": "resident: one CTA per trajectory tile, field and noise in shared memory for all 200 RK4 steps",
            "e2e": m["e2e"], "kernels": m["kernels"], "roofline": m["roofline"], "clocks": m["clocks"],
            "fp32": out["fp32"],
            "cpu_baseline": {"value": 128 * steps / secs, "unit": "traj-steps/s", "cores": 1, "kind": "port",
                             "sample": "one block: 128 trajectories x %d RK4 steps with <|a|^2> and <Re a> at 51 "
                                       "output times (FP64 NumPy oracle, %.1f s)" % (steps, secs)},
            "config": {"workload": "snls_1d: 64 points on [-5, 5], RK4, 51 output times x 4 steps = 200 steps to t = 1, "
                                   "1024 trajectories (8 blocks of 128)"}}
    print(json.dumps(line))


def run_dpo(args):
    """Positive-P DPO (0-D, two complex fields): 8 blocks x 125000 trajectories,
    each block its own pump eps ~ U[0.5, 2], 2000 MP steps, as one batch (one
    graph launch); FP64 and FP32 fields, FP32 observables compared with FP64."""
    import numpy as np
    import torch
    from xspde_matlab_b200 import batch as B
    out = {}
    res = {}
    for prec in ("fp64", "fp32"):
        inst = B.dpo_instances(precision=prec)
        b = B.Batch(inst)
        b.tune(1)
        st = torch.cuda.Stream()
        for _ in range(max(1, args.warmup)):
            b.run(st)
        st.synchronize()
        b.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(torch.cuda.current_device()) as clk:
            e0.record(st)
            for _ in range(args.steps):
                b.run(st)
            e1.record(st)
            e1.synchronize()
        b.sync()
        ms = e0.elapsed_time(e1) / args.steps
        ts = sum(B.trajectory_steps(i) for i in inst)
        res[prec] = [b.results(i) for i in range(len(inst))]
        out[prec] = {"traj_steps_per_s": ts / (ms * 1e-3), "ms_per_run": ms, "tile": b.info(0),
                     "clocks": clk.summary()}
    d = 0.0
    for r64, r32 in zip(res["fp64"], res["fp32"]):
        for o64, o32 in zip(r64, r32):
            d = max(d, float(np.max(np.abs(o32 - o64)) / max(np.max(np.abs(o64)), 1e-300)))
    inst = B.dpo_instances()
    n_final = [float(np.real(r[0][0, -1])) for r in res["fp64"]]
    cpu, sample = _dpo_cpu_sample()
    line = {"metric": "traj-steps/s, positive-P DPO 10^6 trajectories x 2000 steps (one graph launch)",
            "value": out["fp64"]["traj_steps_per_s"], "unit": "traj-steps/s", "dtype": "f64", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "data": "synthetic",
            "fp64": out["fp64"], "fp32": out["fp32"], "fp32_vs_fp64_observables_max_rel": d,
            "eps": [i["params"]["eps"] for i in inst], "final_mean_photon_number": n_final,
            "cpu_baseline": {"value": cpu, "unit": "traj-steps/s", "cores": 1, "kind": "port", "sample": sample},
            "config": {"workload": "dpo_0d: gam=1, chi=1e-3, eps~U[0.5,2] per block (Philox seed 1), 8 blocks x "
                                   "125000 trajectories, 2000 MP steps to t=10, observables <Re(alpha beta)>, "
                                   "<Re alpha> at 11 times"}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ntraj", type=int, default=4096, help="trajectories per GPU (multiple of 256)")
    ap.add_argument("--quick", action="store_true", help="device timing only (no e2e, no CPU sample)")
    ap.add_argument("--method", default="MP", choices=["MP", "RK4"],
                    help="stepper of the 256x256 problem (RK4: FP32 line with e2e and roofline only)")
    ap.add_argument("--cv", action="store_true", help="second headline: time to 1e-3 sampling error, "
                                                      "plain FP64 vs FP32 + learned control variate")
    ap.add_argument("--cv-sets", default="", help="JSON list of noise-feature sets [[region6], steps, windows, gap]")
    ap.add_argument("--cv-train", type=int, default=1 << 16, help="solver-generated training pairs (multiple of 8192)")
    ap.add_argument("--batch", action="store_true", help="uneven batch of independent problems, one graph launch")
    ap.add_argument("--batch-items", type=int, default=512)
    ap.add_argument("--dpo", action="store_true", help="positive-P DPO, 10^6 trajectories x 2000 steps")
    ap.add_argument("--mlp", action="store_true", help="control-variate network inference on M fresh inputs")
    ap.add_argument("--mlp-batch", type=int, default=1 << 20)
    ap.add_argument("--snls", action="store_true", help="1D stochastic NLS, 64 points, 1024 trajectories, RK4")
    ap.add_argument("--ac3d", action="store_true", help="3D stochastic Allen-Cahn 64^3 with DST/DCT boundaries")
    ap.add_argument("--ac3d-traj", type=int, default=256, help="trajectories of --ac3d (multiple of 32)")
    ap.add_argument("--ac3d-path", type=int, default=0, help="--ac3d device path: 0 automatic (3D streaming), 1 resident")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.ac3d:
        import torch
        torch.cuda.set_device(local_rank)
        run_ac3d(args)
        return
    if args.snls:
        import torch
        torch.cuda.set_device(local_rank)
        run_snls(args)
        return
    if args.dpo:
        import torch
        torch.cuda.set_device(local_rank)
        run_dpo(args)
        return
    if args.batch:
        import torch
        torch.cuda.set_device(local_rank)
        run_batch(args)
        return
    if args.mlp:
        import torch
        torch.cuda.set_device(local_rank)
        run_mlp(args)
        return
    if args.cv:
        import torch
        torch.cuda.set_device(local_rank)
        run_cv(args)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
