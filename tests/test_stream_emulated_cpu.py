"""The 2D streaming kernels run on the CPU, without a GPU: the CUDA source the library generates
for a 256 x 256 periodic problem (row pass with the 256-point register FFT, column pass with the
FP64 propagator, observation passes) is compiled with g++ against the host emulation of
tests/test_resident_emulated_cpu.py, and the host's pass sequence of one p.path call (the
merged MP half steps and observation times of launch_stream in csrc/xs_capi.cpp, or its RK4
sequence) is replayed here.  The block means of both check passes equal the oracle's p.path on
the same Philox noise.
"""
import ctypes
import math
import os

import numpy as np
import pytest

from oracle import xspde_ref as X
from tests.gpu_util import oracle_block_av
from tests.test_resident_emulated_cpu import EMU, host_source

RUNNER = r"""// Grid launches of the streaming kernels: the CTAs in turn, each CTA's threads as coroutines.
#include <functional>
#include <string>
alignas(16) unsigned char xs_dsmem_storage[240 * 1024];
unsigned char* xs_dsmem_ptr = xs_dsmem_storage;
static std::function<void()> xs_emu_fn;
static std::vector<std::vector<char>> xs_emu_stacks;
static void xs_emu_entry() {
  xs_emu_fn();
  xs_emu_thr[xs_emu_cur].done = true;
  swapcontext(&xs_emu_thr[xs_emu_cur].ctx, &xs_emu_sched);
}
static unsigned xs_emu_smem = 0;  // exact dynamic shared memory of this launch (0: the static buffer)
static int xs_emu_grid(unsigned gx, unsigned gy, unsigned gz, unsigned nthr, std::function<void()> fn) {
  std::vector<unsigned char> exact(xs_emu_smem);
  xs_dsmem_ptr = xs_emu_smem ? exact.data() : xs_dsmem_storage;
  xs_emu_dyn = xs_emu_smem ? xs_emu_smem : (unsigned)sizeof xs_dsmem_storage;
  blockDim = xs_dim3{nthr, 1, 1};
  gridDim = xs_dim3{gx, gy, gz};
  xs_emu_fn = fn;
  if (xs_emu_stacks.size() < nthr) xs_emu_stacks.resize(nthr);
  for (auto& s : xs_emu_stacks)
    if (s.empty()) s.resize(1 << 17);
  for (unsigned z = 0; z < gz; ++z)
    for (unsigned y = 0; y < gy; ++y)
      for (unsigned x = 0; x < gx; ++x) {
        blockIdx = xs_dim3{x, y, z};
        std::memset(xs_dsmem_ptr, 0x7f, xs_emu_dyn);
        xs_emu_thr.assign(nthr, XsEmuThread());
        for (unsigned t = 0; t < nthr; ++t) {
          XsEmuThread& th = xs_emu_thr[t];
          getcontext(&th.ctx);
          th.ctx.uc_stack.ss_sp = xs_emu_stacks[t].data();
          th.ctx.uc_stack.ss_size = xs_emu_stacks[t].size();
          th.ctx.uc_link = nullptr;
          makecontext(&th.ctx, xs_emu_entry, 0);
        }
        std::vector<unsigned> ord;
        for (;;) {
          bool any = false;
          xs_emu_order(ord, nthr);
          for (unsigned q = 0; q < nthr; ++q) {
            const unsigned t = ord[q];
            XsEmuThread& th = xs_emu_thr[t];
            if (th.done || th.wait) continue;
            any = true;
            xs_emu_cur = (int)t;
            threadIdx = xs_dim3{t, 0, 0};
            swapcontext(&xs_emu_sched, &th.ctx);
          }
          int live = 0, at_cta = 0;
          for (auto& th : xs_emu_thr)
            if (!th.done) { ++live; at_cta += th.wait == 1; }
          if (!live) break;
          bool released = false;
          for (unsigned w = 0; w * 32 < nthr; ++w) {
            int n = 0, m = 0;
            for (unsigned l = w * 32; l < w * 32 + 32 && l < nthr; ++l)
              if (!xs_emu_thr[l].done) { ++n; m += xs_emu_thr[l].wait == 2; }
            if (n && m == n) {
              for (unsigned l = w * 32; l < w * 32 + 32 && l < nthr; ++l) xs_emu_thr[l].wait = 0;
              released = true;
            }
          }
          if (!released && at_cta == live) {
            for (auto& th : xs_emu_thr) th.wait = 0;
            released = true;
          }
          if (!released && !any) return -1;
        }
      }
  return 0;
}
extern "C" int emu_launch(const char* name, unsigned gx, unsigned gy, unsigned gz, unsigned nthr,
                          const XsStreamArgs* A, int extra, unsigned smem) {
  xs_emu_smem = smem;
  const std::string n(name);
  const XsStreamArgs a = *A;
  if (n == "xs_x_init") return xs_emu_grid(gx, gy, gz, nthr, [a] { xs_x_init(a); });
  if (n == "xs_x_nl") return xs_emu_grid(gx, gy, gz, nthr, [a] { xs_x_nl(a); });
  if (n == "xs_x_final") return xs_emu_grid(gx, gy, gz, nthr, [a] { xs_x_final(a); });
  if (n == "xs_s_pass") return xs_emu_grid(gx, gy, gz, nthr, [a] { xs_s_pass(a); });
  if (n == "xs_x_obs") return xs_emu_grid(gx, gy, gz, nthr, [a] { xs_x_obs(a); });
  if (n == "xs_x_obs_combine") return xs_emu_grid(gx, gy, gz, nthr, [a, extra] { xs_x_obs_combine(a, extra); });
  if (n == "xs_stream_scalar") return xs_emu_grid(gx, gy, gz, nthr, [a] { xs_stream_scalar(a); });
  if (n == "xs_x_rk1") return xs_emu_grid(gx, gy, gz, nthr, [a] { xs_x_rk1(a); });
  if (n == "xs_x_rk2") return xs_emu_grid(gx, gy, gz, nthr, [a] { xs_x_rk2(a); });
  if (n == "xs_x_rk3") return xs_emu_grid(gx, gy, gz, nthr, [a] { xs_x_rk3(a); });
  return -2;
}
extern "C" int emu_sizes(int* out) {
  out[0] = XS_RX; out[1] = XS_RY; out[2] = XS_XROWS; out[3] = XS_TX; out[4] = XS_OROWS; out[5] = XS_OBS_STRIDE;
  out[6] = (int)sizeof(XsStreamArgs); out[7] = XS_NRG;
  return 0;
}
"""

V = ctypes.c_void_p


class StreamArgs(ctypes.Structure):
    """XsStreamArgs of csrc/kernels/xs_stream_common.cuh, field for field."""
    _fields_ = [("ntraj", ctypes.c_int), ("ens1", ctypes.c_int), ("block0", ctypes.c_int), ("seq", ctypes.c_int),
                ("seed", ctypes.c_uint), ("draw0", ctypes.c_int), ("draw1", ctypes.c_int), ("m", ctypes.c_int),
                ("n", ctypes.c_int), ("npoints", ctypes.c_int), ("wscale", ctypes.c_double),
                ("vscale", ctypes.c_double), ("dtr", ctypes.c_double), ("t", ctypes.c_double), ("field", V),
                ("prop1", V), ("prop2", V), ("a_in", V), ("a_out", V), ("av", V), ("redpart", V), ("status", V),
                ("params", V), ("tw_x", V), ("tw_y", V), ("opart", V), ("field2", V), ("ndraw0", ctypes.c_int),
                ("ndraw1", ctypes.c_int), ("fuse", ctypes.c_int), ("mat", V), ("xspace", ctypes.c_int)]


GPE = dict(dimensions=3, points=[3, 256, 256], ranges=[0.02, 20.0, 20.0], steps=2, ensembles=[2, 1, 1], noises=2,
           checks=1, order=1)


def _problems(method, precision):
    g = dict(GPE, method=method, precision=precision,
             deriv="@(a,w,p) (1-abs(a).^2).*a - 0.5i*abs(a).^2.*a + 0.05*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) 1 + 0.1*(v(1,:)+1i*v(2,:))/sqrt(2)", linear="@(p) (1i+0.1)*(p.Dx.^2+p.Dy.^2)",
             observe=["@(a,p) abs(a).^2", "@(a,p) Int(abs(a).^2, p)"])
    o = dict(GPE, method=method,
             deriv=lambda a, w, p: (1 - abs(a) ** 2) * a - 0.5j * abs(a) ** 2 * a + 0.05 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: 1 + 0.1 * (v[0:1] + 1j * v[1:2]) / np.sqrt(2),
             linear=lambda p: (1j + 0.1) * (p.Dx ** 2 + p.Dy ** 2),
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: X.Int(abs(a) ** 2, p)])
    return g, o


class StreamEmulated:
    def __init__(self, tmp, g, asan=False):
        import subprocess
        from xspde_matlab_b200 import _lib
        from xspde_matlab_b200.xsim import make_problem, xpreferences
        tmp.mkdir(parents=True, exist_ok=True)
        old = os.environ.get("XSPDE_B200_DUMP"), os.environ.get("XSPDE_B200_CACHE")
        os.environ["XSPDE_B200_DUMP"] = str(tmp / "dump")
        os.environ["XSPDE_B200_CACHE"] = str(tmp / "cache")
        try:
            q = xpreferences([g])[0]
            pr, keep = make_problem(q, path_kind=2)
            log = ctypes.create_string_buffer(1 << 16)
            _lib.check(_lib.lib().xs_compile_check(ctypes.byref(pr), log, len(log)))
        finally:
            for k, v in zip(("XSPDE_B200_DUMP", "XSPDE_B200_CACHE"), old):
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        srcs = [open(tmp / "dump" / f).read() for f in os.listdir(tmp / "dump") if f.startswith("xs_stream")]
        assert len(srcs) == 1
        self.fp64 = "#define XS_FP64 1" in srcs[0]
        cpp = tmp / "emu.cpp"
        cpp.write_text(EMU + host_source(srcs[0]) + RUNNER)
        so = tmp / "emu.so"
        flags = ["-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer"] if asan else ["-O2"]
        subprocess.run(["g++"] + flags + ["-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-o", str(so), str(cpp)],
                       check=True, capture_output=True, text=True)
        self.lib = ctypes.CDLL(str(so))
        self.lib.emu_launch.argtypes = [ctypes.c_char_p] + [ctypes.c_uint] * 4 + [V, ctypes.c_int, ctypes.c_uint]
        sz = (ctypes.c_int * 8)()
        self.lib.emu_sizes(sz)
        self.RX, self.RY, self.XROWS, self.TX, self.OROWS, self.stride, size, self.NRG = list(sz)
        assert ctypes.sizeof(StreamArgs) == size

    def block_means(self, o, block, nc):
        """Block means [points(1)][row] of one block and check pass (launch_stream's sequence)."""
        p = X.xpreferences([o])[0]
        P1, S, E1, checks = p.points[0], p.steps[0], p.ensembles[0], p.checks[0]
        N1, N2 = p.points[1], p.points[2]
        NS = N1 * N2
        real = np.float64 if self.fp64 else np.float32
        a = StreamArgs()
        a.ntraj, a.ens1, a.block0, a.seq, a.seed = E1, E1, block, 0, p.seed & 0xFFFFFFFF
        a.draw0, a.draw1, a.npoints = 0, -1, P1
        a.wscale, a.vscale = math.sqrt(p.nscale * p.noisefactor), math.sqrt(p.noisefactor)
        a.dtr = p.dt / (2 * S) if (checks and nc != 2) else p.dt / S
        a.t = p.origins[0]
        keep = []

        def buf(shape, dtype=np.float64):
            x = np.zeros(shape, dtype=dtype)
            keep.append(x)
            return x.ctypes.data
        a.field = buf((E1 * NS, 2), real)
        a.field2 = buf((E1 * NS, 2), real)
        for name, mult in (("prop1", 1), ("prop2", 2)):  # separable FP64 tables e_x[kx], e_y[ky]
            # exp(mult L dtr / ipsteps): the oracle's propfactor for a pass step of mult dtr
            q = p.copy()
            q.dtr = mult * a.dtr
            pr, _ = q.propfactor(q)
            pr = np.asarray(pr).reshape(-1, order="F")[:NS].reshape(N1, N2, order="F")
            t = np.concatenate([pr[:, 0], pr[0, :] / pr[0, 0]])
            tab = np.ascontiguousarray(np.stack([t.real, t.imag], 1))
            keep.append(tab)
            setattr(a, name, tab.ctypes.data)
        av = np.zeros((1, P1, self.stride, 2))
        keep.append(av)
        a.av = av.ctypes.data
        a.redpart = buf((E1 * self.NRG * 4, 2))
        status = np.zeros(1, dtype=np.int32)
        a.status = status.ctypes.data
        tws = []
        for R in (self.RX, self.RY):  # four-step twiddles exp(-2 pi i t k / R^2), [k][t]
            k, t = np.meshgrid(np.arange(R), np.arange(R), indexing="ij")
            ang = -2 * np.pi * (t * k) / (R * R)
            tws.append(np.ascontiguousarray(np.stack([np.cos(ang).ravel(), np.sin(ang).ravel()], 1).astype(real)))
        keep += tws
        a.tw_x, a.tw_y = tws[0].ctypes.data, tws[1].ctypes.data
        a.opart = buf((4 * NS, 2))
        xgrid, sgrid = E1 * N2 // self.XROWS, E1 * (N1 // self.TX)
        # dynamic shared memory of each launch, as the host's StreamPlan sizes it
        cxs = 16 if self.fp64 else 8
        RX, RY = self.RX, self.RY
        xline = max(RX * RX, RX * (RX + 1))
        smem = {"xs_x_init": (2 * RX * RX + self.XROWS * xline) * cxs,
                "xs_s_pass": (2 * RY * RY + self.TX * RY * RY) * cxs,
                "xs_x_obs": (2 * RX * RX + self.OROWS * RX * (RX + 1)) * cxs,
                "xs_x_rk1": (2 * RX * RX + 2 * self.XROWS * xline) * cxs}
        smem["xs_x_nl"] = smem["xs_x_final"] = smem["xs_x_init"]
        smem["xs_x_rk2"] = smem["xs_x_rk3"] = smem["xs_x_rk1"]

        def launch(name, gx, gy=1, gz=1, nthr=256, extra=0, args=a):
            r = self.lib.emu_launch(name.encode(), gx, gy, gz, nthr, ctypes.byref(args), extra, smem.get(name, 0))
            assert r == 0, name

        def col(m):
            a.m = m
            launch("xs_s_pass", sgrid)

        def observe(n):
            a.n = n
            launch("xs_x_obs", self.NRG, 1, 4, self.OROWS * self.RX)
            launch("xs_x_obs_combine", (NS + 255) // 256, 1, 1, 256, 4)
            launch("xs_stream_scalar", 1, 1, 1, 256)

        ops = []  # (observe, n, draw0, draw1) as xpath.m:29-86 visits them
        draw, prev = 0, -1
        for n in range(P1):
            for step in range(S):
                if n > 0 or step > 0 or P1 == 1:
                    for chk in range(checks + 1):
                        draw += 1
                        if nc == 2 and checks and chk == 0:
                            prev = draw
                            continue
                        ops.append((False, 0, draw, prev if (nc == 2 and checks) else -1))
                if step == 0:
                    ops.append((True, n, 0, -1))
        launch("xs_x_init", xgrid)
        if o.get("method") == "RK4":
            b = StreamArgs.from_buffer_copy(a)
            done = False
            for i, (obs, n, d0, d1) in enumerate(ops):
                if obs:
                    observe(n)
                    continue
                a.draw0, a.draw1, a.fuse = d0, d1, 0

                def col_both():
                    a.m = 1
                    launch("xs_s_pass", sgrid)
                    ctypes.memmove(ctypes.byref(b), ctypes.byref(a), ctypes.sizeof(a))
                    b.field = a.field2
                    launch("xs_s_pass", sgrid, args=b)
                if not done:  # pass 1, unless the previous step's pass 3 did it
                    launch("xs_x_rk1", xgrid)
                col_both()
                launch("xs_x_rk2", xgrid)
                col_both()
                nxt = i + 1 < len(ops) and not ops[i + 1][0]
                a.fuse = 1 if nxt else 0
                if nxt:
                    a.ndraw0, a.ndraw1 = ops[i + 1][2], ops[i + 1][3]
                launch("xs_x_rk3", xgrid)
                done = nxt
                a.t += a.dtr
        else:
            pending = 0
            for obs, n, d0, d1 in ops:
                if obs:
                    if pending:
                        col(pending)
                    pending = 0
                    observe(n)
                    continue
                col(pending + 1)
                a.draw0, a.draw1 = d0, d1
                launch("xs_x_nl", xgrid)
                a.t += a.dtr
                pending = 1
        assert status[0] == 0
        return av[0, ..., 0] + 1j * av[0, ..., 1]


@pytest.mark.parametrize("method,precision,tol", [("MP", "fp64", 1e-13), ("MP", "fp32", 1e-5),
                                                  ("RK4", "fp64", 1e-13)])
def test_emulated_streaming_path_matches_oracle(tmp_path, method, precision, tol):
    """256 x 256 GPE, two trajectories, both check passes: <|a|^2> at every site and its
    integral at every output time against the oracle (FP64 1e-13, FP32 1e-5 relative)."""
    g, o = _problems(method, precision)
    emu = StreamEmulated(tmp_path, g)
    p = X.xpreferences([o])[0]
    NS = p.points[1] * p.points[2]
    for nc in (1, 2):
        got = emu.block_means(o, 0, nc)
        ref, _ = oracle_block_av(o, 0, nc)
        r0 = np.asarray(ref[0]).reshape(p.points[0], NS, order="F")
        r1 = np.asarray(ref[1]).reshape(-1)
        assert np.max(np.abs(got[:, :NS] - r0)) / np.max(np.abs(r0)) < tol, nc
        assert np.max(np.abs(got[:, NS] - r1)) / np.max(np.abs(r1)) < tol, nc


def test_emulated_streaming_passes_have_no_barrier_races(tmp_path):
    """Index order, reversed and fresh random orders of each CTA's threads between barriers give
    bit-identical block means through the row pass's warp-level transposes, the column pass and
    the observation passes (FP32 MP, coarse pass)."""
    g, o = _problems("MP", "fp32")
    emu = StreamEmulated(tmp_path, g)
    runs = []
    for kind in (0, 1, 7):
        emu.lib.emu_set_schedule(kind)
        runs.append(emu.block_means(o, 0, 2))
    emu.lib.emu_set_schedule(0)
    for r in runs[1:]:
        assert np.array_equal(r, runs[0])


ASAN_RUN = r"""
import pathlib, sys
from tests.test_stream_emulated_cpu import StreamEmulated, _problems
tmp = pathlib.Path(sys.argv[1])
# every problem is generated before the first emulated launch switches stacks
cases = [(StreamEmulated(tmp / m, _problems(m, "fp64")[0], asan=True), _problems(m, "fp64")[1], nc)
         for m, nc in (("MP", 2), ("RK4", 1))]
for emu, o, nc in cases:
    emu.block_means(o, 0, nc)
print("clean")
"""


def test_emulated_streaming_passes_stay_in_bounds(tmp_path):
    """Bounds checking without a GPU: the streaming kernels built with AddressSanitizer, each
    launch's dynamic shared memory exactly the host's StreamPlan size and every buffer exactly
    the host's, run the MP path (coarse pass) and the RK4 path (fine pass) without an out-of-bounds access."""
    import subprocess
    import sys
    libs = [subprocess.run(["g++", "-print-file-name=%s" % n], capture_output=True, text=True).stdout.strip()
            for n in ("libasan.so", "libstdc++.so")]
    if not all(x and os.path.exists(x) for x in libs):
        pytest.skip("no AddressSanitizer runtime")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, LD_PRELOAD=" ".join(os.path.realpath(x) for x in libs),
               ASAN_OPTIONS="detect_leaks=0:halt_on_error=1", PYTHONPATH=root)
    r = subprocess.run([sys.executable, "-c", ASAN_RUN, str(tmp_path)], cwd=root, env=env, capture_output=True,
                       text=True, timeout=1200)
    assert "ERROR: AddressSanitizer" not in r.stderr, r.stderr[-4000:]
    assert r.returncode == 0 and "clean" in r.stdout, r.stderr[-4000:]
