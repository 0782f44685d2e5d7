"""The resident kernel run on the CPU, without a GPU: the CUDA source the library generates
for a problem is compiled with g++ against a host emulation of the few CUDA constructs it uses.
Each CTA's threads are coroutines run by one OS thread and switched at every __syncthreads and
warp-level exchange, so barriers keep their CUDA semantics; shared memory starts filled with
garbage bytes.  The block means of whole paths (noise, check passes, steppers, auxiliary cells,
time spectra, compensated observable sums) are compared with the oracle's p.path on the same
Philox noise: the kernel's own arithmetic, independent of the GPU.
"""
import ctypes
import math
import os
import re
import subprocess
import warnings

import numpy as np
import pytest

from oracle import xspde_ref as X
from tests.gpu_util import oracle_block_av

EMU = r"""// Host emulation of the CUDA constructs the resident kernel uses: the threads of one CTA
// are coroutines (ucontext) run by one OS thread, switched at __syncthreads and at the
// warp-level exchanges, so a launch runs its CTAs one after another with exact barrier
// semantics.
#include <ucontext.h>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#define __device__
#define __forceinline__ inline
#define __restrict__
#define __global__
#define __launch_bounds__(...)
#define __align__(n) alignas(n)
#define __shared__ static
struct uint4 { unsigned x, y, z, w; };
inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { return uint4{x, y, z, w}; }
struct double2 { double x, y; };
inline double2 make_double2(double x, double y) { return double2{x, y}; }
struct int2 { int x, y; };
struct float2 { float x, y; };
struct alignas(16) float4 { float x, y, z, w; };
struct alignas(32) double4 { double x, y, z, w; };
#define __host__
struct xs_dim3 { unsigned x, y, z; };
static xs_dim3 threadIdx, blockIdx, blockDim, gridDim;
static unsigned xs_emu_dyn = 1u << 30;  // the launch's dynamic shared memory, as %dynamic_smem_size reads it

struct XsEmuThread {
  ucontext_t ctx;
  std::vector<char> stack;
  int wait = 0;  // 0 runnable, 1 at a CTA barrier, 2 at a warp barrier
  bool done = false;
};
static std::vector<XsEmuThread> xs_emu_thr;
// Order in which the scheduler runs the runnable threads of a CTA in each round: 0 by index,
// 1 reversed, otherwise a fresh pseudo-random permutation every round (xorshift32).  A kernel
// whose result depends on the order between two barriers has a race.
static unsigned xs_emu_sched_kind = 0, xs_emu_rng = 1;
extern "C" void emu_set_schedule(unsigned kind) {
  xs_emu_sched_kind = kind;
  xs_emu_rng = kind * 2654435761u + 12345u;
}
static void xs_emu_order(std::vector<unsigned>& ord, unsigned n) {
  ord.resize(n);
  for (unsigned i = 0; i < n; ++i) ord[i] = xs_emu_sched_kind == 1 ? n - 1 - i : i;
  if (xs_emu_sched_kind > 1)
    for (unsigned i = n - 1; i > 0; --i) {
      xs_emu_rng ^= xs_emu_rng << 13;
      xs_emu_rng ^= xs_emu_rng >> 17;
      xs_emu_rng ^= xs_emu_rng << 5;
      const unsigned j = xs_emu_rng % (i + 1);
      const unsigned tmp = ord[i];
      ord[i] = ord[j];
      ord[j] = tmp;
    }
}
static ucontext_t xs_emu_sched;
static int xs_emu_cur;
static inline void xs_emu_yield(int why) {
  xs_emu_thr[xs_emu_cur].wait = why;
  swapcontext(&xs_emu_thr[xs_emu_cur].ctx, &xs_emu_sched);
}
inline void __syncthreads() { xs_emu_yield(1); }
static int xs_emu_or;
inline int __syncthreads_or(int p) {
  if (p) xs_emu_or = 1;
  __syncthreads();
  const int r = xs_emu_or;
  __syncthreads();
  if (threadIdx.x == 0) xs_emu_or = 0;
  __syncthreads();
  return r;
}
inline void __syncwarp(unsigned = 0xffffffffu) { xs_emu_yield(2); }
static double xs_emu_wbuf[32][32];
inline double __shfl_xor_sync(unsigned, double v, int o) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  xs_emu_wbuf[w][l] = v;
  __syncwarp();
  const double r = xs_emu_wbuf[w][l ^ o];
  __syncwarp();
  return r;
}
inline void __threadfence() {}
inline int atomicOr(int* p, int v) { const int o = *p; *p = o | v; return o; }
inline int atomicAdd(int* p, int v) { const int o = *p; *p = o + v; return o; }
inline float atomicAdd(float* p, float v) { const float o = *p; *p = o + v; return o; }
template <class T> inline T __ldcg(const T* p) { return *p; }
inline size_t __cvta_generic_to_shared(const void* p) { return (size_t)p; }
inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
// separately rounded products (the device's __dmul_rn / __fmul_rn)
inline double __dmul_rn(double a, double b) { volatile double r = a * b; return r; }
inline float __fmul_rn(float a, float b) { volatile float r = a * b; return r; }
inline float __logf(float x) { return std::log(x); }
inline float __expf(float x) { return std::exp(x); }
inline void __sincosf(float x, float* s, float* c) { *s = std::sin(x); *c = std::cos(x); }
inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
inline void sincospi(double x, double* s, double* c) { *s = std::sin(M_PI * x); *c = std::cos(M_PI * x); }
inline void sincos(float x, float* s, float* c) { *s = std::sin(x); *c = std::cos(x); }
template <class T> inline T __ldg(const T* p) { return *p; }
using std::sqrt; using std::log; using std::exp; using std::sin; using std::cos; using std::tan; using std::sinh;
using std::cosh; using std::tanh; using std::atan; using std::atan2; using std::hypot; using std::fabs; using std::floor;
using std::ceil; using std::round; using std::trunc; using std::erf; using std::fmin; using std::fmax; using std::pow;
using std::copysign; using std::fma; using std::isfinite; using std::asin; using std::acos;
"""

RUNNER = r"""// One launch of xs_resident: the CTAs in turn, each as XS_THREADS coroutines.
#ifndef XS_EMU_SMEM_SLACK
#define XS_EMU_SMEM_SLACK 64
#endif
alignas(16) unsigned char xs_smem_storage[XS_SMEM_BYTES + XS_EMU_SMEM_SLACK];
static const XsPathArgs* xs_emu_args;
static void xs_emu_entry() {
  xs_resident(*xs_emu_args);
  xs_emu_thr[xs_emu_cur].done = true;
  swapcontext(&xs_emu_thr[xs_emu_cur].ctx, &xs_emu_sched);
}
extern "C" int emu_run(const XsPathArgs* P, int nctas) {
  xs_emu_dyn = XS_SMEM_BYTES;
  blockDim = xs_dim3{XS_THREADS, 1, 1};
  gridDim = xs_dim3{(unsigned)nctas, 1, 1};
  xs_emu_args = P;
  for (int c = 0; c < nctas; ++c) {
    blockIdx = xs_dim3{(unsigned)c, 0, 0};
    std::memset(xs_smem_storage, 0x7f, sizeof xs_smem_storage);  // shared memory starts as garbage
    xs_emu_thr.assign(XS_THREADS, XsEmuThread());
    for (int t = 0; t < XS_THREADS; ++t) {
      XsEmuThread& th = xs_emu_thr[t];
      th.stack.resize(1 << 18);
      getcontext(&th.ctx);
      th.ctx.uc_stack.ss_sp = th.stack.data();
      th.ctx.uc_stack.ss_size = th.stack.size();
      th.ctx.uc_link = nullptr;
      makecontext(&th.ctx, xs_emu_entry, 0);
    }
    std::vector<unsigned> ord;
    for (;;) {
      bool any = false;
      xs_emu_order(ord, XS_THREADS);
      for (unsigned q = 0; q < (unsigned)XS_THREADS; ++q) {
        const int t = (int)ord[q];
        XsEmuThread& th = xs_emu_thr[t];
        if (th.done || th.wait) continue;
        any = true;
        xs_emu_cur = t;
        threadIdx = xs_dim3{(unsigned)t, 0, 0};
        swapcontext(&xs_emu_sched, &th.ctx);
      }
      int live = 0, at_cta = 0;
      for (auto& th : xs_emu_thr)
        if (!th.done) { ++live; at_cta += th.wait == 1; }
      if (!live) break;
      bool released = false;
      for (int w = 0; w * 32 < XS_THREADS; ++w) {  // warps whose live lanes all wait at a warp barrier
        int n = 0, m = 0;
        for (int l = w * 32; l < w * 32 + 32 && l < XS_THREADS; ++l)
          if (!xs_emu_thr[l].done) { ++n; m += xs_emu_thr[l].wait == 2; }
        if (n && m == n) {
          for (int l = w * 32; l < w * 32 + 32 && l < XS_THREADS; ++l) xs_emu_thr[l].wait = 0;
          released = true;
        }
      }
      if (!released && at_cta == live) {
        for (auto& th : xs_emu_thr) th.wait = 0;
        released = true;
      }
      if (!released && !any) return -1;  // threads wait at different barriers: divergent barrier
    }
  }
  return 0;
}
extern "C" int emu_sizes(int* out) {
  out[0] = XS_G; out[1] = XS_THREADS; out[2] = XS_OBS_STRIDE; out[3] = (int)sizeof(XsPathArgs);
  return 0;
}
"""

V = ctypes.c_void_p


class PathArgs(ctypes.Structure):
    """XsPathArgs of csrc/kernels/xs_resident.cuh, field for field."""
    _fields_ = [("ntraj", ctypes.c_int), ("ens1", ctypes.c_int), ("block0", ctypes.c_int), ("nc", ctypes.c_int),
                ("checks", ctypes.c_int), ("npoints", ctypes.c_int), ("steps", ctypes.c_int), ("seq", ctypes.c_int),
                ("seed", ctypes.c_uint), ("pad0", ctypes.c_int), ("wscale", ctypes.c_double),
                ("vscale", ctypes.c_double), ("dtr", ctypes.c_double), ("t0", ctypes.c_double), ("prop", V),
                ("tmat", V), ("tmat_off", ctypes.c_int * 4), ("a_in", V), ("a_out", V), ("obs", V), ("status", V),
                ("single_step", ctypes.c_int), ("pad1", ctypes.c_int), ("w_in", V), ("params", V), ("gfield", V),
                ("prop2", V), ("bval", V), ("bda", V), ("bval_n", ctypes.c_int), ("pad3", ctypes.c_int),
                ("aft", V), ("twt", V), ("nt", ctypes.c_int), ("pad4", ctypes.c_int), ("fscn", ctypes.c_double),
                ("raw", V), ("kfilt", V), ("rfilt", V), ("kwscale", ctypes.c_double), ("kvscale", ctypes.c_double)]


def host_source(src):
    """The generated CUDA source made host C++: the dynamic shared-memory size query reads the
    emulated launch's size and every other inline-asm statement becomes an empty statement
    (they serve the cp.async, mbarrier and TMA paths of device-memory lattices, the TMA column
    pass and the 3D passes, which these tests do not take); the dynamic shared-memory arrays
    become the emulator's buffers."""
    out, i = [], 0
    while True:
        j = src.find("asm volatile(", i)
        if j < 0:
            out.append(src[i:])
            break
        out.append(src[i:j])
        k, depth, instr = j + len("asm volatile("), 1, False
        while depth:
            c = src[k]
            if instr:
                if c == "\\":
                    k += 1
                elif c == '"':
                    instr = False
            elif c == '"':
                instr = True
            elif c == "(":
                depth += 1
            elif c == ")":
                depth -= 1
            k += 1
        while src[k] != ";":
            k += 1
        stmt = src[j:k]
        if "dynamic_smem_size" in stmt:
            out.append("dyn = xs_emu_dyn;")
        else:
            out.append(";")
        i = k + 1
    src = "".join(out)
    src = src.replace("extern __shared__ __align__(16) unsigned char xs_smem[];",
                      "extern unsigned char xs_smem_storage[];\n#define xs_smem xs_smem_storage")
    src = src.replace("extern __shared__ __align__(16) unsigned char xs_dsmem[];",
                      "extern unsigned char* xs_dsmem_ptr;\n#define xs_dsmem xs_dsmem_ptr")
    return src.replace("__grid_constant__", "")


class Emulated:
    """The resident kernel of one 0-D problem (no lattice, no linear term), compiled for the host."""

    def __init__(self, tmp, g, patch=None, asan=False):
        from xspde_matlab_b200 import _lib
        from xspde_matlab_b200.xsim import make_problem, xpreferences
        tmp.mkdir(parents=True, exist_ok=True)
        old = os.environ.get("XSPDE_B200_DUMP"), os.environ.get("XSPDE_B200_CACHE")
        os.environ["XSPDE_B200_DUMP"] = str(tmp / "dump")
        os.environ["XSPDE_B200_CACHE"] = str(tmp / "cache")
        try:
            q = xpreferences([g])[0]
            pr, keep = make_problem(q)
            log = ctypes.create_string_buffer(1 << 16)
            _lib.check(_lib.lib().xs_compile_check(ctypes.byref(pr), log, len(log)))
        finally:
            for k, v in zip(("XSPDE_B200_DUMP", "XSPDE_B200_CACHE"), old):
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        srcs = [open(tmp / "dump" / f).read() for f in os.listdir(tmp / "dump") if f.startswith("xs_resident")]
        assert len(srcs) == 1
        src = srcs[0]
        self.defs = {k: v for k, v in re.findall(r"#define (XS_\w+) (-?\d+)\s*$", src, re.M)}
        src = host_source(src)
        if patch is not None:
            src = patch(src)
        tmp.mkdir(parents=True, exist_ok=True)
        cpp = tmp / "emu.cpp"
        cpp.write_text(EMU + src + RUNNER)
        so = tmp / "emu.so"
        # with asan: AddressSanitizer, and shared memory exactly the launch's XS_SMEM_BYTES
        flags = ["-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer", "-DXS_EMU_SMEM_SLACK=0"] if asan else ["-O2"]
        subprocess.run(["g++"] + flags + ["-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-o", str(so), str(cpp)],
                       check=True, capture_output=True, text=True)
        self.lib = ctypes.CDLL(str(so))
        sz = (ctypes.c_int * 4)()
        self.lib.emu_sizes(sz)
        self.G, self.threads, self.stride, size = list(sz)
        assert ctypes.sizeof(PathArgs) == size

    def block_means(self, o, block, nc):
        """Block means [points(1)][row] of one ensemble block and check pass (xs_obs_reduce's
        sum over the block's CTAs, divided by ensembles(1))."""
        p = X.xpreferences([o])[0]
        P1, S, E1 = p.points[0], p.steps[0], p.ensembles[0]
        G = self.G
        assert E1 % G == 0
        nctas = E1 // G
        a = PathArgs()
        a.ntraj, a.ens1, a.block0, a.nc, a.checks = E1, E1, block, nc, p.checks[0]
        a.npoints, a.steps, a.seq, a.seed = P1, S, 0, p.seed & 0xFFFFFFFF
        a.wscale, a.vscale = math.sqrt(p.nscale * p.noisefactor), math.sqrt(p.noisefactor)
        a.dtr = p.dt / (2 * S) if (p.checks[0] and nc != 2) else p.dt / S
        a.t0 = p.origins[0]
        keep = []
        NS, PC = int(self.defs["XS_NS"]), int(self.defs["XS_PROP_COMPS"])
        if p.dimensions == 1 or not int(self.defs.get("XS_HAS_PROP", 0)):
            prop = np.zeros((PC * NS, 2))
            prop[:, 0] = 1  # exp(L dt) with L = 0
            keep.append(prop)
            a.prop = a.prop2 = prop.ctypes.data
        else:
            for name, mult in (("prop", 1), ("prop2", 2)):
                # exp(mult L dtr / ipsteps) on the k lattice, [components][sites], x fastest
                q = p.copy()
                q.dtr = mult * a.dtr
                pr, _ = q.propfactor(q)
                pr = np.asarray(pr, dtype=complex).reshape(-1, order="F")
                pr = np.broadcast_to(pr, (PC * NS,)) if pr.size == 1 else pr[:PC * NS]
                tab = np.ascontiguousarray(np.stack([pr.real, pr.imag], 1))
                keep.append(tab)
                setattr(a, name, tab.ctypes.data)
            # Stockham twiddles exp(-2 pi i m / n) of every FFT dimension, in dimension order
            tw, off = [], [0, 0, 0, 0]
            for d in range(p.dimensions - 1):
                off[d + 1] = len(tw)
                n = p.points[d + 1]
                assert int(self.defs.get("XS_FFTD%d" % (d + 1), 0)), "dense transforms are not emulated"
                tw += list(np.exp(-2j * np.pi * np.arange(n) / n))
            real = np.float64 if int(self.defs["XS_FP64"]) else np.float32
            tw = np.ascontiguousarray(np.stack([np.real(tw), np.imag(tw)], 1).astype(real))
            keep.append(tw)
            a.tmat = tw.ctypes.data
            for d in range(4):
                a.tmat_off[d] = off[d]
        obs = np.zeros((P1, nctas, self.stride, 2))
        a.obs = obs.ctypes.data
        status = np.zeros(1, dtype=np.int32)
        a.status = status.ctypes.data
        if int(self.defs.get("XS_SPEC", 0)):
            F, NS, NA = (int(self.defs[k]) for k in ("XS_F", "XS_NS", "XS_NA"))
            nt = P1 * S
            row = (1 + (NA + F - 1) // F) * G * F * NS
            real = np.float64 if int(self.defs["XS_FP64"]) else np.float32
            aft = np.zeros((nctas * (nt + P1) * row, 2), dtype=real)
            k = np.arange(nt)
            twt = np.ascontiguousarray(np.stack([np.cos(2 * np.pi * k / nt), np.sin(2 * np.pi * k / nt)], 1))
            keep += [aft, twt]
            a.aft, a.twt, a.nt = aft.ctypes.data, twt.ctypes.data, nt
            a.fscn = math.sqrt(2 * np.pi) / (2 * np.pi / (p.ranges[0] + p.dt)) / nt
        assert self.lib.emu_run(ctypes.byref(a), nctas) == 0
        assert status[0] == 0
        m = obs[..., 0] + 1j * obs[..., 1]
        return m.sum(axis=1) / E1


def _rel(got, ref):
    ref = np.asarray(ref).reshape(-1)
    return float(np.max(np.abs(got - ref)) / max(1.0, float(np.max(np.abs(ref)))))


def test_emulated_resident_kernel_quantum_auxiliary_spectra(tmp_path):
    """Examples/SDE_1D/Quantum.m (auxiliary input/output fields, time spectra, step-halving
    check with order 2): both passes of two blocks equal the oracle's block means to 1e-13,
    and the input field's spectrum is the same in both passes bit for bit, so its step
    error is exactly zero as in the reference."""
    from tests.test_host_mirror_cpu import _quantum
    g, o = _quantum()
    emu = Emulated(tmp_path, g)
    for b in (0, 7):
        means = {}
        for nc in (1, 2):
            got = emu.block_means(o, b, nc)
            ref, _ = oracle_block_av(o, b, nc)
            for k in range(4):
                assert _rel(got[:, k], ref[k]) < 1e-13, (b, nc, k)
            means[nc] = got
        assert np.array_equal(means[1][:, 1], means[2][:, 1])


def test_emulated_resident_kernel_positive_p_dpo(tmp_path):
    """The positive-P parametric oscillator (two fields, complex-sqrt multiplicative noise,
    Stratonovich-corrected drift, MP) against the oracle to 1e-12."""
    from xspde_matlab_b200.problems import DPO_0D
    base = dict(DPO_0D, ensembles=[64, 2, 1], points=[4], steps=15, ranges=[0.6], precision="fp64")
    gam, eps, chi = (base["params"][k] for k in ("gam", "eps", "chi"))

    def deriv(a, w, p):
        a1, a2 = a[0:1], a[1:2]
        return np.concatenate([
            -gam * a1 + eps * a2 - chi * a1 ** 2 * a2 + 0.5 * chi * a1 + np.sqrt(-chi * a1 ** 2 + 0j) * w[0:1],
            -gam * a2 + eps * a1 - chi * a2 ** 2 * a1 + 0.5 * chi * a2 + np.sqrt(-chi * a2 ** 2 + 0j) * w[1:2]])

    o = {k: v for k, v in base.items() if k not in ("deriv", "initial", "observe", "params", "precision")}
    o.update(deriv=deriv, initial=lambda v, p: np.array([[1.0 + 0j], [1.0 + 0j]]),
             observe=[lambda a, p: np.real(a[0:1] * a[1:2]), lambda a, p: np.real(a[0:1])])
    emu = Emulated(tmp_path, base)
    for b in (0, 1):
        got = emu.block_means(o, b, 1)
        ref, _ = oracle_block_av(o, b, 1)
        for k in range(2):
            assert _rel(got[:, k], ref[k]) < 1e-12, (b, k)


@pytest.mark.parametrize("method,precision,tol", [("RK4", "fp64", 1e-13), ("RK4", "fp32", 2e-5),
                                                  ("Euler", "fp64", 1e-13), ("RK2", "fp64", 1e-13)])
def test_emulated_resident_kernel_steppers_with_checks(tmp_path, method, precision, tol):
    """A driven damped oscillator with multiplicative noise through RK4, Euler and RK2 with the
    step-halving check (both passes), FP64 at 1e-13 and FP32 within its rounding."""
    base = dict(points=[6], ranges=[1.0], steps=4, ensembles=[32, 1, 1], noises=2, checks=1, order=1,
                method=method)
    g = dict(base, precision=precision, deriv="@(a,w,p) -(0.5+1i)*a + 0.3*a.*w(1,:) + 0.2i*w(2,:)",
             initial="@(v,p) 1 + 0.1*(v(1,:) + 1i*v(2,:))", observe=["@(a,p) abs(a).^2", "@(a,p) real(a)"])
    o = dict(base, deriv=lambda a, w, p: -(0.5 + 1j) * a + 0.3 * a * w[0:1] + 0.2j * w[1:2],
             initial=lambda v, p: 1 + 0.1 * (v[0:1] + 1j * v[1:2]),
             observe=[lambda a, p: abs(a) ** 2, lambda a, p: np.real(a)])
    emu = Emulated(tmp_path, g)
    for nc in (1, 2):
        got = emu.block_means(o, 0, nc)
        ref, _ = oracle_block_av(o, 0, nc)
        for k in range(2):
            assert _rel(got[:, k], ref[k]) < tol, (nc, k)


class EmulatedPath:
    """Stands in for GpuPath in the host xsim: p.path of each block from the emulated kernel
    (0-D problems whose observables are one line each)."""

    def __init__(self, emu, o):
        self.emu, self.o = emu, o
        q = X.xpreferences([o])[0]
        self.shapes = [tuple(s) for s in q.d_av]
        self.per_block = 2 * sum(int(np.prod(s)) for s in self.shapes)

    def av_shapes(self):
        return self.shapes

    def run_path(self, first, nblocks, nc, a_in=None, a_out=False, raw=False):
        av = []
        for b in range(first, first + nblocks):
            m = self.emu.block_means(self.o, b, nc)
            av.append([m[:, k].reshape(s, order="F") for k, s in enumerate(self.shapes)])
        return av, None


def _fused(src):
    """The coarse noise formed with a fused multiply-add, round(z2 s + round(z1 s)) / 2,
    as a compiler that contracts the product into the add produces it."""
    old = "W[j] = (v + Wp[j]) * (real)0.5;"
    assert old in src
    return src.replace(old, "W[j] = fma(z[c], (real)P.wscale, Wp[j]) * (real)0.5;")


def test_emulated_kernel_through_xsim_matches_oracle_error_vector(monkeypatch, tmp_path):
    """The Quantum example end to end: the host xsim over the emulated kernel's blocks gives the
    oracle's error vector (the assertion of the GPU test).  With the coarse noise fused into a
    multiply-add instead, the input field's spectrum differs between the passes in the last
    bit, its step error is counted, and the step-error entry becomes sqrt(3/4) of the oracle's
    with every data column unchanged (the GPU's result before the kernels rounded the two
    scaled draws separately: 1.03452598e-3 against 1.19456771e-3)."""
    import importlib
    from tests.test_host_mirror_cpu import _quantum
    M = importlib.import_module("xspde_matlab_b200.xsim")
    g, o = _quantum()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        eo, do, _ = X.xsim(o)
    eo = np.asarray(eo)
    keep = [i for i in range(len(eo)) if i != 5]
    res = {}
    for name, patch in (("rounded", None), ("fused", _fused)):
        emu = Emulated(tmp_path / name, g, patch)
        monkeypatch.setattr(M, "GpuPath", lambda p, path_kind=0, runtime_params=False, emu=emu: EmulatedPath(emu, o))
        e, d, _ = M.xsim(g)
        res[name] = (np.asarray(e), d)
    e, d = res["rounded"]
    assert np.allclose(e[keep], eo[keep], rtol=1e-8, atol=1e-14)
    assert np.all(np.asarray(d[0][1])[:, 1] == 0)
    e, d = res["fused"]
    assert np.isclose(e[1], eo[1] * math.sqrt(3 / 4), rtol=1e-6)
    assert np.isclose(e[1], 1.03452598e-3, rtol=1e-6) and np.isclose(eo[1], 1.19456771e-3, rtol=1e-6)
    assert np.isclose(e[2], eo[2], rtol=1e-10)
    for a, b in zip(d[0], do[0]):
        assert np.allclose(np.asarray(a)[:, 0], np.asarray(b)[:, 0], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("method,checks", [("MP", 1), ("RK4", 1), ("RK4", 0)])
def test_emulated_resident_kernel_snls_lattice(tmp_path, method, checks):
    """The 1D stochastic NLS of the benchmark set (64 periodic points, i d2a/dx2 through the
    shared-memory Stockham FFT and the FP64 propagator, MP with merged half-step propagators
    or RK4) against the oracle: every site, output time and check pass to 1e-12."""
    base = dict(dimensions=2, points=[4, 64], ranges=[0.3, 10.0], steps=3, ensembles=[16, 2, 1], noises=2,
                method=method, checks=checks, order=1)
    g = dict(base, precision="fp64", deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2", observe=["@(a,p) a.*conj(a)", "@(a,p) real(a)"])
    o = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.01 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2,
             observe=[lambda a, p: a * np.conj(a), lambda a, p: np.real(a)])
    emu = Emulated(tmp_path, g)
    NS = 64
    for nc in ((1, 2) if checks else (1,)):
        for b in (0, 1):
            got = emu.block_means(o, b, nc)
            ref, _ = oracle_block_av(o, b, nc)
            for k in range(2):
                r = np.asarray(ref[k]).reshape(base["points"][0], NS, order="F")
                assert _rel(got[:, k * NS:(k + 1) * NS].reshape(-1), r.reshape(-1)) < 1e-12, (nc, b, k)


def test_emulated_resident_kernel_has_no_barrier_races(tmp_path):
    """The same launches with the threads of each CTA run in index order, reversed and in fresh
    random orders between barriers give bit-identical block means: no result depends on an
    order that a missing __syncthreads or __syncwarp would leave open (the Quantum example's
    auxiliary cells, spectrum record and reductions; the 64-point lattice's Stockham FFT)."""
    from tests.test_host_mirror_cpu import _quantum
    g, o = _quantum()
    cases = [(Emulated(tmp_path / "q", g), o, 1)]
    base = dict(dimensions=2, points=[3, 64], ranges=[0.2, 10.0], steps=2, ensembles=[16, 1, 1], noises=2,
                method="MP", checks=1, order=1)
    gs = dict(base, precision="fp64", deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)",
              initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2", observe=["@(a,p) a.*conj(a)", "@(a,p) real(a)"])
    os_ = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.01 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
               initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2,
               observe=[lambda a, p: a * np.conj(a), lambda a, p: np.real(a)])
    cases.append((Emulated(tmp_path / "s", gs), os_, 2))
    for emu, oo, nc in cases:
        runs = []
        for kind in (0, 1, 7, 12345):
            emu.lib.emu_set_schedule(kind)
            runs.append(emu.block_means(oo, 0, nc))
        emu.lib.emu_set_schedule(0)
        for r in runs[1:]:
            assert np.array_equal(r, runs[0])


def test_schedule_check_catches_a_missing_barrier(tmp_path):
    """The check above has teeth: with the barrier before the Stockham FFT of xs_tr taken out
    (on the CPU copy of the source only), the FFT may read elements another thread has not yet
    written, and some thread order changes the result."""
    old = "    __syncthreads();\n    xs_fft_d<D>(X, T, P.tmat + P.tmat_off[D], dir);"

    def drop_barrier(src):
        assert old in src
        return src.replace(old, "    xs_fft_d<D>(X, T, P.tmat + P.tmat_off[D], dir);")
    base = dict(dimensions=2, points=[3, 64], ranges=[0.2, 10.0], steps=2, ensembles=[16, 1, 1], noises=2,
                method="MP", checks=1, order=1)
    g = dict(base, precision="fp64", deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2", observe=["@(a,p) a.*conj(a)", "@(a,p) real(a)"])
    o = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.01 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2,
             observe=[lambda a, p: a * np.conj(a), lambda a, p: np.real(a)])
    emu = Emulated(tmp_path, g, drop_barrier)
    runs = []
    for kind in (0, 1, 7):
        emu.lib.emu_set_schedule(kind)
        runs.append(emu.block_means(o, 0, 1))
    emu.lib.emu_set_schedule(0)
    assert any(not np.array_equal(r, runs[0]) for r in runs[1:])


ASAN_RUN = r"""
import pathlib, sys
import numpy as np
from tests.test_resident_emulated_cpu import Emulated, _snls
from tests.test_host_mirror_cpu import _quantum
tmp = pathlib.Path(sys.argv[1])
# every problem is generated before the first emulated launch switches stacks, which the
# sanitizer tracks only approximately
cases = [(Emulated(tmp / name, g, asan=True), o, passes)
         for name, (g, o), passes in (("quantum", _quantum(), (1, 2)), ("snls", _snls("MP", 1), (2,)),
                                      ("snls_rk4", _snls("RK4", 1), (1,)))]
for emu, o, passes in cases:
    for nc in passes:
        emu.block_means(o, 1, nc)
print("clean")
"""


def _snls(method, checks):
    base = dict(dimensions=2, points=[3, 64], ranges=[0.2, 10.0], steps=2, ensembles=[16, 1, 1], noises=2,
                method=method, checks=checks, order=1)
    g = dict(base, precision="fp64", deriv="@(a,w,p) 1i*a.*conj(a).*a + 0.01*(w(1,:)+1i*w(2,:))/sqrt(2)",
             initial="@(v,p) exp(-p.x.^2)", linear="@(p) 1i*p.Dx.^2", observe=["@(a,p) a.*conj(a)", "@(a,p) real(a)"])
    o = dict(base, deriv=lambda a, w, p: 1j * a * np.conj(a) * a + 0.01 * (w[0:1] + 1j * w[1:2]) / np.sqrt(2),
             initial=lambda v, p: np.exp(-p.x ** 2), linear=lambda p: 1j * p.Dx ** 2,
             observe=[lambda a, p: a * np.conj(a), lambda a, p: np.real(a)])
    return g, o


def test_emulated_resident_kernel_stays_in_bounds(tmp_path):
    """Bounds checking without a GPU (compute-sanitizer is closed on this pool): the emulated
    kernel built with AddressSanitizer, its shared memory exactly the launch's size and every
    launch buffer exactly the size the host allocates, runs the Quantum example (auxiliary
    cells, spectrum record; both passes) and the 64-point lattice (MP coarse pass, RK4 fine pass)
    without an out-of-bounds access."""
    import sys
    libs = [subprocess.run(["g++", "-print-file-name=%s" % n], capture_output=True, text=True).stdout.strip()
            for n in ("libasan.so", "libstdc++.so")]
    if not all(x and os.path.exists(x) for x in libs):
        pytest.skip("no AddressSanitizer runtime")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    # the sanitizer runtime first, and the C++ runtime with it so that its exception interceptor
    # binds at start-up (the library throws and catches exceptions internally)
    env = dict(os.environ, LD_PRELOAD=" ".join(os.path.realpath(x) for x in libs),
               ASAN_OPTIONS="detect_leaks=0:halt_on_error=1", PYTHONPATH=root)
    r = subprocess.run([sys.executable, "-c", ASAN_RUN, str(tmp_path)], cwd=root, env=env, capture_output=True,
                       text=True, timeout=900)
    assert "ERROR: AddressSanitizer" not in r.stderr, r.stderr[-4000:]
    assert r.returncode == 0 and "clean" in r.stdout, r.stderr[-4000:]


ASAN_PLANTED = r"""
import pathlib, sys
from tests.test_resident_emulated_cpu import Emulated
from tests.test_host_mirror_cpu import _quantum
old = "double2* out = P.obs + ((size_t)n * nctas + cta) * XS_OBS_STRIDE;"
g, o = _quantum()
emu = Emulated(pathlib.Path(sys.argv[1]), g, lambda src: src.replace(old, old[:-1] + " + 1;"), asan=True)
emu.block_means(o, 0, 1)
print("not caught")
"""


def test_bounds_check_catches_an_overrun(tmp_path):
    """The check above has teeth: the observable rows shifted by one element (on a CPU copy
    of the source only) make the last CTA write past the partial-sum buffer, and the
    sanitizer stops the run with a heap-buffer-overflow."""
    import sys
    libs = [subprocess.run(["g++", "-print-file-name=%s" % n], capture_output=True, text=True).stdout.strip()
            for n in ("libasan.so", "libstdc++.so")]
    if not all(x and os.path.exists(x) for x in libs):
        pytest.skip("no AddressSanitizer runtime")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, LD_PRELOAD=" ".join(os.path.realpath(x) for x in libs),
               ASAN_OPTIONS="detect_leaks=0:halt_on_error=1", PYTHONPATH=root)
    r = subprocess.run([sys.executable, "-c", ASAN_PLANTED, str(tmp_path)], cwd=root, env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode != 0 and "heap-buffer-overflow" in r.stderr, (r.returncode, r.stdout[-500:])
