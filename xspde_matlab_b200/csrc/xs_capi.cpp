// Host side of the B200 xSPDE path: problem set-up (grids, FP64 tables),
// kernel generation, NVRTC compilation with an on-disk cubin cache, device
// buffers and launches.  Exposes the C ABI of include/xspde_b200.h.
#include "xspde_b200.h"

#include <cuda.h>
#include <cuda_runtime.h>
#include <atomic>
#include <functional>
#include <numeric>
#include <thread>
#include <nvrtc.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

#include "xs_expr.hpp"
#include "xs_noalloc.hpp"
#include "xs_mlp.hpp"
#include "xs_aot.hpp"

extern const char* xs_kernel_source_prelude;
extern const char* xs_kernel_source_noise;
extern const char* xs_kernel_source_resident;
extern const char* xs_kernel_source_stream;
extern const char* xs_kernel_source_stream_common;
extern const char* xs_kernel_source_stream3;
extern const char* xs_kernel_source_stream3_tc;

namespace {

using cd = std::complex<double>;

thread_local std::string g_err;

struct XsError {
  xs_status code;
  std::string msg;
};

[[noreturn]] void raise(xs_status code, const std::string& msg) { throw XsError{code, msg}; }

#define CUDA_CHECK(x)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess) raise(XS_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------------------
// Driver API entry points (resolved through the runtime; no link to libcuda)
// ---------------------------------------------------------------------------
typedef CUresult (*PFN_ModuleLoadData)(CUmodule*, const void*);
typedef CUresult (*PFN_ModuleUnload)(CUmodule);
typedef CUresult (*PFN_ModuleGetFunction)(CUfunction*, CUmodule, const char*);
typedef CUresult (*PFN_FuncSetAttribute)(CUfunction, CUfunction_attribute, int);
typedef CUresult (*PFN_LaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                                     unsigned, CUstream, void**, void**);
typedef CUresult (*PFN_GetErrorString)(CUresult, const char**);
typedef CUresult (*PFN_Occupancy)(int*, CUfunction, int, size_t);
typedef CUresult (*PFN_TensorMapEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                            const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                            CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                            CUtensorMapFloatOOBfill);

struct Driver {
  PFN_ModuleLoadData load = nullptr;
  PFN_ModuleUnload unload = nullptr;
  PFN_ModuleGetFunction getfn = nullptr;
  PFN_FuncSetAttribute setattr = nullptr;
  PFN_LaunchKernel launch = nullptr;
  PFN_GetErrorString errstr = nullptr;
  PFN_Occupancy occupancy = nullptr;
  PFN_TensorMapEncodeTiled tmap_encode = nullptr;
};

template <class T>
void resolve(const char* name, T& fn) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
    raise(XS_ERR_CUDA, std::string("cannot resolve driver entry point ") + name);
  fn = reinterpret_cast<T>(p);
}

Driver& driver() {
  static Driver d;
  static std::once_flag once;
  static std::string err;
  std::call_once(once, [] {
    try {
      resolve("cuModuleLoadData", d.load);
      resolve("cuModuleUnload", d.unload);
      resolve("cuModuleGetFunction", d.getfn);
      resolve("cuFuncSetAttribute", d.setattr);
      resolve("cuLaunchKernel", d.launch);
      resolve("cuGetErrorString", d.errstr);
      resolve("cuOccupancyMaxActiveBlocksPerMultiprocessor", d.occupancy);
      resolve("cuTensorMapEncodeTiled", d.tmap_encode);
    } catch (const XsError& e) {
      err = e.msg;
    }
  });
  if (!err.empty()) raise(XS_ERR_CUDA, err);
  return d;
}

void cu_check(CUresult r, const char* what) {
  if (r == CUDA_SUCCESS) return;
  const char* s = "?";
  if (driver().errstr) driver().errstr(r, &s);
  raise(XS_ERR_CUDA, std::string(what) + ": " + s);
}

void ensure_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) raise(XS_ERR_NODEVICE, "no CUDA device available");
  CUDA_CHECK(cudaFree(nullptr));  // create the primary context
}

// ---------------------------------------------------------------------------
// NVRTC with on-disk cache
// ---------------------------------------------------------------------------
uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ull) {
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

// XSPDE_B200_TRACE=1: one line on stderr per module load step and per kernel launch (name, grid,
// block, dynamic shared memory), flushed before the call it describes.
bool trace_on() {
  static const bool on = [] {
    const char* e = getenv("XSPDE_B200_TRACE");
    return e && *e && *e != '0';
  }();
  return on;
}

// NVTX range over one public call (header-only NVTX 3: a no-op unless a profiler
// such as Nsight Compute attaches, which can then filter launches by range name)
struct NvtxRange {
  explicit NvtxRange(const char* fmt, ...) {
    char buf[160];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    nvtxRangePushA(buf);
  }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

void trace(const char* fmt, ...) {
  if (!trace_on()) return;
  va_list ap;
  va_start(ap, fmt);
  fputs("[xspde_b200] ", stderr);
  vfprintf(stderr, fmt, ap);
  fputc('\n', stderr);
  fflush(stderr);
  va_end(ap);
}

std::string cache_dir() {
  const char* e = getenv("XSPDE_B200_CACHE");
  if (e && *e) return e;
  const char* home = getenv("HOME");
  return std::string(home && *home ? home : "/tmp") + "/.cache/xspde_b200";
}

void mkdirs(const std::string& path) {
  std::string cur;
  std::stringstream ss(path);
  std::string part;
  if (!path.empty() && path[0] == '/') cur = "/";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    cur += part + "/";
    mkdir(cur.c_str(), 0755);
  }
}

std::string nvrtc_compile(const std::string& src, const std::string& name, std::string* log_out) {
  std::vector<std::string> opts = {"--gpu-architecture=sm_100a", "-std=c++17", "--device-as-default-execution-space",
                                   "-lineinfo", "--extra-device-vectorization", "-DXS_NVRTC=1"};
  if (const char* v = getenv("XSPDE_B200_PTXAS_VERBOSE"))
    if (*v && *v != '0') opts.push_back("--ptxas-options=-v");
  // XSPDE_B200_DEFINES="-DNAME=value ...": extra preprocessor definitions for the generated
  // kernels (tuning knobs such as XS_SPASS_MINB, the column pass's minimum CTAs per SM)
  if (const char* dv = getenv("XSPDE_B200_DEFINES")) {
    std::stringstream ds(dv);
    std::string d;
    while (ds >> d)
      if (d.rfind("-D", 0) == 0) opts.push_back(d);
  }
  int maj = 0, min = 0;
  nvrtcVersion(&maj, &min);
  std::string key = src;
  for (auto& o : opts) key += "\n" + o;
  key += "\nnvrtc" + std::to_string(maj) + "." + std::to_string(min);
  char hb[32];
  snprintf(hb, sizeof hb, "%016llx", (unsigned long long)fnv1a(key));
  std::string dir = cache_dir();
  std::string path = dir + "/" + name + "_" + hb + ".cubin";
  if (const char* dd = getenv("XSPDE_B200_DUMP"))  // generated CUDA C++ source, for inspection
    if (*dd) {
      mkdirs(dd);
      std::ofstream f(std::string(dd) + "/" + name + "_" + hb + ".cu");
      f << src;
    }
  {
    std::ifstream f(path, std::ios::binary);
    if (f) {
      std::string data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
      if (!data.empty()) return data;
    }
  }
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.c_str(), (name + ".cu").c_str(), 0, nullptr, nullptr) != NVRTC_SUCCESS)
    raise(XS_ERR_NVRTC, "nvrtcCreateProgram failed");
  std::vector<const char*> copts;
  for (auto& o : opts) copts.push_back(o.c_str());
  nvrtcResult r = nvrtcCompileProgram(prog, (int)copts.size(), copts.data());
  size_t lsz = 0;
  nvrtcGetProgramLogSize(prog, &lsz);
  std::string log(lsz, '\0');
  if (lsz) nvrtcGetProgramLog(prog, &log[0]);
  if (log_out) *log_out = log;
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    raise(XS_ERR_NVRTC, "NVRTC compilation failed:\n" + log);
  }
  size_t csz = 0;
  nvrtcGetCUBINSize(prog, &csz);
  std::string cubin(csz, '\0');
  nvrtcGetCUBIN(prog, &cubin[0]);
  nvrtcDestroyProgram(&prog);
  mkdirs(dir);
  std::string tmp = path + ".tmp" + std::to_string((long)getpid()) + "_" +
                    std::to_string(std::hash<std::thread::id>{}(std::this_thread::get_id()));
  {
    std::ofstream f(tmp, std::ios::binary);
    f.write(cubin.data(), (std::streamsize)cubin.size());
  }
  rename(tmp.c_str(), path.c_str());
  return cubin;
}

// ---------------------------------------------------------------------------
// Problem description and FP64 host tables
// ---------------------------------------------------------------------------
struct ObsInfo {
  int lines = 1;
  bool spatial = true;
  int red_off = 0;      // offset of its reductions in the combined red[] array
  int out_off = 0;      // offset in the site (spatial) or scalar output lists
  bool kspace = false;  // evaluated on the Fourier-transformed field (p.transforms{n})
  bool tspec = false;   // evaluated on the time spectrum of the field (p.transforms{n}(1))
  xs::Generated gen;
  // Int/Ave over a subset of the space dimensions that is the whole observable (Int.m:48-70,
  // Ave.m): the device evaluates the integrand as a site observable and the host sums the
  // block means over the reduced dimensions (a linear map: it commutes with the ensemble mean).
  // pw[d] > 0: dimension d reduced with weight pw[d] (Int: dx or dk; Ave: 1 / points);
  // bounds plo[d] < phi[d] restrict an Int to the points of Int.m's rule.
  bool partial = false;
  double pw[3] = {0, 0, 0}, plo[3] = {0, 0, 0}, phi[3] = {0, 0, 0};
};

struct Problem {
  xs_problem p{};
  std::string deriv, initial, linear;
  std::vector<std::string> observe;
  xs::Scalars scalars;
  std::vector<std::string> runtime_names;  // named scalars read at run time (prm[k])
  std::vector<std::vector<int>> obs_tr;    // per observable: p.transforms{n} flags (time, x, y, z)
  int ktr[3] = {0, 0, 0};                  // space dimensions the k-space observables transform
  bool kobs = false;                       // some observable is evaluated in Fourier space
  bool stencil = false;                    // some observable uses D1/D2 (neighbouring sites)
  bool dstencil = false;                   // the drift uses D1/D2: no fused MP iterations
  bool bvals = false;                      // boundary values of p.boundfun supplied per pass
  bool spec = false;                       // some observable is evaluated on the time spectrum
  int NK = 0, NKV = 0;                     // k-filtered noises / initial randoms (xnoise.m:39-50, xrandom.m:24-29)
  int NA = 0;                              // auxiliary cell components (p.auxfields, p.define)
  std::string define;
  std::vector<double> kfilt, rfilt;        // [NK][NS] / [NKV][NS] complex filter factors (empty: identity)
  std::vector<double> runtime_defaults;
  std::vector<int> bnd;  // [D][F][2]
  int D = 0, F = 1, NW = 0, NV = 0, NS = 1, E1 = 1;
  int N[3] = {1, 1, 1};
  double dx[XS_MAXDIM] = {1, 1, 1, 1}, dk[XS_MAXDIM] = {0, 0, 0, 0};
  double dt = 0, nscale = 0, noisefactor = 1, dv = 1;
  std::vector<double> xc[3];
  std::vector<std::vector<std::vector<double>>> kprop;  // [F][D][N]
  bool has_linear = false, setbound = false;
  std::vector<cd> L;  // [Lc][NS]
  int Lc = 1;
  std::vector<ObsInfo> obs;
  int nred = 0, nout_site = 0, nout_scalar = 0;
  int type(int d, int f) const {  // boundary type b1 + 2*b2 (xtransform.m:30)
    if (bnd.empty()) return 0;
    return bnd[(d * F + f) * 2] + 2 * bnd[(d * F + f) * 2 + 1];
  }
};

const char* method_name(int m) {
  switch (m) {
    case XS_METHOD_MP: return "MP";
    case XS_METHOD_RK4: return "RK4";
    case XS_METHOD_EULER: return "Euler";
    case XS_METHOD_RK2: return "RK2";
    case XS_METHOD_IMPLICIT: return "Implicit";
  }
  return "?";
}

void setup_problem(const xs_problem* in, Problem& P) {
  if (!in) raise(XS_ERR_ARG, "null problem");
  P.p = *in;
  const xs_problem& p = P.p;
  if (p.dimensions < 1 || p.dimensions > XS_MAXDIM)
    raise(XS_ERR_UNSUPPORTED, "dimensions must be 1..4 (time + up to 3 space dimensions)");
  if (p.fields < 1 || p.fields > 16) raise(XS_ERR_SHAPE, "fields must be 1..16");
  if (p.noises < 0 || p.noises > 32 || p.inrandoms < 0 || p.inrandoms > 32) raise(XS_ERR_SHAPE, "noises/inrandoms must be 0..32");
  if (p.steps < 1 || p.points[0] < 1) raise(XS_ERR_SHAPE, "points(1) and steps must be positive");
  if (p.checks < 0 || p.checks > 1) raise(XS_ERR_SHAPE, "checks(1) must be 0 or 1");
  if (p.sequence < 0 || p.sequence > 32767) raise(XS_ERR_ARG, "sequence index must be 0..32767");
  if (p.method < 0 || p.method > 4) raise(XS_ERR_ARG, "unknown method");
  if (p.iterations < 1) raise(XS_ERR_ARG, "iterations must be >= 1");
  if (p.ipsteps < 1) raise(XS_ERR_ARG, "ipsteps must be >= 1");
  for (int i = 0; i < 3; ++i)
    if (p.ensembles[i] < 1) raise(XS_ERR_SHAPE, "ensembles must be >= 1");
  P.D = p.dimensions - 1;
  P.F = p.fields;
  P.NW = p.noises;
  P.NV = p.inrandoms;
  P.E1 = p.ensembles[0];
  P.NS = 1;
  for (int d = 0; d < P.D; ++d) {
    if (p.points[d + 1] < 1) raise(XS_ERR_SHAPE, "space points must be positive");
    P.N[d] = p.points[d + 1];
    P.NS *= P.N[d];
  }
  P.deriv = p.deriv ? p.deriv : "@(a,w,p) 0*a";
  P.initial = p.initial ? p.initial : "@(v,p) 0";
  P.linear = (p.linear && *p.linear) ? p.linear : "";
  for (int i = 0; i < p.nobserve; ++i) P.observe.push_back(p.observe && p.observe[i] ? p.observe[i] : "@(a,p) a");
  if (P.observe.empty()) P.observe.push_back("@(a,p) a");
  for (int i = 0; i < p.nparams; ++i) {
    if (p.runtime_params) {
      P.runtime_names.push_back(p.param_names[i]);
      P.runtime_defaults.push_back(p.param_values[i]);
    } else {
      P.scalars.values[p.param_names[i]] = p.param_values[i];
    }
  }
  if (p.runtime_params && !P.linear.empty()) {
    // p.linear is evaluated on the host once: it reads the default values
    for (int i = 0; i < p.nparams; ++i) P.scalars.values[p.param_names[i]] = p.param_values[i];
  }
  for (int i = 0; i < p.nobserve || (i == 0 && p.nobserve == 0); ++i) {
    std::vector<int> tr(4, 0);
    if (p.transforms && i < p.nobserve)
      for (int d = 0; d < 4; ++d) tr[d] = p.transforms[i * 4 + d] ? 1 : 0;
    P.obs_tr.push_back(tr);
  }
  P.p.transforms = nullptr;
  P.p.deriv = P.p.initial = P.p.linear = nullptr;
  P.p.observe = nullptr;
  P.p.param_names = nullptr;
  P.p.param_values = nullptr;
  if (p.boundaries) {
    P.bnd.assign(in->boundaries, in->boundaries + (size_t)P.D * P.F * 2);
    for (int v : P.bnd)
      if (v < -1 || v > 1) raise(XS_ERR_ARG, "boundary flags must be -1, 0 or 1");
    for (int d = 0; d < P.D; ++d)
      for (int f = 0; f < P.F; ++f) {
        int t = P.type(d, f);
        if (t != 0 && t != 3 && t != -3 && t != 1 && t != -1)
          raise(XS_ERR_ARG, "invalid boundary pair");
        if (t != 0) P.setbound = true;
      }
  }
  P.p.boundaries = nullptr;
  if (p.knoises < 0 || p.knoises > 32 || p.krandoms < 0 || p.krandoms > 32)
    raise(XS_ERR_SHAPE, "knoises/krandoms must be 0..32");
  P.NK = p.knoises;
  P.NKV = p.krandoms;
  if (P.NK || P.NKV) {
    if (P.D == 0) raise(XS_ERR_UNSUPPORTED, "k-filtered noises need at least one space dimension");
    for (int d = 0; d < P.D; ++d)
      for (int f = 0; f < P.F; ++f)
        if (P.type(d, f) != 0)
          raise(XS_ERR_UNSUPPORTED, "k-filtered noises need periodic space dimensions (xift.m: inverse DFT)");
    if (p.nfilter && P.NK) P.kfilt.assign(p.nfilter, p.nfilter + (size_t)2 * P.NK * P.NS);
    if (p.rfilter && P.NKV) P.rfilt.assign(p.rfilter, p.rfilter + (size_t)2 * P.NKV * P.NS);
  }
  P.p.nfilter = P.p.rfilter = nullptr;
  if (p.auxfields < 0 || p.auxfields > 16) raise(XS_ERR_SHAPE, "auxfields must be 0..16");
  P.NA = p.auxfields;
  if (P.NA) {
    if (!p.define || !*p.define) raise(XS_ERR_ARG, "auxfields given without p.define");
    P.define = p.define;
  }
  P.p.define = nullptr;
  if (p.boundary_values) {
    if (P.bnd.empty()) raise(XS_ERR_ARG, "boundary values given but every boundary is periodic");
    if (p.method != XS_METHOD_MP) raise(XS_ERR_UNSUPPORTED, "boundary values (p.boundfun) are supported with MP");
    P.bvals = true;
  }
  // k-space observables (xdata.m, xnft.m): one common set of periodic space dimensions
  for (auto& tr : P.obs_tr) {
    if (tr[0]) P.spec = true;  // time spectrum (xpath.m:46-106)
    int k[3] = {0, 0, 0};
    bool any = false;
    for (int d = 0; d < P.D; ++d)
      if (tr[d + 1] && P.N[d] > 1) {
        for (int f = 0; f < P.F; ++f)
          if (P.type(d, f) != 0)
            raise(XS_ERR_UNSUPPORTED, "k-space observables are supported along periodic dimensions only");
        k[d] = 1;
        any = true;
      }
    if (!any) {
      for (int d = 1; d < 4; ++d) tr[d] = 0;
      continue;
    }
    if (P.kobs && (k[0] != P.ktr[0] || k[1] != P.ktr[1] || k[2] != P.ktr[2]))
      raise(XS_ERR_UNSUPPORTED, "k-space observables must all transform the same dimensions");
    for (int d = 0; d < 3; ++d) P.ktr[d] = k[d];
    P.kobs = true;
  }
  if (P.kobs && P.NA) raise(XS_ERR_UNSUPPORTED, "k-space observables with auxiliary fields are not supported on the device");
  // grid constants (Simulator/xpreferences.m:133-175, spdpreferences.m:16-70)
  for (int d = 0; d < p.dimensions; ++d) {
    int n = p.points[d];
    P.dx[d] = n == 1 ? 1.0 : p.ranges[d] / std::max(1, n - 1);
  }
  P.dv = 1;
  for (int d = 1; d < p.dimensions; ++d) P.dv *= P.dx[d];
  P.noisefactor = 1.0 / P.dv;
  for (int d = 1; d < p.dimensions; ++d) P.dk[d] = 2 * M_PI / (p.points[d] * P.dx[d]);
  P.dk[0] = 2 * M_PI / (p.points[0] * P.dx[0]) / p.steps;
  P.dt = p.ranges[0] / std::max(1, p.points[0] - 1);
  P.nscale = p.steps * (1.0 + p.checks) / P.dt;
  P.kprop.assign(P.F, std::vector<std::vector<double>>(P.D));
  for (int d = 0; d < P.D; ++d) {
    int n = P.N[d];
    P.xc[d].resize(n);
    for (int i = 0; i < n; ++i) P.xc[d][i] = p.origins[d + 1] + i * P.dx[d + 1];
    double dkd = P.dk[d + 1];
    double dkp = n > 1 ? M_PI / ((n - 1) * P.dx[d + 1]) : 0.0;
    for (int f = 0; f < P.F; ++f) {
      std::vector<double>& k = P.kprop[f][d];
      k.resize(n);
      int t = P.type(d, f);
      for (int i = 0; i < n; ++i) {
        if (t == 0) {
          int j = (i + n / 2) % n;  // ifftshift of kc = (j - floor(n/2)) dk
          k[i] = (j - n / 2) * dkd;
        } else if (t == 3 || t == -3) {
          k[i] = i * dkp;
        } else if (t == -1) {
          k[i] = i == 0 ? 0.0 : (i - 0.5) * dkp;
        } else {  // t == 1
          k[i] = i == n - 1 ? 0.0 : (i + 0.5) * dkp;
        }
      }
    }
  }
  // linear operator -> L(k) in FP64 (xpropfactor.m:30-39)
  if (!P.linear.empty()) {
    xs::AnonFn fn = xs::parse_anon(P.linear);
    if (P.D == 0) raise(XS_ERR_UNSUPPORTED, "p.linear needs at least one space dimension");
    xs::GridInfo g;
    g.ndim = P.D;
    g.nfield = P.F;
    for (int d = 0; d < P.D; ++d) {
      g.n.push_back(P.N[d]);
      g.x.push_back(P.xc[d]);
    }
    g.k.assign(P.F, std::vector<std::vector<double>>(P.D));
    for (int f = 0; f < P.F; ++f)
      for (int d = 0; d < P.D; ++d) g.k[f][d] = P.kprop[f][d];
    P.L = xs::eval_linear(fn, g, P.scalars, &P.Lc);
    P.has_linear = true;
  }
  if (P.D > 0 && !P.has_linear && P.setbound == false) {
    // nothing: no propagation (xprop skips unit propagators)
  }
}

// Host restatements of the reference's non-periodic transforms, applied to
// unit vectors to obtain their (real) matrices.  They follow
// Applications/SPDE/xdct1.m, xdst1.m, xdct2.m, xdct3.m, xdst2.m, xdst3.m with a
// direct DFT in place of fft.
std::vector<cd> dft(const std::vector<cd>& x) {
  size_t M = x.size();
  std::vector<cd> y(M);
  for (size_t k = 0; k < M; ++k) {
    cd acc = 0;
    for (size_t n = 0; n < M; ++n) acc += x[n] * std::polar(1.0, -2 * M_PI * (double)((k * n) % M) / M);
    y[k] = acc;
  }
  return y;
}

std::vector<double> transform_real(int type, bool inv, const std::vector<double>& a) {
  int N = (int)a.size();
  std::vector<double> out(N, 0.0);
  if (N < 2) return a;
  auto kind = type == -3 ? 0 : type == 3 ? 1 : type == -1 ? (inv ? 3 : 2) : (inv ? 5 : 4);
  // 0 dct1, 1 dst1, 2 dst3 (fwd DN), 3 dst2 (inv DN), 4 dct3 (fwd ND), 5 dct2 (inv ND)
  int M = N - 1;
  if (kind == 0) {
    std::vector<cd> e(2 * M);
    for (int i = 0; i < N; ++i) e[i] = a[i];
    for (int i = 1; i < N - 1; ++i) e[N - 1 + i] = a[N - 1 - i];
    auto y = dft(e);
    for (int k = 0; k < N; ++k) out[k] = y[k].real() * std::sqrt(1.0 / (2.0 * M));
  } else if (kind == 1) {
    std::vector<cd> e(2 * M);
    for (int i = 1; i < N - 1; ++i) e[i] = a[i];
    for (int i = 0; i < N - 2; ++i) e[N + i] = -a[N - 2 - i];
    auto y = dft(e);
    for (int k = 1; k < N - 1; ++k) out[k] = (y[k] * std::sqrt(2.0 / M) / cd(0, -2)).real();
  } else if (kind == 5) {  // xdct2
    std::vector<cd> e(2 * M);
    for (int i = 0; i < M; ++i) e[i] = a[i];
    auto y = dft(e);
    for (int k = 0; k < M; ++k) out[k] = (y[k] * std::polar(1.0, -M_PI / (2.0 * M) * k)).real() * std::sqrt(2.0 / M);
  } else if (kind == 4) {  // xdct3
    std::vector<cd> e(2 * M);
    for (int i = 1; i < M; ++i) e[i] = a[i] * std::polar(1.0, -M_PI / (2.0 * M) * i);
    auto y = dft(e);
    for (int k = 0; k < M; ++k) out[k] = (y[k].real() + 0.5 * a[0]) * std::sqrt(2.0 / M);
  } else if (kind == 3) {  // xdst2
    std::vector<cd> e(2 * M);
    for (int i = 0; i < M; ++i) e[i] = a[i + 1] * std::polar(1.0, -M_PI / M * i);
    auto y = dft(e);
    for (int k = 0; k < M; ++k)
      out[k + 1] = -(y[k] * std::polar(1.0, -M_PI / (2.0 * M) * (k + 1))).imag() * std::sqrt(2.0 / M);
  } else {  // xdst3
    std::vector<cd> e(2 * M);
    for (int i = 0; i < M - 1; ++i) e[i] = a[i + 1] * std::polar(1.0, -M_PI / (2.0 * M) * i);
    auto y = dft(e);
    for (int k = 0; k < M; ++k) {
      double alt = (k % 2 == 0) ? -1.0 : 1.0;  // cumprod(-ones): -1, +1, -1, ...
      out[k + 1] = (-(y[k] * std::polar(1.0, -M_PI / M * (k + 0.5))).imag() - 0.5 * alt * a[N - 1]) * std::sqrt(2.0 / M);
    }
  }
  return out;
}

// Matrix stored as M[n*N + k] = coefficient of input n in output k.
std::vector<cd> transform_matrix(int type, bool inv, int N) {
  std::vector<cd> M((size_t)N * N);
  if (type == 0) {
    for (int n = 0; n < N; ++n)
      for (int k = 0; k < N; ++k) {
        double ang = 2 * M_PI * (double)(((long long)k * n) % N) / N;
        M[(size_t)n * N + k] = inv ? std::polar(1.0 / N, ang) : std::polar(1.0, -ang);
      }
    return M;
  }
  for (int n = 0; n < N; ++n) {
    std::vector<double> e(N, 0.0);
    e[n] = 1.0;
    auto col = transform_real(type, inv, e);
    for (int k = 0; k < N; ++k) M[(size_t)n * N + k] = col[k];
  }
  return M;
}

// Mirror symmetry of an n x n transform matrix: 1 + p when M[n-1-i][k] = (-1)^(k+p) M[i][k] for
// every i, k (DCT-I and DCT-II: p = 0; DST-I on xSPDE's endpoint-inclusive lattice: p = 1), else 0.
int fold_parity(const std::vector<cd>& M, int n) {
  double mx = 0;
  for (const auto& v : M) mx = std::max(mx, std::abs(v));
  for (int par = 0; par < 2; ++par) {
    bool ok = true;
    for (int i = 0; i < n && ok; ++i)
      for (int k = 0; k < n && ok; ++k) {
        const cd x = M[(size_t)(n - 1 - i) * n + k], y = M[(size_t)i * n + k] * ((k + par) % 2 ? -1.0 : 1.0);
        if (std::abs(x - y) > 1e-12 * mx) ok = false;
      }
    if (ok) return 1 + par;
  }
  return 0;
}

// Mirror symmetry of a transform matrix about a centre c in n-1, n-2 or n (the 3D streaming
// kernels): kind 1, input fold, M[c-i][k] = (-1)^(k+p) M[i][k] with every row whose partner lies
// outside the matrix zero; kind 2, output fold, the same for columns; kind 0 none.
struct FoldInfo {
  int kind = 0, c = 0, p = 0;
};

FoldInfo fold_info(const std::vector<cd>& M, int n) {
  double mx = 0;
  for (const auto& v : M) mx = std::max(mx, std::abs(v));
  auto at = [&](int i, int k, bool cols) { return cols ? M[(size_t)k * n + i] : M[(size_t)i * n + k]; };
  for (int kind = 1; kind <= 2; ++kind)
    for (int cc : {n - 1, n - 2, n})
      for (int par = 0; par < 2; ++par) {
        bool ok = true;
        for (int i = 0; i < n && ok; ++i) {
          const int m = cc - i;
          for (int k = 0; k < n && ok; ++k) {
            const cd x = at(i, k, kind == 2);
            if (m < 0 || m >= n) {
              if (std::abs(x) > 1e-12 * mx) ok = false;
            } else if (std::abs(at(m, k, kind == 2) - x * ((k + par) % 2 ? -1.0 : 1.0)) > 1e-12 * mx) {
              ok = false;
            }
          }
        }
        if (ok) return {kind, cc, par};
      }
  return {};
}

// The half of a folded matrix that the kernels read, M[n*N + k] convention: kind 1, rows
// r(j) = j + (c == n) for j < n/2 ([n/2][n]); kind 2, columns r(j) ([n][n/2]).  Entries the
// symmetry makes zero (a row or column that is its own partner, odd parity) are set to 0.
std::vector<double> pack_folded(const std::vector<cd>& M, int n, const FoldInfo& f) {
  if (f.kind == 0) {
    std::vector<double> out(M.size());
    for (size_t i = 0; i < M.size(); ++i) out[i] = M[i].real();
    return out;
  }
  const int h = n / 2;
  std::vector<double> out((size_t)n * h);
  for (int j = 0; j < h; ++j) {
    const int r = j + (f.c == n ? 1 : 0);
    const bool self = f.c - r == r;
    for (int i = 0; i < n; ++i) {
      // kind 1: row r, column i (parity of the output i); kind 2: row i, column r (parity of the input i)
      double v = f.kind == 1 ? M[(size_t)r * n + i].real() : M[(size_t)i * n + r].real();
      if (self && (i + f.p) % 2) v = 0;
      if (f.kind == 1) out[(size_t)j * n + i] = v;
      else out[(size_t)i * h + j] = v;
    }
  }
  return out;
}

// ---------------------------------------------------------------------------
// Code generation
// ---------------------------------------------------------------------------
// dynamic shared memory of xs_p_nl_tc (xs_stream3_tc.cuh, tc3::SMEM_BYTES): B hi/lo of four
// 64 x 64 TF32 matrices, A hi and lo (128 x 64), mbarrier and tensor-memory slot, alignment slack
constexpr size_t kTc3Smem = 8 * 16384 + 2 * 32768 + 16 + 1024;
constexpr unsigned kTc3Threads = 512;  // tc3::NTH

std::string fmt(double v) {
  char b[64];
  snprintf(b, sizeof b, "%.17g", v);
  return b;
}

xs::GenCtx make_ctx(const Problem& P, std::vector<xs::Role> roles, bool reduce) {
  xs::GenCtx c;
  c.roles = std::move(roles);
  c.nfield = P.F;
  c.nnoise = P.NW;
  c.nrand = P.NV;
  c.nknoise = P.NK;
  c.nkrand = P.NKV;
  c.naux = P.NA;
  c.ndim = P.D;
  c.allow_reduce = reduce;
  c.kgrid = reduce;  // observe functions may read p.kx/ky/kz
  c.scalars = &P.scalars;
  c.runtime = P.runtime_names.empty() ? nullptr : &P.runtime_names;
  for (int d = 0; d < P.p.dimensions; ++d) {
    c.dx.push_back(P.dx[d]);
    c.dk.push_back(P.dk[d]);
    c.origins.push_back(P.p.origins[d]);
    c.ranges.push_back(P.p.ranges[d]);
  }
  c.dt = P.dt;
  return c;
}

void generate_functions(Problem& P, std::ostringstream& os) {
  using xs::Role;
  // deriv(a, w, p): xSPDE calls p.deriv{c}(a{:}, xi{:}, p) (MP.m:16)
  {
    auto fn = xs::parse_anon(P.deriv);
    // noise cells in xnoise.m order: Gaussian (absent when noises = 0 and knoises > 0), k-filtered
    std::vector<Role> roles = {Role::Field};
    if (P.NW > 0 || P.NK == 0) roles.push_back(Role::Noise);
    if (P.NK > 0) roles.push_back(Role::KNoise);
    roles.push_back(Role::Params);
    auto g = xs::generate(fn, make_ctx(P, roles, false));
    if (g.len != P.F && g.len != 1)
      raise(XS_ERR_SHAPE, "p.deriv returns " + std::to_string(g.len) + " components, fields = " + std::to_string(P.F));
    P.dstencil = g.stencil;
    os << "#define XS_STENCIL " << (g.stencil ? 1 : 0) << "\n";
    os << "__device__ __forceinline__ cx xs_fd1(const cx* __restrict__ fld, int g, int s, int f, int d);\n";
    os << "__device__ __forceinline__ cx xs_fd2(const cx* __restrict__ fld, int g, int s, int f, int d);\n";
    os << "__device__ __forceinline__ void xs_deriv(const cx* __restrict__ a, const real* __restrict__ w, const cx* __restrict__ zk, real x, real y, real z, real t, const double* __restrict__ prm, const cx* __restrict__ fld, int g, int s, cx* __restrict__ out) {\n";
    os << "  (void)a; (void)w; (void)zk; (void)x; (void)y; (void)z; (void)t; (void)prm; (void)fld; (void)g; (void)s;\n";
    auto body = [&](const xs::Generated& gg) {
      if (gg.len == 1 && P.F > 1) {
        os << "  cx o1[1];\n  { cx* out = o1;\n" << gg.code << "  }\n";
        os << "  for (int f = 0; f < " << P.F << "; ++f) out[f] = o1[0];\n";
      } else {
        os << gg.code;
      }
    };
    body(g);
    os << "}\n";
    // the drift's field-independent terms (noise, sources) apart, for MP's midpoint iterations:
    // xs_deriv_c0: c0 = a0 + h inv once per site, then xs_deriv_step: a = c0 + h dep(a)
    xs::Generated g0, gs;
    const bool split = xs::generate_split(fn, make_ctx(P, roles, false), g0, gs) && g0.len == g.len && gs.len == g.len;
    os << "#define XS_DSPLIT " << (split ? 1 : 0) << "\n";
    if (split) {
      const char* args = "(const cx* __restrict__ a, const cx* __restrict__ c0, real h, const real* __restrict__ w, const cx* __restrict__ zk, real x, real y, real z, real t, const double* __restrict__ prm, const cx* __restrict__ fld, int g, int s, cx* __restrict__ out) {\n";
      const char* unused = "  (void)a; (void)c0; (void)h; (void)w; (void)zk; (void)x; (void)y; (void)z; (void)t; (void)prm; (void)fld; (void)g; (void)s;\n";
      os << "__device__ __forceinline__ void xs_deriv_c0" << args << unused;
      body(g0);
      os << "}\n__device__ __forceinline__ void xs_deriv_step" << args << unused;
      body(gs);
      os << "}\n";
    }
  }
  // define(a, w, p): the auxiliary cell (xpath.m:36-45, xensemble.m:74-77), noise cells as for deriv
  {
    os << "#define XS_NA " << P.NA << "\n#define XS_NAC " << (P.NA + P.F - 1) / P.F << "\n";
    os << "__device__ __forceinline__ void xs_define(const cx* __restrict__ a, const real* __restrict__ w, const cx* __restrict__ zk, real x, real y, real z, real t, const double* __restrict__ prm, const cx* __restrict__ fld, int g, int s, cx* __restrict__ out) {\n";
    os << "  (void)a; (void)w; (void)zk; (void)x; (void)y; (void)z; (void)t; (void)prm; (void)fld; (void)g; (void)s; (void)out;\n";
    if (P.NA) {
      auto fn = xs::parse_anon(P.define);
      std::vector<Role> roles = {Role::Field};
      if (P.NW > 0 || P.NK == 0) roles.push_back(Role::Noise);
      if (P.NK > 0) roles.push_back(Role::KNoise);
      roles.push_back(Role::Params);
      auto g = xs::generate(fn, make_ctx(P, roles, false));
      if (g.len != P.NA && g.len != 1)
        raise(XS_ERR_SHAPE, "p.define returns " + std::to_string(g.len) + " components, auxfields = " + std::to_string(P.NA));
      if (g.stencil) raise(XS_ERR_UNSUPPORTED, "D1/D2 in p.define are not supported on the device");
      if (g.len == 1 && P.NA > 1) {
        os << "  cx o1[1];\n  { cx* out = o1;\n" << g.code << "  }\n";
        os << "  for (int f = 0; f < " << P.NA << "; ++f) out[f] = o1[0];\n";
      } else {
        os << g.code;
      }
    }
    os << "}\n";
  }
  // initial(v, p) (xensemble.m:60)
  {
    auto fn = xs::parse_anon(P.initial);
    std::vector<Role> roles;  // random cells in xrandom.m order: Gaussian, k-filtered
    if (P.NV > 0 || P.NKV == 0) roles.push_back(Role::Random);
    if (P.NKV > 0) roles.push_back(Role::KRandom);
    roles.push_back(Role::Params);
    auto g = xs::generate(fn, make_ctx(P, roles, false));
    if (g.len != P.F && g.len != 1)
      raise(XS_ERR_SHAPE, "p.initial returns " + std::to_string(g.len) + " components, fields = " + std::to_string(P.F));
    os << "__device__ __forceinline__ void xs_initial(const real* __restrict__ v, const cx* __restrict__ vk, real x, real y, real z, const double* __restrict__ prm, cx* __restrict__ out) {\n";
    os << "  (void)v; (void)vk; (void)x; (void)y; (void)z; (void)prm; const real t = (real)" << fmt(P.p.origins[0]) << "; (void)t;\n";
    if (g.len == 1 && P.F > 1) {
      os << "  cx o1[1];\n  { cx* out = o1;\n" << g.code << "  }\n";
      os << "  for (int f = 0; f < " << P.F << "; ++f) out[f] = o1[0];\n";
    } else {
      os << g.code;
    }
    os << "}\n";
  }
  // observe{n}(a, p) (xdata.m:30)
  P.obs.clear();
  P.nred = P.nout_site = P.nout_scalar = 0;
  for (size_t oi = 0; oi < P.observe.size(); ++oi) {
    const std::string& txt = P.observe[oi];
    ObsInfo o;
    o.kspace = oi < P.obs_tr.size() && (P.obs_tr[oi][1] || P.obs_tr[oi][2] || P.obs_tr[oi][3]);
    o.tspec = oi < P.obs_tr.size() && P.obs_tr[oi][0];
    auto fn = xs::parse_anon(txt);
    // observe{n}(a{:}, p): the field, then the auxiliary cell when there is one (xdata.m:29)
    o.gen = xs::generate(fn, make_ctx(P, P.NA ? std::vector<Role>{Role::Field, Role::Aux, Role::Params}
                                              : std::vector<Role>{Role::Field, Role::Params}, true));
    o.lines = o.gen.len;
    o.spatial = o.gen.spatial;  // depends on the field or the site (0-D: one site)
    if (o.gen.stencil) P.stencil = true;
    o.red_off = P.nred;
    bool subset = false;
    for (auto& r : o.gen.reductions) subset = subset || (int)r.dims.size() != P.D;
    if (subset) {
      const xs::NodeP& body = fn.body;
      const bool top = body->kind == xs::NK::Index && body->kids.size() >= 3 && body->kids[0]->kind == xs::NK::Var &&
                       (body->kids[0]->name == "Int" || body->kids[0]->name == "Ave") &&
                       o.gen.reductions.size() == 1;
      if (!top)
        raise(XS_ERR_UNSUPPORTED,
              "Int/Ave over a subset of the space dimensions must be the whole observable on the device");
      const xs::Reduction R = o.gen.reductions[0];
      bool bounded = false;
      for (size_t k = 0; k < R.dims.size(); ++k) {
        const int d = R.dims[k] - 1;  // space dimension, 0 = x
        o.pw[d] = R.ave ? 1.0 / P.N[d] : R.weight[k];
        o.plo[d] = R.lo[d + 1];
        o.phi[d] = R.hi[d + 1];
        bounded = bounded || o.plo[d] < o.phi[d];
      }
      if (bounded && o.kspace) raise(XS_ERR_UNSUPPORTED, "Int bounds over a subset of k-space dimensions");
      xs::AnonFn f2 = fn;
      f2.body = body->kids[1];  // the integrand, one value per site
      o.gen = xs::generate(f2, make_ctx(P, P.NA ? std::vector<Role>{Role::Field, Role::Aux, Role::Params}
                                                : std::vector<Role>{Role::Field, Role::Params}, true));
      if (!o.gen.reductions.empty()) raise(XS_ERR_UNSUPPORTED, "nested Int/Ave");
      o.lines = o.gen.len;
      o.spatial = true;
      o.partial = true;
    }
    for (auto& r : o.gen.reductions) P.nred += r.lines;
    if (o.spatial) {
      o.out_off = P.nout_site;
      P.nout_site += o.lines;
    } else {
      o.out_off = P.nout_scalar;
      P.nout_scalar += o.lines;
    }
    P.obs.push_back(o);
  }
  os << "#define XS_NRED " << P.nred << "\n#define XS_NOUT_SITE " << P.nout_site << "\n#define XS_NOUT_SCALAR "
     << P.nout_scalar << "\n#define XS_OBS_STRIDE (XS_NOUT_SITE * XS_NS + XS_NOUT_SCALAR)\n";
  // output slots evaluated on the time spectrum (1) or on the field at the output time (0), and
  // slots whose values can have an imaginary part (real ones skip the imaginary moment sums)
  {
    std::vector<int> site(std::max(P.nout_site, 1), 0), scal(std::max(P.nout_scalar, 1), 0);
    std::vector<int> csite(std::max(P.nout_site, 1), 0), cscal(std::max(P.nout_scalar, 1), 0);
    for (auto& o : P.obs)
      for (int l = 0; l < o.lines; ++l) {
        (o.spatial ? site : scal)[o.out_off + l] = o.tspec ? 1 : 0;
        (o.spatial ? csite : cscal)[o.out_off + l] = o.gen.is_complex ? 1 : 0;
      }
    // inline switch functions: with the slot index a constant (unrolled loops) they fold away
    auto table = [&](const char* name, const std::vector<int>& v) {
      os << "__device__ __forceinline__ int " << name << "(int k) {\n  switch (k) {\n";
      for (size_t i = 0; i < v.size(); ++i) os << "    case " << i << ": return " << v[i] << ";\n";
      os << "    default: return 0;\n  }\n}\n";
    };
    os << "#define XS_SPEC " << (P.spec ? 1 : 0) << "\n";
    table("xs_ospec_site", site);
    table("xs_ospec_scalar", scal);
    table("xs_ocplx_site", csite);
    table("xs_ocplx_scalar", cscal);
  }
  // k-space observables: transformed dimensions, normalisation prod kfact = prod dx/sqrt(2 pi) (xnft.m),
  // k grids of the observe functions (p.kx ... in propagation order)
  {
    double kf = 1;
    for (int d = 0; d < 3; ++d)
      if (P.ktr[d]) kf *= P.dx[d + 1] / std::sqrt(2 * M_PI);
    os << "#define XS_KOBS " << (P.kobs ? 1 : 0) << "\n#define XS_KTR1 " << P.ktr[0] << "\n#define XS_KTR2 "
       << P.ktr[1] << "\n#define XS_KTR3 " << P.ktr[2] << "\n#define XS_KFACT " << fmt(kf) << "\n";
    for (int d = 0; d < 3; ++d) {
      os << "__device__ const double xs_kt" << d + 1 << "[] = {";
      if (d < P.D && !P.kprop.empty())
        for (size_t i = 0; i < P.kprop[0][d].size(); ++i) os << (i ? "," : "") << fmt(P.kprop[0][d][i]);
      else
        os << "0";
      os << "};\n";
    }
  }
  // D1/D2 of the field at site s of trajectory g (Applications/SPDE/D1.m:62-105, D2.m:21-77):
  // central differences with periodic wrap; at a Neumann end D1 is the boundary value and D2 the
  // one-sided form, at a Dirichlet end D2 repeats its neighbour (boundary values zero)
  os << "__device__ const int xs_btab[3][" << P.F << "][2] = {";
  for (int d = 0; d < 3; ++d) {
    os << (d ? "," : "") << "{";
    for (int f = 0; f < P.F; ++f) {
      const int lo = (d < P.D && !P.bnd.empty()) ? P.bnd[(d * P.F + f) * 2] : 0;
      const int hi = (d < P.D && !P.bnd.empty()) ? P.bnd[(d * P.F + f) * 2 + 1] : 0;
      os << (f ? "," : "") << "{" << lo << "," << hi << "}";
    }
    os << "}";
  }
  os << "};\n";
  os << R"(__device__ __forceinline__ void xs_fd_geom(int s, int d, int& n, int& sd, int& id, real& dx) {
  if (d == 1) { n = XS_N1; sd = 1; id = s % XS_N1; dx = (real)XS_DX1; }
  else if (d == 2) { n = XS_N2; sd = XS_N1; id = (s / XS_N1) % XS_N2; dx = (real)XS_DX2; }
  else { n = XS_N3; sd = XS_N1 * XS_N2; id = s / (XS_N1 * XS_N2); dx = (real)XS_DX3; }
}
__device__ __forceinline__ cx xs_fd1(const cx* __restrict__ fld, int g, int s, int f, int d) {
  int n, sd, id; real dx;
  xs_fd_geom(s, d, n, sd, id, dx);
  const cx* b = fld + (size_t)(g * XS_F + f) * XS_NS;
  const int sp = s + ((id + 1) % n - id) * sd, sm = s + ((id + n - 1) % n - id) * sd;
  cx o = (b[sp] - b[sm]) / ((real)2 * dx);
  if (id == 0 && xs_btab[d - 1][f][0] == -1) o = mkcx((real)0, (real)0);
  if (id == n - 1 && xs_btab[d - 1][f][1] == -1) o = mkcx((real)0, (real)0);
  return o;
}
__device__ __forceinline__ cx xs_fd2(const cx* __restrict__ fld, int g, int s, int f, int d) {
  int n, sd, id; real dx;
  xs_fd_geom(s, d, n, sd, id, dx);
  const cx* b = fld + (size_t)(g * XS_F + f) * XS_NS;
  const int sp = s + ((id + 1) % n - id) * sd, sm = s + ((id + n - 1) % n - id) * sd;
  cx o = (b[sp] + b[sm] - (real)2 * b[s]) / (dx * dx);
  const int lo = xs_btab[d - 1][f][0], hi = xs_btab[d - 1][f][1];
  if (lo != 0 && n > 2) {
    if (id == 0) o = lo == -1 ? (real)2 * ((b[s + sd] - b[s]) / dx) / dx : (b[s + 2 * sd] + b[s] - (real)2 * b[s + sd]) / (dx * dx);
    if (id == n - 1) o = hi == -1 ? (real)2 * ((b[s - sd] - b[s]) / dx) / dx : (b[s] + b[s - 2 * sd] - (real)2 * b[s - sd]) / (dx * dx);
  }
  return o;
}
)";
  // integrands with bounds masks and weights
  os << "__device__ __forceinline__ void xs_integrands(const cx* __restrict__ a, const cx* __restrict__ ak, const cx* __restrict__ xa, const cx* __restrict__ fld, int g, int s, int i1, int i2, int i3, real x, real y, real z, real t, const double* __restrict__ prm, cx* __restrict__ rr) {\n";
  os << "  (void)a; (void)ak; (void)xa; (void)fld; (void)g; (void)s; (void)i1; (void)i2; (void)i3; (void)x; (void)y; (void)z; (void)t; (void)rr; (void)prm;\n";
  int off = 0;
  for (auto& o : P.obs) {
    for (auto& r : o.gen.reductions) {
      double w = 1;
      std::string mask = "true";
      for (size_t q = 0; q < r.dims.size(); ++q) {
        int d = r.dims[q] - 1;  // 0-based space dim
        int n = P.N[d];
        if (r.ave) w *= 1.0 / n;
        else w *= r.weight[q];
        double lo = r.lo[r.dims[q]], hi = r.hi[r.dims[q]];
        if (!r.ave && lo < hi) {
          // Int.m:62-66: j = 1+floor((lo-x(1))/d); while x(j) <= hi
          double step = r.weight[q];
          int j0 = (int)std::floor((lo - P.xc[d][0]) / step);
          if (j0 < 0) j0 = 0;
          int j = j0;
          while (j < n && P.xc[d][j] <= hi) ++j;
          const char* iv = d == 0 ? "i1" : d == 1 ? "i2" : "i3";
          mask += std::string(" && ") + iv + " >= " + std::to_string(j0) + " && " + iv + " < " + std::to_string(j);
        }
      }
      os << "  {\n    cx* r = rr + " << off << ";\n" << (o.kspace ? "    const cx* a = ak; (void)a;\n" : "")
         << r.integrand_code;
      os << "    const real wgt = (" << mask << ") ? (real)" << fmt(w) << " : (real)0;\n";
      os << "    for (int k = 0; k < " << r.lines << "; ++k) r[k] = r[k] * wgt;\n  }\n";
      off += r.lines;
    }
  }
  os << "}\n";
  os << "__device__ __forceinline__ void xs_obs_site(const cx* __restrict__ a, const cx* __restrict__ ak, const cx* __restrict__ xa, const cx* __restrict__ fld, int g, int s, const cx* __restrict__ redall, real x, real y, real z, int i1, int i2, int i3, real t, const double* __restrict__ prm, cx* __restrict__ outall) {\n";
  os << "  (void)a; (void)ak; (void)xa; (void)fld; (void)g; (void)s; (void)redall; (void)x; (void)y; (void)z; (void)i1; (void)i2; (void)i3; (void)t; (void)outall; (void)prm;\n";
  for (auto& o : P.obs)
    if (o.spatial)
      os << "  {\n    const cx* red = redall + " << o.red_off << "; (void)red;\n    cx* out = outall + " << o.out_off
         << ";\n" << (o.kspace ? "    const cx* a = ak; (void)a;\n" : "") << o.gen.code << "  }\n";
  os << "}\n";
  os << "__device__ __forceinline__ void xs_obs_scalar(const cx* __restrict__ redall, real t, const double* __restrict__ prm, cx* __restrict__ outall) {\n";
  os << "  (void)redall; (void)t; (void)outall; (void)prm; const cx* a = nullptr; const real x = 0, y = 0, z = 0; (void)a; (void)x; (void)y; (void)z;\n";
  os << "  const cx* xa = nullptr; (void)xa;\n";
  os << "  const int i1 = 0, i2 = 0, i3 = 0; (void)i1; (void)i2; (void)i3;\n";
  os << "  const cx* fld = nullptr; const int g = 0, s = 0; (void)fld; (void)g; (void)s;\n";
  for (auto& o : P.obs)
    if (!o.spatial)
      os << "  {\n    const cx* red = redall + " << o.red_off << "; (void)red;\n    cx* out = outall + " << o.out_off
         << ";\n" << o.gen.code << "  }\n";
  os << "}\n";
  // Dirichlet boundary mask (xsetbound.m:40-53, zero boundary values)
  os << "__device__ __forceinline__ bool xs_dirichlet(int f, int i1, int i2, int i3) {\n  (void)f; (void)i1; (void)i2; (void)i3;\n";
  if (!P.bnd.empty()) {
    for (int f = 0; f < P.F; ++f) {
      std::string cond = "false";
      for (int d = 0; d < P.D; ++d) {
        const char* iv = d == 0 ? "i1" : d == 1 ? "i2" : "i3";
        if (P.N[d] <= 1) continue;
        if (P.bnd[(d * P.F + f) * 2] == 1) cond += std::string(" || ") + iv + " == 0";
        if (P.bnd[(d * P.F + f) * 2 + 1] == 1) cond += std::string(" || ") + iv + " == " + std::to_string(P.N[d] - 1);
      }
      os << "  if (f == " << f << ") return " << cond << ";\n";
    }
  }
  os << "  return false;\n}\n";
  // boundary values: Dirichlet ends (xsetbound.m, later dimensions last) and the xpatch.m patch of
  // the last non-periodic dimension (xpatch.m recomputes it per dimension), in FP64
  os << "#define XS_BVAL " << (P.bvals ? 1 : 0) << "\n";
  os << "__device__ __forceinline__ bool xs_dirichlet_val(int f, int i1, int i2, int i3, const double2* __restrict__ bv, cx& v) {\n"
        "  (void)f; (void)i1; (void)i2; (void)i3; (void)bv; (void)v; bool hit = false;\n";
  if (P.bvals)
    for (int d = 0; d < P.D; ++d) {
      if (P.N[d] <= 1) continue;
      const char* iv = d == 0 ? "i1" : d == 1 ? "i2" : "i3";
      for (int f = 0; f < P.F; ++f)
        for (int e = 0; e < 2; ++e)
          if (P.bnd[(d * P.F + f) * 2 + e] == 1)
            os << "  if (f == " << f << " && " << iv << " == " << (e ? P.N[d] - 1 : 0) << ") { const double2 q = bv["
               << (d * P.F + f) * 2 + e << "]; v = mkcx((real)q.x, (real)q.y); hit = true; }\n";
    }
  os << "  return hit;\n}\n";
  os << "__device__ __forceinline__ cx xs_bpatch(int f, int i1, int i2, int i3, const double2* __restrict__ bv, const double2* __restrict__ da, cx& lp) {\n"
        "  (void)f; (void)i1; (void)i2; (void)i3; (void)bv; (void)da; lp = mkcx((real)0, (real)0);\n";
  {
    int dl = -1;
    for (int d = 0; d < P.D; ++d) {
      bool any = false;
      for (int f = 0; f < P.F; ++f) any = any || P.type(d, f) != 0;
      if (any && P.N[d] > 1) dl = d;
    }
    if (P.bvals && dl >= 0) {
      const char* iv = dl == 0 ? "i1" : dl == 1 ? "i2" : "i3";
      os << "  const double x = (double)" << iv << " * " << fmt(P.dx[dl + 1]) << ", R = " << fmt(P.p.ranges[dl + 1])
         << ";\n";
      for (int f = 0; f < P.F; ++f) {
        const int t = P.type(dl, f);
        const int o = (dl * P.F + f) * 2;
        os << "  if (f == " << f << ") {\n    const double2 b0 = bv[" << o << "], b1 = bv[" << o + 1 << "];\n"
           << "    (void)b0; (void)b1;\n";
        if (t == -3)  // Neumann both ends: b0 x + x^2 db / 2, and db * da
          os << "    const double2 db = make_double2((b1.x - b0.x) / R, (b1.y - b0.y) / R);\n"
                "    const double2 q = da[" << dl * P.F + f << "];\n"
                "    lp = mkcx((real)(db.x * q.x - db.y * q.y), (real)(db.x * q.y + db.y * q.x));\n"
                "    return mkcx((real)(b0.x * x + 0.5 * x * x * db.x), (real)(b0.y * x + 0.5 * x * x * db.y));\n";
        else if (t == -1)  // Dirichlet lower, Neumann upper: b0 + x b1
          os << "    return mkcx((real)(b0.x + x * b1.x), (real)(b0.y + x * b1.y));\n";
        else if (t == 1)  // Neumann lower, Dirichlet upper: b1 + (x - R) b0
          os << "    return mkcx((real)(b1.x + (x - R) * b0.x), (real)(b1.y + (x - R) * b0.y));\n";
        else if (t == 3)  // Dirichlet both ends: linear interpolation
          os << "    return mkcx((real)(b0.x + x * (b1.x - b0.x) / R), (real)(b0.y + x * (b1.y - b0.y) / R));\n";
        os << "  }\n";
      }
      os << "  (void)x; (void)R;\n";
    }
  }
  os << "  return mkcx((real)0, (real)0);\n}\n";
}

// ---------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void ensure(size_t b) {
    if (b <= bytes) return;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    CUDA_CHECK(cudaMalloc(&p, b));
    bytes = b;
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

struct ResidentPlan {
  int G = 1, threads = 32, narr = 2;
  size_t smem = 0;
  bool gfield = false;  // field + scratch in per-CTA device-memory slices (lattice beyond shared memory)
};

// Streaming plan: 2D lattice with NX = RX^2, NY = RY^2 (RX, RY in {8, 16, 32}).
struct StreamPlan {
  int RX = 0, RY = 0, XROWS = 0, TX = 0, OROWS = 0;
  size_t xsmem = 0, ssmem = 0, osmem = 0, tsmem = 0;
  size_t rksmem = 0;  // RK4 row passes: twiddles + two stages per row
  // 3D: z-line tile width, per matrix (x, y, z; forward, inverse) its fold (0 or 1 + parity) and
  // offset in the matrix table, shared memory of the plane passes (to K state, step, final), the
  // z-line pass and the observation pass
  int QT = 0, LSX = 0, LSQ = 0;
  int fold3[6] = {0, 0, 0, 0, 0, 0}, cen3[6] = {0, 0, 0, 0, 0, 0}, par3[6] = {0, 0, 0, 0, 0, 0};
  int moff3[6] = {0, 0, 0, 0, 0, 0};
  size_t psmem3[3] = {0, 0, 0}, zsmem3 = 0, osmem3 = 0;
};

}  // namespace

struct xs_handle {
  Problem P;
  std::string header;     // generated problem header
  std::string source;     // full kernel source
  bool fp64 = true;
  int kind = 1;           // 1 resident, 2 streaming (2D), 3 streaming (3D, DST/DCT)
  ResidentPlan rp;
  // device state
  bool loaded = false;
  CUmodule mod = nullptr;
  CUfunction f_resident = nullptr, f_reduce = nullptr, f_noise = nullptr, f_random = nullptr, f_feat = nullptr;
  CUfunction f_xcomb = nullptr;  // adds the trajectory splits of xs_x_obs
  CUfunction f_xinit = nullptr, f_xnl = nullptr, f_xfinal = nullptr, f_spass = nullptr, f_xobs = nullptr,
             f_scalar = nullptr;
  CUfunction f_xrk[3] = {nullptr, nullptr, nullptr};  // RK4 row passes 1, 2, 3 (streaming)
  DevBuf d_field2;                                      // RK4: second streaming field
  CUfunction f_pinit = nullptr, f_ptok = nullptr, f_pnl = nullptr, f_pfinal = nullptr, f_zpass = nullptr,
             f_pobs = nullptr;  // 3D
  DevBuf d_mat3;                                        // 3D: real transform matrices
  bool tc3 = false;                                     // 3D: plane pass on the tensor cores
  CUfunction f_pnl_tc = nullptr;
  DevBuf d_mat3tc;                                      // its transforms: FP32 B_m[k][n] = M[n][k]
  int grid_p = 0, grid_z = 0, grid_tc = 0;                           // 3D: persistent grids of the plane and z-line passes
  StreamPlan sp;
  int path_kind = 0;
  int force_G = 0, force_threads = 0;  // resident tile fixed by the caller (uneven batch)
  CUfunction f_spass_tma = nullptr;    // column pass fed by TMA (NY <= 256)
  CUfunction f_rc = nullptr;           // fused row pass (one half) + column pass (other half)
  bool fuse = false;                   // run the two halves of the trajectories one pass apart, fused
  bool tma = false;
  CUtensorMap tmap{};                  // field as [rows][2*NX] reals, box [NY][2*TX]
  const void* tmap_ptr = nullptr;
  long long tmap_rows = -1;
  int tma_grid = 0;
  bool sep = false;                    // streaming: L(kx, ky) = Lx(kx) + Ly(ky), 1D propagator tables
  CUfunction f_batch = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t cstream = nullptr;    // copies of the pipelined streaming xs_run_path
  std::vector<cudaEvent_t> pipe_ev;  // its per-group events (copy in done, group done)
  DevBuf d_prop[2], d_prop2[2], d_tmat, d_obs, d_av, d_ain, d_aout, d_status, d_w, d_field, d_redpart, d_pstep,
      d_params, d_gfield, d_twiddle, d_tmp, d_avm, d_bval[2], d_bda[2], d_aft, d_twt, d_raw, d_kfilt, d_rfilt,
      d_opart;
  int bval_n[2] = {0, 0};
  int twt_n = 0;
  void* raw_dev = nullptr;  // raw trajectories of the current resident launch (xs_run_path_raw)
  bool kfilt_up = false;    // k-noise filter tables uploaded
  double pstep_dtr = -1;
  double prop_dtr[2] = {-1, -1}, prop2_dtr[2] = {-1, -1};
  // launch accounting (xs_kernel_stats)
  bool timing = false;
  long long launches[XS_KERNEL_KINDS] = {};
  double kms[XS_KERNEL_KINDS] = {};
  struct Pending {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> event_pool;
  std::vector<int> tmat_off;
  ~xs_handle() {
    for (auto& p : pending) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    for (auto e : event_pool) cudaEventDestroy(e);
    for (auto e : pipe_ev) cudaEventDestroy(e);
    if (mod && driver().unload) driver().unload(mod);
    if (stream) cudaStreamDestroy(stream);
    if (cstream) cudaStreamDestroy(cstream);
  }
};

namespace {

// Tiles of the line transforms when the field lives in device memory: lines
// per tile TL (a divisor of the line count that keeps the three tile buffers -
// current, scratch, next in flight - within ~64 KB) and padded row stride LSP,
// per space dimension; elems = the larger tile buffer in complex elements.
void tile_plan(const Problem& P, bool fp64, int tl[3], int lsp[3], size_t& elems) {
  const size_t cxs = fp64 ? 16 : 8, cap = 64 * 1024;
  elems = 0;
  int sd = 1;
  for (int d = 0; d < 3; ++d) {
    tl[d] = lsp[d] = 1;
    const int nd = d < P.D ? P.N[d] : 1;
    if (nd > 1) {
      const int lines = sd == 1 ? P.NS / nd : sd;  // lines per (g, f) group (d = 0) or per line group
      int best = 1;
      for (int t = 1; t <= (sd == 1 ? lines : std::min(lines, 32)); ++t) {
        if (lines % t) continue;
        const int lp = t % 2 ? t : t + 1;
        if (3 * (size_t)nd * lp * cxs > cap) break;
        best = t;
      }
      tl[d] = best;
      lsp[d] = best % 2 ? best : best + 1;
      elems = std::max(elems, (size_t)nd * lsp[d]);
    }
    if (d < P.D) sd *= P.N[d];
  }
}

// Field-sized complex arrays of the k-filtered noise: the current and the
// first coarse draw (ceil(NK/F) chunks each), then the k-filtered randoms, then
// the auxiliary cell (ceil(NA/F) chunks).
int knarr(const Problem& P) {
  return 2 * ((P.NK + P.F - 1) / P.F) + (P.NKV + P.F - 1) / P.F + (P.NA + P.F - 1) / P.F;
}

bool fft_dim(const Problem& P, int d);

// Reals of the shared-memory copy of a real (DST/DCT) transform matrix used by the tiled
// transforms when the field lives in device memory: the largest N_d^2 over such dimensions.
size_t msm_reals(const Problem& P) {
  size_t m = 0;
  for (int d = 0; d < P.D; ++d) {
    if (P.N[d] < 2 || fft_dim(P, d)) continue;
    bool real_m = true;
    for (int f = 0; f < P.F && real_m; ++f) real_m = P.type(d, f) != 0;
    if (real_m) m = std::max(m, (size_t)P.N[d] * P.N[d]);
  }
  return m;
}

// MP with its midpoint iterations fused per site (noise in registers); not
// possible when the drift reads neighbouring sites.
bool lean_mp(const Problem& P) { return P.p.method == XS_METHOD_MP && !P.dstencil && P.NA == 0; }

size_t resident_smem(const xs_handle& h, int G, int narr) {
  const Problem& P = h.P;
  size_t cxs = h.fp64 ? 16 : 8, rs = h.fp64 ? 8 : 4;
  size_t nred = std::max(P.nred, 1);
  size_t nws = std::max(P.NW, 1);
  size_t warr = lean_mp(P) ? 0 : 2;  // fused MP keeps its noise in registers
  size_t tiles = 0;
  if (narr == 0) warr = 0;  // field in device memory: the noise arrays live in the CTA's slice too
  if (narr > 0 && P.kobs) narr += 1;  // the k-space copy of the field for transformed observables
  if (narr > 0) narr += knarr(P);      // k-filtered noise arrays (in the slice when the field is in device memory)
  size_t ms_bytes = 0;
  if (narr == 0) {  // field in device memory: two transform tiles (and a real matrix) in shared memory
    int tl[3], lsp[3];
    tile_plan(P, h.fp64, tl, lsp, tiles);
    ms_bytes = (msm_reals(P) * rs + 15) / 16 * 16;
  }
  return (size_t)narr * G * P.F * P.NS * cxs + 3 * tiles * cxs + ms_bytes + (size_t)G * nred * cxs + 32 * 2 * nred * 8 +
         warr * (size_t)G * nws * P.NS * rs;
}

int method_arrays(const Problem& P) {
  switch (P.p.method) {
    case XS_METHOD_MP: return lean_mp(P) ? 2 : 3;  // field + scratch (fused), or + a0 copy
    case XS_METHOD_RK4: return 5;
    case XS_METHOD_EULER: return 2;
    case XS_METHOD_RK2: return 3;
    default: return 3;
  }
}

void plan_resident(xs_handle& h, int total_traj) {
  const Problem& P = h.P;
  ResidentPlan rp;
  rp.narr = method_arrays(P);
  const size_t limit = 200 * 1024;
  if (resident_smem(h, 1, rp.narr) > limit) {
    // lattice beyond shared memory: one trajectory per CTA, field, scratch and noise arrays in device memory
    if (h.force_G > 1) raise(XS_ERR_UNSUPPORTED, "lattices beyond shared memory take one trajectory per CTA");
    rp.gfield = true;
    rp.G = 1;
    rp.threads = h.force_threads ? h.force_threads : 512;
    rp.smem = resident_smem(h, 1, 0);
    h.rp = rp;
    return;
  }
  if (h.force_G > 0) {
    if (resident_smem(h, h.force_G, rp.narr) > limit) raise(XS_ERR_UNSUPPORTED, "tile does not fit in shared memory");
    if (h.force_threads % 32 || h.force_threads < 0 || h.force_threads > 1024)
      raise(XS_ERR_ARG, "threads per CTA must be a multiple of 32, at most 1024");
    rp.G = h.force_G;
    const int items = rp.G * P.NS * P.F;
    rp.threads = h.force_threads ? h.force_threads : std::min(256, std::max(32, (items + 31) / 32 * 32));
    rp.smem = resident_smem(h, rp.G, rp.narr);
    h.rp = rp;
    return;
  }
  int best = 1;
  for (int G = 1; G <= P.E1 && G <= 1024; ++G) {
    if (P.E1 % G) continue;
    if ((size_t)G * P.NS > 1024 && G > 1) break;
    if (resident_smem(h, G, rp.narr) > limit) break;
    if (G > 1 && total_traj / G < 296 && P.NS > 1) break;
    best = G;
  }
  rp.G = best;
  int items = rp.G * P.NS * P.F;
  rp.threads = std::min(256, std::max(32, (items + 31) / 32 * 32));
  rp.smem = resident_smem(h, rp.G, rp.narr);
  h.rp = rp;
}

// A space dimension (0-based d) is transformed by the shared-memory Stockham
// FFT when it is periodic for every field and its length is a power of two.
bool fft_dim(const Problem& P, int d) {
  if (d >= P.D) return false;
  const int n = P.N[d];
  if (n < 2 || (n & (n - 1)) || n > 4096) return false;
  for (int f = 0; f < P.F; ++f)
    if (P.type(d, f) != 0) return false;
  return true;
}

// Stage list of a shared-memory tile (TL lines of length n, row stride lsp);
// returns the buffer that holds the result.
std::string gen_fft_tile_stages(int D, int n, int tl, int lsp) {
  int k = 0;
  while ((1 << k) < n) ++k;
  const int S = (k + 2) / 3;
  std::vector<int> bits(S, k / S);
  for (int i = 0; i < k % S; ++i) ++bits[i];
  std::ostringstream os;
  os << "template <> __device__ __forceinline__ cx* xs_fft_tile_d<" << D
     << ">(cx* S, cx* S2, const cx* __restrict__ tw, int inv) { ";
  int nsp = 1;
  for (int i = 0; i < S; ++i) {
    const int R = 1 << bits[i];
    os << "xs_fft_tstage<" << n << ", " << R << ", " << nsp << ", " << (i == 0 ? "true" : "false") << ", "
       << (i == S - 1 ? "true" : "false") << ", " << tl << ", " << lsp << ">(" << (i % 2 ? "S2, S" : "S, S2")
       << ", tw, inv); __syncthreads(); ";
    nsp *= R;
  }
  os << "return " << (S % 2 ? "S2" : "S") << "; } ";
  return os.str();
}

// Stockham stage sequence of one dimension (length n, site stride sd): an even
// number of stages (so the result lands back in X) of radix 2, 4 or 8 with
// the larger radices first; a lone radix-2 stage is followed by a copy.
std::string gen_fft_stages(int D, int n, int sd) {
  int k = 0;
  while ((1 << k) < n) ++k;
  int S = (k + 2) / 3;
  if (S % 2 == 1 && k >= S + 1) ++S;
  std::vector<int> bits(S, k / S);
  for (int i = 0; i < k % S; ++i) ++bits[i];
  std::ostringstream os;
  os << "template <> __device__ __forceinline__ void xs_fft_d<" << D
     << ">(cx* X, cx* T, const cx* __restrict__ tw, int inv) { ";
  int nsp = 1;
  for (int i = 0; i < S; ++i) {
    const int R = 1 << bits[i];
    os << "xs_fft_stage<" << n << ", " << sd << ", " << R << ", " << nsp << ", " << (i == 0 ? "true" : "false") << ", "
       << (i == S - 1 ? "true" : "false") << ">(" << (i % 2 ? "T, X" : "X, T") << ", tw, inv); __syncthreads(); ";
    nsp *= R;
  }
  if (S % 2)
    os << "for (int i = threadIdx.x; i < XS_G * XS_F * XS_NS; i += blockDim.x) X[i] = T[i]; __syncthreads(); ";
  os << "} ";
  return os.str();
}

// True when the 2D linear operator is additively separable, L(kx, ky) =
// Lx(kx) + Ly(ky), to FP64 rounding (then exp(L dt) factors into 1D tables).
bool separable(const Problem& P) {
  if (P.D != 2 || P.Lc != 1 || !P.has_linear) return false;
  const int N1 = P.N[0], N2 = P.N[1];
  double mx = 0;
  for (auto& v : P.L) mx = std::max(mx, std::abs(v));
  for (int i2 = 0; i2 < N2; ++i2)
    for (int i1 = 0; i1 < N1; ++i1) {
      const cd d = P.L[(size_t)i2 * N1 + i1] - (P.L[i1] + P.L[(size_t)i2 * N1] - P.L[0]);
      if (std::abs(d) > 1e-13 * mx + 1e-300) return false;
    }
  return true;
}

int isqrt_pow2(int n) {
  for (int r : {8, 16, 32})
    if (r * r == n) return r;
  return 0;
}

// Reason why the streaming path cannot run this problem, or "" when it can.
// Observables, noises and drifts the streaming passes do not cover (2D and 3D).
std::string stream_common_blocker(const Problem& P) {
  if (!P.has_linear) return "the streaming path needs p.linear";
  for (auto& o : P.obs)
    if (o.spatial && !o.gen.reductions.empty()) return "site observables that use Int/Ave are not streamed";
  if (P.kobs) return "k-space observables (p.transforms) are not streamed";
  if (P.spec) return "time-spectrum observables (p.transforms{n}(1)) are not streamed";
  if (P.NK || P.NKV) return "k-filtered noises are not streamed";
  if (P.NA) return "auxiliary fields (p.define) are not streamed";
  if (P.stencil) return "observables with D1/D2 finite differences are not streamed";
  if (P.dstencil) return "drifts with D1/D2 finite differences are not streamed";
  return "";
}

std::string stream_blocker(const Problem& P) {
  if (P.D != 2) return "the streaming path covers two space dimensions";
  if (!isqrt_pow2(P.N[0]) || !isqrt_pow2(P.N[1])) return "streaming lattices need 64, 256 or 1024 points per dimension";
  for (int v : P.bnd)
    if (v) return "the streaming path covers periodic boundaries";
  if (P.p.method != XS_METHOD_MP && P.p.method != XS_METHOD_RK4) return "the streaming path integrates with MP or RK4";
  return stream_common_blocker(P);
}

// 3D lattices with a DST/DCT transform in every dimension (xs_stream3.cuh).
std::string stream3_blocker(const Problem& P) {
  if (P.D != 3) return "the 3D streaming path covers three space dimensions";
  for (int d = 0; d < 3; ++d)
    if (P.N[d] < 8 || P.N[d] > 64 || P.N[d] % 4)
      return "3D streaming lattices need 8 to 64 points per dimension, a multiple of 4";
  if ((P.N[0] * P.N[1]) % 64) return "3D streaming needs N1*N2 to be a multiple of 64";
  if (P.F != 1) return "the 3D streaming path covers one field component";
  for (int d = 0; d < 3; ++d)
    if (P.type(d, 0) == 0) return "the 3D streaming path covers non-periodic (DST/DCT) boundaries in every dimension";
  if (P.p.method != XS_METHOD_MP) return "the 3D streaming path integrates with MP";
  if (P.bvals) return "boundary values (p.boundfun) are not streamed";
  return stream_common_blocker(P);
}

// Straight-line radix-2 DIT DFT of R points (forward, exp(-2 pi i n k / R)),
// emitted with literal twiddles; trivial twiddles (1, -i) cost no multiply.  A
// butterfly u +- W v with a general twiddle W = c + i s is evaluated as
// u +- c (v (1 + i s/c)) (or u +- s (v (c/s + i)) when |s| > |c|, keeping the
// ratio within [-1, 1]): two fused multiply-adds for the scaled v and four for
// the two outputs, instead of a complex multiply (four operations) and four
// additions.
std::string gen_dft(int R) {
  std::ostringstream os;
  int bits = 0;
  while ((1 << bits) < R) ++bits;
  auto rev = [&](int i) {
    int r = 0;
    for (int b = 0; b < bits; ++b)
      if (i & (1 << b)) r |= 1 << (bits - 1 - b);
    return r;
  };
  os << "template <> __device__ __forceinline__ void xs_dftR<" << R << ">(cx (&v)[" << R << "]) {\n";
  std::vector<std::string> cur(R);
  for (int i = 0; i < R; ++i) cur[i] = "v[" + std::to_string(rev(i)) + "]";
  int tmp = 0;
  for (int len = 2; len <= R; len <<= 1) {
    std::vector<std::string> nxt(R);
    for (int i = 0; i < R; i += len)
      for (int k = 0; k < len / 2; ++k) {
        int u = i + k, w = i + k + len / 2;
        std::string tw = "q" + std::to_string(tmp++);
        std::string a = "q" + std::to_string(tmp++), b = "q" + std::to_string(tmp++);
        const std::string& U = cur[u];
        const std::string& V = cur[w];
        if (k == 0 || 4 * k == len) {
          if (k == 0) os << "  const cx " << tw << " = " << V << ";\n";
          else os << "  const cx " << tw << " = mkcx(" << V << ".im, -" << V << ".re);\n";
          os << "  const cx " << a << " = " << U << " + " << tw << ";\n";
          os << "  const cx " << b << " = " << U << " - " << tw << ";\n";
        } else {
          const double c = std::cos(2 * M_PI * k / len), s = -std::sin(2 * M_PI * k / len);
          auto snap = [](double r) { return std::fabs(std::fabs(r) - 1.0) < 1e-14 ? (r > 0 ? 1.0 : -1.0) : r; };
          double f;
          if (std::fabs(c) >= std::fabs(s)) {  // W v = c (v (1 + i tau)), tau = s / c
            const double tau = snap(s / c);
            f = c;
            os << "  const cx " << tw << " = mkcx(xs_fma((real)" << fmt(-tau) << ", " << V << ".im, " << V
               << ".re), xs_fma((real)" << fmt(tau) << ", " << V << ".re, " << V << ".im));\n";
          } else {  // W v = s (v (sigma + i)), sigma = c / s
            const double sig = snap(c / s);
            f = s;
            os << "  const cx " << tw << " = mkcx(xs_fma((real)" << fmt(sig) << ", " << V << ".re, -" << V
               << ".im), xs_fma((real)" << fmt(sig) << ", " << V << ".im, " << V << ".re));\n";
          }
          os << "  const cx " << a << " = mkcx(xs_fma((real)" << fmt(f) << ", " << tw << ".re, " << U
             << ".re), xs_fma((real)" << fmt(f) << ", " << tw << ".im, " << U << ".im));\n";
          os << "  const cx " << b << " = mkcx(xs_fma((real)" << fmt(-f) << ", " << tw << ".re, " << U
             << ".re), xs_fma((real)" << fmt(-f) << ", " << tw << ".im, " << U << ".im));\n";
        }
        nxt[u] = a;
        nxt[w] = b;
      }
    cur = nxt;
  }
  for (int i = 0; i < R; ++i) os << "  v[" << i << "] = " << cur[i] << ";\n";
  os << "}\n";
  return os.str();
}

void plan_stream(xs_handle& h) {
  const Problem& P = h.P;
  StreamPlan sp;
  sp.RX = isqrt_pow2(P.N[0]);
  sp.RY = isqrt_pow2(P.N[1]);
  sp.XROWS = 256 / sp.RX;
  sp.TX = 256 / sp.RY;
  sp.OROWS = std::max(1, 64 / sp.RX);
  size_t cxs = h.fp64 ? 16 : 8;
  const size_t xline = std::max<size_t>((size_t)P.F * sp.RX * sp.RX, (size_t)sp.RX * (sp.RX + 1));
  // twiddle tables: W and W/N (2 R^2 elements, xs_fill_twiddles)
  sp.xsmem = (2 * sp.RX * sp.RX + sp.XROWS * xline) * cxs;
  sp.ssmem = (size_t)(2 * sp.RY * sp.RY + sp.TX * sp.RY * sp.RY) * cxs;
  // TMA column pass: two [NY][TX] stages (each the transpose scratch of its tile), twiddles, two
  // mbarriers, alignment slack
  sp.tsmem = 2 * (size_t)P.N[1] * sp.TX * cxs + 2 * (size_t)sp.RY * sp.RY * cxs + 16 + 128;
  sp.osmem = (size_t)(2 * sp.RX * sp.RX + sp.OROWS * sp.RX * (sp.RX + 1)) * cxs;
  sp.rksmem = (2 * sp.RX * sp.RX + 2 * sp.XROWS * xline) * cxs;
  if (P.N[1] % sp.XROWS || P.N[1] % sp.OROWS || P.N[0] % sp.TX)
    raise(XS_ERR_SHAPE, "internal: streaming tile sizes do not divide the lattice");
  h.sp = sp;
}

// 3D streaming plan: matrix i = 2 d + inverse (d = x, y, z) at offset moff3[i] of the table, folded
// when it is mirror-symmetric; shared memory of each pass as xs_stream3.cuh lays it out (matrices
// in `real`, then the plane [N2][LSX] or the z-line tile [N3][LSQ] in complex `real`; the row
// strides are padded by 2 in FP32, keeping rows 16-byte aligned, and by 1 in FP64).
void plan_stream3(xs_handle& h) {
  const Problem& P = h.P;
  StreamPlan sp;
  sp.QT = 64;
  sp.LSX = P.N[0] + (h.fp64 ? 1 : 2);
  sp.LSQ = sp.QT + (h.fp64 ? 1 : 2);
  const size_t rs = h.fp64 ? 8 : 4, cxs = 2 * rs;
  int off = 0;
  size_t msize[6];
  for (int i = 0; i < 6; ++i) {
    const int d = i / 2, n = P.N[d];
    sp.moff3[i] = off;
    off += n * n;
    const FoldInfo f = fold_info(transform_matrix(P.type(d, 0), i % 2 == 1, n), n);
    sp.fold3[i] = f.kind;
    sp.cen3[i] = f.c;
    sp.par3[i] = f.p;
    msize[i] = (size_t)(f.kind ? n / 2 : n) * n;
  }
  const size_t plane = (size_t)P.N[1] * sp.LSX * cxs;
  // plane and z-line passes: two buffers (the current plane or tile and the next, in flight)
  sp.psmem3[0] = (msize[0] + msize[2]) * rs + 2 * plane;
  sp.psmem3[1] = (msize[0] + msize[1] + msize[2] + msize[3]) * rs + 2 * plane;
  sp.psmem3[2] = (msize[1] + msize[3]) * rs + 2 * plane;
  sp.osmem3 = (msize[1] + msize[3]) * rs + plane;
  sp.zsmem3 = (msize[4] + msize[5]) * rs + 2 * (size_t)P.N[2] * sp.LSQ * cxs;
  if ((P.N[0] * P.N[1]) % sp.QT) raise(XS_ERR_SHAPE, "internal: z-line tiles do not divide the plane");
  for (size_t b : {sp.psmem3[0], sp.psmem3[1], sp.psmem3[2], sp.zsmem3, sp.osmem3})
    if (b > 227 * 1024) raise(XS_ERR_UNSUPPORTED, "3D streaming passes need more than 227 KB of shared memory");
  h.sp = sp;
}

void emit_common_header(const xs_handle& h, std::ostringstream& os) {
  const Problem& P = h.P;
  os << "// generated problem header\n";
  os << "#define XS_FP64 " << (h.fp64 ? 1 : 0) << "\n#define XS_REAL " << (h.fp64 ? "double" : "float") << "\n";
  os << xs_kernel_source_prelude << "\n";
  os << "#define XS_F " << P.F << "\n#define XS_NW " << P.NW << "\n#define XS_NWS " << std::max(P.NW, 1)
     << "\n#define XS_NV " << P.NV << "\n#define XS_ND " << P.D << "\n";
  os << "#define XS_N1 " << P.N[0] << "\n#define XS_N2 " << P.N[1] << "\n#define XS_N3 " << P.N[2]
     << "\n#define XS_NS " << P.NS << "\n";
  for (int d = 0; d < 3; ++d) {
    double o = d < P.D ? P.p.origins[d + 1] : 0.0;
    double dx = d < P.D ? P.dx[d + 1] : 0.0;
    os << "#define XS_O" << d + 1 << " " << fmt(o) << "\n#define XS_DX" << d + 1 << " " << fmt(dx) << "\n";
  }
  os << "#define XS_METHOD " << P.p.method << "\n#define XS_ITER " << P.p.iterations << "\n";
  os << "#define XS_HAS_PROP " << ((P.has_linear && P.D > 0) ? 1 : 0) << "\n#define XS_PROP_COMPS " << P.Lc << "\n";
  os << "#define XS_SETBOUND " << (P.setbound ? 1 : 0) << "\n";
  os << "#define XS_NK " << P.NK << "\n#define XS_NKV " << P.NKV << "\n#define XS_NKC " << (P.NK + P.F - 1) / P.F
     << "\n#define XS_NKVC " << (P.NKV + P.F - 1) / P.F << "\n#define XS_KNARR " << knarr(P) << "\n";
  os << xs_kernel_source_noise << "\n";
}

void build_source(xs_handle& h) {
  Problem& P = h.P;
  std::ostringstream fns;
  generate_functions(P, fns);  // fixes P.nred / nout_* before the launch plan
  if (P.bvals && (P.stencil || P.dstencil))
    raise(XS_ERR_UNSUPPORTED, "D1/D2 use zero boundary values on the device: not combined with p.boundfun values");
  const bool fits = resident_smem(h, 1, method_arrays(P)) <= 200 * 1024;
  const std::string why = P.D == 3 ? stream3_blocker(P) : stream_blocker(P);
  // too large for shared memory: the streaming path when it covers the problem, else the resident
  // path with the field in device memory (MP)
  if (h.path_kind == 2 || (h.path_kind == 0 && !fits && why.empty())) {
    if (!why.empty()) {
      if (!fits) raise(XS_ERR_UNSUPPORTED, "field too large for the resident path, and " + why);
      raise(XS_ERR_UNSUPPORTED, why);
    }
    if (P.D == 3) {
      h.kind = 3;
      plan_stream3(h);
      std::ostringstream os;
      emit_common_header(h, os);
      os << "#define XS3_QT " << h.sp.QT << "\n#define XS3_LSX " << h.sp.LSX << "\n#define XS3_LSQ " << h.sp.LSQ << "\n";
      for (int i = 0; i < 6; ++i)
        os << "#define XS3_MOFF" << i << " " << h.sp.moff3[i] << "\n#define XS3_FOLD" << i << " " << h.sp.fold3[i]
           << "\n#define XS3_CEN" << i << " " << h.sp.cen3[i] << "\n#define XS3_PAR" << i << " " << h.sp.par3[i] << "\n";
      // plane pass on the tensor cores (xs_stream3_tc.cuh): 64 x 64 planes, FP32 fields;
      // XSPDE_B200_TC3=0 keeps the CUDA-core plane pass
      const char* tce = getenv("XSPDE_B200_TC3");
      h.tc3 = !h.fp64 && P.N[0] == 64 && P.N[1] == 64 && P.F == 1 && !(tce && *tce == '0');
      os << "#define XS3_TC " << (h.tc3 ? 1 : 0) << "\n";
      os << fns.str();
      os << xs_kernel_source_stream_common << "\n" << xs_kernel_source_stream3 << "\n" << xs_kernel_source_stream3_tc
         << "\n";
      h.source = os.str();
      return;
    }
    h.kind = 2;
    plan_stream(h);
    h.sep = separable(P);
    std::ostringstream os;
    emit_common_header(h, os);
    os << "#define XS_SEP " << (h.sep ? 1 : 0) << "\n";
    os << "#define XS_FFT_RX " << h.sp.RX << "\n#define XS_FFT_RY " << h.sp.RY << "\n#define XS_OBS_ROWS " << h.sp.OROWS
       << "\n";
    os << fns.str();
    os << "template <int R> __device__ __forceinline__ void xs_dftR(cx (&v)[R]);\n";
    os << gen_dft(h.sp.RX);
    if (h.sp.RY != h.sp.RX) os << gen_dft(h.sp.RY);
    os << xs_kernel_source_stream_common << "\n" << xs_kernel_source_stream << "\n";
    h.source = os.str();
    return;
  }
  h.kind = 1;
  plan_resident(h, P.E1 * P.p.ensembles[1] * P.p.ensembles[2]);
  std::ostringstream os;
  emit_common_header(h, os);
  os << "#define XS_G " << h.rp.G << "\n#define XS_THREADS " << h.rp.threads << "\n#define XS_NARR " << h.rp.narr << "\n";
  os << "#define XS_KARR " << (P.kobs ? 1 : 0) << "\n";
  os << "#define XS_LEAN " << (lean_mp(P) ? 1 : 0) << "\n#define XS_WARR " << (lean_mp(P) ? 0 : 2)
     << "\n#define XS_GFIELD " << (h.rp.gfield ? 1 : 0) << "\n";
  os << "#define XS_SMEM_BYTES " << h.rp.smem << "\n";
  {
    std::string stages;
    int sd = 1;
    for (int d = 0; d < 3; ++d) {
      const bool f = fft_dim(P, d);
      os << "#define XS_FFTD" << d + 1 << " " << (f ? 1 : 0) << "\n";
      if (f) stages += gen_fft_stages(d + 1, P.N[d], sd);
      if (d < P.D) sd *= P.N[d];
    }
    os << "#define XS_FFT_STAGES " << stages << "\n";
    int tl[3] = {1, 1, 1}, lsp[3] = {1, 1, 1};
    size_t elems = 0;
    std::string tstages;
    if (h.rp.gfield) {
      tile_plan(P, h.fp64, tl, lsp, elems);
      for (int d = 0; d < 3; ++d)
        if (fft_dim(P, d)) tstages += gen_fft_tile_stages(d + 1, P.N[d], tl[d], lsp[d]);
    }
    for (int d = 0; d < 3; ++d) os << "#define XS_TL" << d + 1 << " " << tl[d] << "\n#define XS_LSP" << d + 1 << " " << lsp[d] << "\n";
    os << "#define XS_TILE_ELEMS " << elems << "\n#define XS_FFT_TILE_STAGES " << tstages << "\n";
    os << "#define XS_MSM " << (h.rp.gfield ? msm_reals(P) : 0) << "\n";
    for (int d = 0; d < 3; ++d) {  // real transform matrices: every field non-periodic along d
      bool real_m = d < P.D;
      for (int f = 0; f < P.F && real_m; ++f) real_m = P.type(d, f) != 0;
      os << "#define XS_REALM" << d + 1 << " " << (real_m ? 1 : 0) << "\n";
      // mirror symmetry M[N-1-n][k] = (-1)^(k+p) M[n][k] of every matrix along d, one parity p for
      // all (DCT-I and DCT-II: p = 0; DST-I on xSPDE's endpoint-inclusive lattice: p = 1; DCT-III
      // has none): the tiled dense transform folds each line and halves its multiply-adds.
      // XS_FOLD = 1 + p, or 0.
      int fold = (real_m && h.rp.gfield && !fft_dim(P, d) && P.N[d] % 4 == 0) ? -1 : 0;
      for (int f = 0; f < P.F && fold; ++f)
        for (int dir = 0; dir < 2 && fold; ++dir) {
          const int found = fold_parity(transform_matrix(P.type(d, f), dir == 1, P.N[d]), P.N[d]);
          fold = (found && (fold < 0 || fold == found)) ? found : 0;
        }
      os << "#define XS_FOLD" << d + 1 << " " << (fold > 0 ? fold : 0) << "\n";
    }
  }
  os << fns.str();
  os << xs_kernel_source_resident << "\n";
  h.source = os.str();
}

void upload_params(xs_handle& h) {
  const Problem& P = h.P;
  if (P.runtime_defaults.empty()) return;
  h.d_params.ensure(P.runtime_defaults.size() * 8);
  CUDA_CHECK(cudaMemcpy(h.d_params.p, P.runtime_defaults.data(), P.runtime_defaults.size() * 8,
                        cudaMemcpyHostToDevice));
}

void load_module(xs_handle& h) {
  if (h.loaded) return;
  ensure_device();
  upload_params(h);
  if (h.kind == 3) {
    trace("load: compile xs_stream3");
    std::string cubin = nvrtc_compile(h.source, "xs_stream3", nullptr);
    Driver& d = driver();
    trace("load: module (%zu bytes)", cubin.size());
    cu_check(d.load(&h.mod, cubin.data()), "cuModuleLoadData");
    const StreamPlan& sp = h.sp;
    struct {
      CUfunction* f;
      const char* name;
      size_t smem;
    } fns[] = {{&h.f_pinit, "xs_p_init", 0}, {&h.f_ptok, "xs_p_tok", sp.psmem3[0]}, {&h.f_pnl, "xs_p_nl", sp.psmem3[1]},
               {&h.f_pfinal, "xs_p_final", sp.psmem3[2]}, {&h.f_zpass, "xs_z_pass", sp.zsmem3},
               {&h.f_pobs, "xs_p_obs", sp.osmem3}, {&h.f_scalar, "xs_stream_scalar", 0},
               {&h.f_xcomb, "xs_x_obs_combine", 0}, {&h.f_noise, "xs_export_noise", 0},
               {&h.f_random, "xs_export_random", 0}, {&h.f_feat, "xs_noise_features", 0}};
    for (auto& f : fns) {
      cu_check(d.getfn(f.f, h.mod, f.name), f.name);
      if (f.smem > 48 * 1024)
        cu_check(d.setattr(*f.f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)f.smem), f.name);
    }
    {  // persistent grids: every SM filled with as many CTAs as fit
      int dev = 0, sms = 0, occ_p = 0, occ_z = 0;
      CUDA_CHECK(cudaGetDevice(&dev));
      CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      trace("load: occupancy (plane pass %zu B, z-line pass %zu B of shared memory)", sp.psmem3[1], sp.zsmem3);
      cu_check(d.occupancy(&occ_p, h.f_pnl, 256, sp.psmem3[1]), "occupancy");
      cu_check(d.occupancy(&occ_z, h.f_zpass, 256, sp.zsmem3), "occupancy");
      trace("load: %d SMs, %d plane-pass and %d z-line-pass CTAs per SM", sms, occ_p, occ_z);
      if (occ_p < 1 || occ_z < 1) raise(XS_ERR_UNSUPPORTED, "3D streaming passes cannot be resident on an SM");
      h.grid_p = sms * occ_p;
      h.grid_z = sms * occ_z;
    }
    CUDA_CHECK(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    {  // the reference's transforms as real matrices M[n*N + k], FP64-built, folded halves packed
      const Problem& P = h.P;
      std::vector<double> all;
      for (int i = 0; i < 6; ++i) {
        const int dd = i / 2, n = P.N[dd];
        const auto M = transform_matrix(P.type(dd, 0), i % 2 == 1, n);
        FoldInfo f;
        f.kind = sp.fold3[i];
        f.c = sp.cen3[i];
        f.p = sp.par3[i];
        std::vector<double> pk = pack_folded(M, n, f);
        pk.resize((size_t)n * n, 0.0);  // each matrix keeps an N x N slot
        all.insert(all.end(), pk.begin(), pk.end());
      }
      if (h.fp64) {
        h.d_mat3.ensure(all.size() * 8);
        CUDA_CHECK(cudaMemcpy(h.d_mat3.p, all.data(), all.size() * 8, cudaMemcpyHostToDevice));
      } else {
        std::vector<float> f32(all.begin(), all.end());
        h.d_mat3.ensure(f32.size() * 4);
        CUDA_CHECK(cudaMemcpy(h.d_mat3.p, f32.data(), f32.size() * 4, cudaMemcpyHostToDevice));
      }
    }
    if (h.tc3) {  // x inverse, y inverse, x forward, y forward as B[k][n] = M[n][k] (xs_stream3_tc.cuh)
      const size_t smem = kTc3Smem;
      cu_check(d.getfn(&h.f_pnl_tc, h.mod, "xs_p_nl_tc"), "xs_p_nl_tc");
      cu_check(d.setattr(h.f_pnl_tc, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem), "xs_p_nl_tc");
      int occ = 0, dev = 0, sms = 0;
      cu_check(d.occupancy(&occ, h.f_pnl_tc, kTc3Threads, smem), "occupancy");
      if (occ < 1) raise(XS_ERR_UNSUPPORTED, "tensor-core plane pass cannot be resident on an SM");
      CUDA_CHECK(cudaGetDevice(&dev));
      CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      h.grid_tc = sms * occ;
      const Problem& P = h.P;
      std::vector<float> bt;
      for (int i : {1, 3, 0, 2}) {
        const int dd = i / 2, n = P.N[dd];
        const auto M = transform_matrix(P.type(dd, 0), i % 2 == 1, n);
        for (int k = 0; k < n; ++k)
          for (int q = 0; q < n; ++q) bt.push_back((float)M[(size_t)q * n + k].real());
      }
      h.d_mat3tc.ensure(bt.size() * 4);
      CUDA_CHECK(cudaMemcpy(h.d_mat3tc.p, bt.data(), bt.size() * 4, cudaMemcpyHostToDevice));
    }
    h.d_status.ensure(sizeof(int));
    h.loaded = true;
    return;
  }
  if (h.kind == 2) {
    std::string cubin = nvrtc_compile(h.source, "xs_stream", nullptr);
    Driver& d = driver();
    cu_check(d.load(&h.mod, cubin.data()), "cuModuleLoadData");
    struct {
      CUfunction* f;
      const char* name;
      size_t smem;
    } fns[] = {{&h.f_xinit, "xs_x_init", h.sp.xsmem}, {&h.f_xnl, "xs_x_nl", h.sp.xsmem},
               {&h.f_xfinal, "xs_x_final", h.sp.xsmem}, {&h.f_spass, "xs_s_pass", h.sp.ssmem},
               {&h.f_xobs, "xs_x_obs", h.sp.osmem}, {&h.f_scalar, "xs_stream_scalar", 0},
               {&h.f_xcomb, "xs_x_obs_combine", 0}};
    cu_check(d.getfn(&h.f_noise, h.mod, "xs_export_noise"), "xs_export_noise");
    cu_check(d.getfn(&h.f_random, h.mod, "xs_export_random"), "xs_export_random");
    {
      // opt-in (measured slower than the plain column pass at this tile size: 1.07 vs 0.94 ms per
      // launch at 4096 trajectories, 24 vs 32 warps per SM)
      const char* e = getenv("XSPDE_B200_TMA");
      h.tma = h.P.N[1] <= 256 && e && *e == '1' && h.P.p.method == XS_METHOD_MP;
      if (h.tma) {
        cu_check(d.getfn(&h.f_spass_tma, h.mod, "xs_s_pass_tma"), "xs_s_pass_tma");
        if (h.sp.tsmem > 48 * 1024)
          cu_check(d.setattr(h.f_spass_tma, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)h.sp.tsmem),
                   "xs_s_pass_tma smem");
        int dev = 0, sms = 0, occ = 0;
        CUDA_CHECK(cudaGetDevice(&dev));
        CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        cu_check(d.occupancy(&occ, h.f_spass_tma, 256, h.sp.tsmem), "occupancy");
        if (occ < 1) raise(XS_ERR_UNSUPPORTED, "TMA column pass cannot be resident on an SM");
        h.tma_grid = sms * occ;
      }
    }
    if (h.P.p.method == XS_METHOD_RK4) {
      const char* names[3] = {"xs_x_rk1", "xs_x_rk2", "xs_x_rk3"};
      for (int i = 0; i < 3; ++i) {
        cu_check(d.getfn(&h.f_xrk[i], h.mod, names[i]), names[i]);
        if (h.sp.rksmem > 48 * 1024)
          cu_check(d.setattr(h.f_xrk[i], CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)h.sp.rksmem), names[i]);
      }
    }
    cu_check(d.getfn(&h.f_feat, h.mod, "xs_noise_features"), "xs_noise_features");
    {
      // opt-in (measured: 1.39 ms per fused launch against 1.41 ms per row + column pass pair at
      // 4096 trajectories of the 256x256 GPE, within run-to-run spread)
      const char* e = getenv("XSPDE_B200_FUSE");
      h.fuse = e && *e == '1';
      cu_check(d.getfn(&h.f_rc, h.mod, "xs_rc_pass"), "xs_rc_pass");
      const size_t rsm = std::max(h.sp.xsmem, h.sp.ssmem);
      if (rsm > 48 * 1024)
        cu_check(d.setattr(h.f_rc, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)rsm), "xs_rc_pass smem");
    }
    for (auto& f : fns) {
      cu_check(d.getfn(f.f, h.mod, f.name), f.name);
      if (f.smem > 48 * 1024)
        cu_check(d.setattr(*f.f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)f.smem), f.name);
    }
    CUDA_CHECK(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    {  // four-step twiddles exp(-2 pi i t k / R^2), [k][t], rows then columns
      std::vector<double> tw;
      for (int R : {h.sp.RX, h.sp.RY})
        for (int k = 0; k < R; ++k)
          for (int t = 0; t < R; ++t) {
            const double ang = -2.0 * M_PI * (double)(t * k) / (double)(R * R);
            tw.push_back(std::cos(ang));
            tw.push_back(std::sin(ang));
          }
      if (h.fp64) {
        h.d_twiddle.ensure(tw.size() * 8);
        CUDA_CHECK(cudaMemcpy(h.d_twiddle.p, tw.data(), tw.size() * 8, cudaMemcpyHostToDevice));
      } else {
        std::vector<float> tf(tw.begin(), tw.end());
        h.d_twiddle.ensure(tf.size() * 4);
        CUDA_CHECK(cudaMemcpy(h.d_twiddle.p, tf.data(), tf.size() * 4, cudaMemcpyHostToDevice));
      }
    }
    h.d_status.ensure(sizeof(int));
    h.loaded = true;
    return;
  }
  std::string cubin = nvrtc_compile(h.source, "xs_resident", nullptr);
  Driver& d = driver();
  cu_check(d.load(&h.mod, cubin.data()), "cuModuleLoadData");
  cu_check(d.getfn(&h.f_resident, h.mod, "xs_resident"), "cuModuleGetFunction(xs_resident)");
  cu_check(d.getfn(&h.f_batch, h.mod, "xs_batch"), "cuModuleGetFunction(xs_batch)");
  cu_check(d.getfn(&h.f_reduce, h.mod, "xs_obs_reduce"), "cuModuleGetFunction(xs_obs_reduce)");
  cu_check(d.getfn(&h.f_noise, h.mod, "xs_export_noise"), "cuModuleGetFunction(xs_export_noise)");
  cu_check(d.getfn(&h.f_random, h.mod, "xs_export_random"), "cuModuleGetFunction(xs_export_random)");
  cu_check(d.getfn(&h.f_feat, h.mod, "xs_noise_features"), "cuModuleGetFunction(xs_noise_features)");
  if (h.rp.smem > 48 * 1024) {
    cu_check(d.setattr(h.f_resident, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)h.rp.smem),
             "cuFuncSetAttribute(max dynamic smem)");
    cu_check(d.setattr(h.f_batch, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)h.rp.smem),
             "cuFuncSetAttribute(max dynamic smem)");
  }
  CUDA_CHECK(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
  // dense transform matrices (per space dim, per component, fwd/inv)
  const Problem& P = h.P;
  std::vector<cd> all;
  h.tmat_off.assign(4, 0);
  for (int d = 0; d < P.D; ++d) {
    h.tmat_off[d + 1] = (int)all.size();
    int n = P.N[d];
    if (n <= 1) continue;
    if (h.kind == 1 && fft_dim(P, d)) {  // Stockham twiddles exp(-2 pi i m / n)
      for (int m = 0; m < n; ++m) all.push_back(std::polar(1.0, -2 * M_PI * (double)m / n));
      continue;
    }
    for (int f = 0; f < P.F; ++f)
      for (int dir = 0; dir < 2; ++dir) {
        auto M = transform_matrix(P.type(d, f), dir == 1, n);
        all.insert(all.end(), M.begin(), M.end());
      }
  }
  if (all.empty()) all.push_back(0);
  if (h.fp64) {
    h.d_tmat.ensure(all.size() * 16);
    CUDA_CHECK(cudaMemcpy(h.d_tmat.p, all.data(), all.size() * 16, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f32(all.size() * 2);
    for (size_t i = 0; i < all.size(); ++i) {
      f32[2 * i] = (float)all[i].real();
      f32[2 * i + 1] = (float)all[i].imag();
    }
    h.d_tmat.ensure(f32.size() * 4);
    CUDA_CHECK(cudaMemcpy(h.d_tmat.p, f32.data(), f32.size() * 4, cudaMemcpyHostToDevice));
  }
  h.d_status.ensure(sizeof(int));
  h.loaded = true;
}

double pass_dtr(const Problem& P, int nc) {
  return (P.p.checks && nc != 2) ? P.dt / (2.0 * P.p.steps) : P.dt / P.p.steps;  // xensemble.m:41-45
}

// exp(L dt) in the layout the kernels read: [Lc][NS] (xpropfactor.m:39), or,
// for a separable streaming problem, ex[kx] = exp(L(kx, 0) dt) followed by
// ey[ky] = exp((L(0, ky) - L(0, 0)) dt).
std::vector<cd> prop_values(const xs_handle& h, double dt) {
  const Problem& P = h.P;
  if (h.kind == 2 && h.sep) {
    const int N1 = P.N[0], N2 = P.N[1];
    std::vector<cd> pr((size_t)N1 + N2);
    for (int i1 = 0; i1 < N1; ++i1) pr[i1] = std::exp(P.L[i1] * dt);
    for (int i2 = 0; i2 < N2; ++i2) pr[(size_t)N1 + i2] = std::exp((P.L[(size_t)i2 * N1] - P.L[0]) * dt);
    return pr;
  }
  std::vector<cd> pr(P.L.size());
  for (size_t i = 0; i < P.L.size(); ++i) pr[i] = std::exp(P.L[i] * dt);
  return pr;
}

const void* ensure_prop(xs_handle& h, int nc) {
  const Problem& P = h.P;
  int slot = nc == 2 ? 1 : 0;
  double dtr = pass_dtr(P, nc);
  if (!P.has_linear) {
    h.d_prop[slot].ensure(16);
    return h.d_prop[slot].p;
  }
  if (h.prop_dtr[slot] == dtr) return h.d_prop[slot].p;
  double dt = dtr / P.p.ipsteps;  // xpropfactor.m:28
  std::vector<cd> pr = prop_values(h, dt);
  h.d_prop[slot].ensure(pr.size() * 16);
  CUDA_CHECK(cudaMemcpy(h.d_prop[slot].p, pr.data(), pr.size() * 16, cudaMemcpyHostToDevice));
  h.prop_dtr[slot] = dtr;
  return h.d_prop[slot].p;
}

struct PathArgsHost {
  int ntraj, ens1, block0, nc, checks, npoints, steps, seq;
  unsigned seed;
  int pad0;
  double wscale, vscale, dtr, t0;
  const void* prop;
  const void* tmat;
  int tmat_off[4];
  const void* a_in;
  void* a_out;
  void* obs;
  int* status;
  int single_step;
  int pad1;
  const double* w_in;
  const double* params;
  void* gfield;
  const void* prop2;
  const void* bval;
  const void* bda;
  int bval_n;
  int pad3;
  void* aft;
  const void* twt;
  int nt;
  int pad4;
  double fscn;
  void* raw;
  const void* kfilt;
  const void* rfilt;
  double kwscale;
  double kvscale;
};

size_t av_stride(const Problem& P) { return (size_t)P.nout_site * P.NS + P.nout_scalar; }

// sites of observable o in the MATLAB av{o} layout: the lattice, the lattice with its reduced
// dimensions of size 1 (a partial Int/Ave), or one
size_t obs_sites(const Problem& P, const ObsInfo& o) {
  if (!o.spatial) return 1;
  if (!o.partial) return P.NS;
  size_t n = 1;
  for (int d = 0; d < P.D; ++d) n *= o.pw[d] > 0 ? 1 : (size_t)P.N[d];
  return n;
}

bool any_partial(const Problem& P) {
  for (auto& o : P.obs)
    if (o.partial) return true;
  return false;
}

size_t av_doubles_per_block(const Problem& P) {
  size_t n = 0;
  for (auto& o : P.obs) n += (size_t)2 * o.lines * P.p.points[0] * obs_sites(P, o);
  return n;
}

cudaEvent_t take_event(xs_handle& h) {
  if (!h.event_pool.empty()) {
    cudaEvent_t e = h.event_pool.back();
    h.event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  CUDA_CHECK(cudaEventCreate(&e));
  return e;
}

void xs_launch(xs_handle& h, int kind, CUfunction f, unsigned gx, unsigned gy, unsigned gz, unsigned bx,
               unsigned smem, cudaStream_t st, void** params, const char* what) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (h.timing) {
    a = take_event(h);
    b = take_event(h);
    CUDA_CHECK(cudaEventRecord(a, st));
  }
  trace("launch %s grid (%u, %u, %u) block %u smem %u", what, gx, gy, gz, bx, smem);
  cu_check(driver().launch(f, gx, gy, gz, bx, 1, 1, smem, (CUstream)st, params, nullptr), what);
  h.launches[kind]++;
  if (h.timing) {
    CUDA_CHECK(cudaEventRecord(b, st));
    h.pending.push_back({kind, a, b});
  }
}

const void* ensure_prop2(xs_handle& h, int nc);

// Grid of a resident launch over nctas trajectory tiles.  With the field in
// device memory the grid is persistent: one slice per CTA, as many CTAs as
// are resident at once, but no more slices than ~96 MB (L2-sized) when at
// least one slice per SM fits that budget.
int resident_grid(xs_handle& h, CUfunction f, int nctas) {
  if (!h.rp.gfield) return nctas;
  int dev = 0, sms = 0, occ = 0;
  CUDA_CHECK(cudaGetDevice(&dev));
  CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  cu_check(driver().occupancy(&occ, f, h.rp.threads, h.rp.smem), "occupancy");
  const size_t warr = lean_mp(h.P) ? 0 : 2;
  const size_t slice = (size_t)(h.rp.narr + (h.P.kobs ? 1 : 0) + knarr(h.P)) * h.rp.G * h.P.F * h.P.NS * (h.fp64 ? 16 : 8) +
                       warr * h.rp.G * std::max(h.P.NW, 1) * h.P.NS * (h.fp64 ? 8 : 4);
  const int l2 = (int)std::max<size_t>(1, (96u << 20) / slice);
  // slices that fit L2 for a full wave: cap the grid there; larger slices stream from HBM anyway,
  // so take every CTA the SMs can hold (latency hiding)
  const int cap = l2 >= sms ? l2 : sms * std::max(occ, 1);
  const int grid = std::max(1, std::min({nctas, sms * std::max(occ, 1), cap}));
  h.d_gfield.ensure((size_t)grid * slice);
  return grid;
}

// Time spectrum (Simulator/xpath.m:25-106): the field at every step count, Nt = points(1) x steps
// rows per trajectory tile, then points(1) rows of its inverse DFT at the frequencies
// (0..P1-1) - floor(P1/2) (ifft, fftshift and p.specpts), scaled by p.fsc / Nt with
// p.fsc = sqrt(2 pi) / p.dw, p.dw = 2 pi / (ranges(1) + dt) (xpreferences.m:246-249).
// exp(2 pi i k / Nt) in FP64 for the DFT sums.
void spectrum_buffers(xs_handle& h, int nctas, PathArgsHost& a) {
  const Problem& P = h.P;
  const int P1 = P.p.points[0];
  const int nt = P1 * P.p.steps;
  const size_t rows = (size_t)nt + P1;
  const size_t chunks = 1 + (size_t)(P.NA + P.F - 1) / P.F;  // field, then the auxiliary cell
  const size_t bytes = (size_t)nctas * rows * chunks * h.rp.G * P.F * P.NS * (h.fp64 ? 16 : 8);
  size_t free_b = 0, total_b = 0;
  CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
  if (bytes > free_b + h.d_aft.bytes)
    raise(XS_ERR_SHAPE, "the time-spectrum record (" + std::to_string(bytes >> 20) +
                            " MiB) exceeds free device memory: run fewer ensemble blocks per call");
  h.d_aft.ensure(bytes);
  if (h.twt_n != nt) {
    std::vector<double> w(2 * (size_t)nt);
    for (int k = 0; k < nt; ++k) {
      const double ph = 2 * M_PI * (double)k / nt;
      w[2 * k] = std::cos(ph);
      w[2 * k + 1] = std::sin(ph);
    }
    h.d_twt.ensure(w.size() * 8);
    CUDA_CHECK(cudaMemcpy(h.d_twt.p, w.data(), w.size() * 8, cudaMemcpyHostToDevice));
    h.twt_n = nt;
  }
  const double dw = 2 * M_PI / (P.p.ranges[0] + P.dt);
  a.aft = h.d_aft.p;
  a.twt = h.d_twt.p;
  a.nt = nt;
  a.fscn = std::sqrt(2 * M_PI) / dw / nt;
}

// Launch the resident path; av_dev receives [nblocks][npoints][stride] complex.
void launch_resident(xs_handle& h, int first_block, int nblocks, int nc, const void* a_in_dev, void* av_dev,
                     void* a_out_dev, cudaStream_t st) {
  const Problem& P = h.P;
  const int total = nblocks * P.E1;
  const int G = h.rp.G;
  const int nctas = total / G;
  const size_t stride = av_stride(P);
  const int npts = P.p.points[0];
  h.d_obs.ensure(std::max<size_t>(1, (size_t)npts * nctas * stride) * 16);
  PathArgsHost a{};
  a.ntraj = total;
  a.ens1 = P.E1;
  a.block0 = first_block;
  a.nc = nc;
  a.checks = P.p.checks;
  a.npoints = npts;
  a.steps = P.p.steps;
  a.seq = P.p.sequence;
  a.seed = (unsigned)(P.p.seed & 0xffffffffu);
  a.wscale = std::sqrt(P.nscale * P.noisefactor);  // xnoise.m:32
  a.vscale = std::sqrt(P.noisefactor);              // xrandom.m:22
  a.dtr = pass_dtr(P, nc);
  a.t0 = P.p.origins[0];
  a.prop = ensure_prop(h, nc);
  a.prop2 = ensure_prop2(h, nc);
  if (P.bvals) {
    const int slot = nc == 2 ? 1 : 0;
    if (!h.bval_n[slot]) raise(XS_ERR_ARG, "boundary values of this check pass were not set (xs_set_boundary_values)");
    a.bval = h.d_bval[slot].p;
    a.bda = h.d_bda[slot].p;
    a.bval_n = h.bval_n[slot];
  }
  a.tmat = h.d_tmat.p;
  for (int i = 0; i < 4; ++i) a.tmat_off[i] = h.tmat_off[i];
  a.a_in = a_in_dev;
  a.a_out = a_out_dev;
  a.obs = h.d_obs.p;
  a.status = (int*)h.d_status.p;
  a.params = (const double*)h.d_params.p;
  if (P.spec) spectrum_buffers(h, nctas, a);
  a.raw = h.raw_dev;
  if (P.NK || P.NKV) {
    // k-filtered noise (xnoise.m:43) and randoms (xrandom.m:27): knoisefactor = prod(space points) / dv
    if (!h.kfilt_up) {
      if (!P.kfilt.empty()) {
        h.d_kfilt.ensure(P.kfilt.size() * 8);
        CUDA_CHECK(cudaMemcpy(h.d_kfilt.p, P.kfilt.data(), P.kfilt.size() * 8, cudaMemcpyHostToDevice));
      }
      if (!P.rfilt.empty()) {
        h.d_rfilt.ensure(P.rfilt.size() * 8);
        CUDA_CHECK(cudaMemcpy(h.d_rfilt.p, P.rfilt.data(), P.rfilt.size() * 8, cudaMemcpyHostToDevice));
      }
      h.kfilt_up = true;
    }
    const double kf = (double)P.NS / P.dv;
    a.kfilt = P.kfilt.empty() ? nullptr : h.d_kfilt.p;
    a.rfilt = P.rfilt.empty() ? nullptr : h.d_rfilt.p;
    a.kwscale = std::sqrt(P.nscale * kf);
    a.kvscale = std::sqrt(kf);
  }
  const int grid = resident_grid(h, h.f_resident, nctas);
  a.gfield = h.d_gfield.p;
  void* params[] = {&a};
  xs_launch(h, XS_KERNEL_RESIDENT, h.f_resident, grid, 1, 1, h.rp.threads, (unsigned)h.rp.smem, st, params,
            "launch xs_resident");
  if (stride > 0) {
    const void* part = h.d_obs.p;
    int ctas_per_block = P.E1 / G;
    int strd = (int)stride;
    double inv = 1.0 / P.E1;
    void* rparams[] = {&part, &av_dev, (void*)&npts, (void*)&nctas, &ctas_per_block, &strd, &inv};
    unsigned gx = (unsigned)((stride + 127) / 128);
    xs_launch(h, XS_KERNEL_OBS_REDUCE, h.f_reduce, gx, (unsigned)npts, (unsigned)nblocks, 128, 0, st, rparams,
              "launch xs_obs_reduce");
  }
}

// exp(2 L dtr/ipsteps): two consecutive half-step propagators merged into one.
const void* ensure_prop2(xs_handle& h, int nc) {
  const Problem& P = h.P;
  int slot = nc == 2 ? 1 : 0;
  ensure_prop(h, nc);
  double dt = 2.0 * pass_dtr(P, nc) / P.p.ipsteps;
  if (h.prop2_dtr[slot] == dt) return h.d_prop2[slot].p;
  std::vector<cd> pr = prop_values(h, dt);
  h.d_prop2[slot].ensure(std::max<size_t>(pr.size(), 1) * 16);
  CUDA_CHECK(cudaMemcpy(h.d_prop2[slot].p, pr.data(), pr.size() * 16, cudaMemcpyHostToDevice));
  h.prop2_dtr[slot] = dt;
  return h.d_prop2[slot].p;
}

struct StreamArgsHost {
  int ntraj, ens1, block0, seq;
  unsigned seed;
  int draw0, draw1, m, n, npoints;
  double wscale, vscale, dtr, t;
  void* field;
  const void* prop1;
  const void* prop2;
  const void* a_in;
  void* a_out;
  void* av;
  void* redpart;
  int* status;
  const double* params;
  const void* tw_x;
  const void* tw_y;
  void* opart;
  void* field2;
  int ndraw0, ndraw1;
  int fuse;
  const void* mat;
  int xspace;
};

// Observation pass: each block's trajectories split over kObsSplit CTAs (grid z) for latency
// hiding, then xs_x_obs_combine adds the splits into the block means.
constexpr int kObsSplit = 4;
void launch_observe(xs_handle& h, void** prm, int nrg, int nb, cudaStream_t st) {
  const StreamPlan& sp = h.sp;
  xs_launch(h, XS_KERNEL_X_OBS, h.f_xobs, (unsigned)nrg, (unsigned)nb, kObsSplit, (unsigned)(sp.OROWS * sp.RX),
            (unsigned)sp.osmem, st, prm, "observation pass");
  if (h.P.nout_site) {
    int nsplit = kObsSplit;
    void* cprm[] = {prm[0], &nsplit};
    const unsigned gx = (unsigned)(((size_t)h.P.nout_site * h.P.NS + 255) / 256);
    xs_launch(h, XS_KERNEL_X_OBS, h.f_xcomb, gx, (unsigned)nb, 1, 256, 0, st, cprm, "observation combine");
  }
}

// The pass sequence of one streaming p.path call (Simulator/xpath.m:29-86 with merged MP
// half steps): initial field, then per step a column pass (exp(L dt)^m, m = 2 when the previous
// step's second half is merged in) and a row pass (drift and noise), and at output times the
// pending half step and the observables.
struct StreamOp {
  enum Kind { INIT, COL, ROW, OBS, FINAL } kind;
  int m, draw0, draw1, n;
  double t;
};

std::vector<StreamOp> stream_ops(const Problem& P, int nc, bool final_field) {
  std::vector<StreamOp> ops;
  double t = P.p.origins[0];
  const double dtr = pass_dtr(P, nc);
  ops.push_back({StreamOp::INIT, 0, 0, -1, 0, t});
  int pending = 0, draw = 0, prev_draw = -1;
  const int npts = P.p.points[0], S = P.p.steps, checks = P.p.checks;
  for (int n = 0; n < npts; ++n)
    for (int step = 0; step < S; ++step) {
      if (n > 0 || step > 0 || npts == 1)
        for (int chk = 0; chk <= checks; ++chk) {
          ++draw;
          if (nc == 2 && checks && chk == 0) {
            prev_draw = draw;
            continue;
          }
          ops.push_back({StreamOp::COL, pending + 1, 0, -1, 0, t});
          ops.push_back({StreamOp::ROW, 0, draw, (nc == 2 && checks) ? prev_draw : -1, 0, t});
          t += dtr;
          pending = 1;
        }
      if (step == 0) {
        if (pending) ops.push_back({StreamOp::COL, pending, 0, -1, 0, t});
        pending = 0;
        ops.push_back({StreamOp::OBS, 0, 0, -1, n, t});
      }
    }
  if (final_field) {
    if (pending) ops.push_back({StreamOp::COL, pending, 0, -1, 0, t});
    ops.push_back({StreamOp::FINAL, 0, 0, -1, 0, t});
  }
  return ops;
}

// The two halves of the blocks (independent trajectories) run the same pass sequence one pass
// apart, so that wherever one half's row pass meets the other half's column pass the two go into
// one xs_rc_pass launch: the issue-bound row pass and the HBM-bound column pass share the SMs.
void launch_stream_halves(xs_handle& h, const StreamArgsHost& a, int nblocks, int nc, void* av_dev, cudaStream_t st) {
  const Problem& P = h.P;
  const StreamPlan& sp = h.sp;
  const size_t cxs = h.fp64 ? 16 : 8;
  const int nb = nblocks / 2, th = nb * P.E1;
  const int nrg = P.N[1] / sp.OROWS;
  const size_t stride = av_stride(P);
  StreamArgsHost half[2] = {a, a};
  for (int hf = 0; hf < 2; ++hf) {
    StreamArgsHost& b = half[hf];
    const size_t e0 = (size_t)hf * th;
    b.ntraj = th;
    b.block0 = a.block0 + hf * nb;
    b.field = (char*)a.field + e0 * P.F * P.NS * cxs;
    if (a.a_in) b.a_in = (const char*)a.a_in + e0 * P.F * P.NS * 16;
    if (a.a_out) b.a_out = (char*)a.a_out + e0 * P.F * P.NS * 16;
    b.av = (char*)av_dev + (size_t)hf * nb * P.p.points[0] * stride * 16;
    if (a.redpart) b.redpart = (char*)a.redpart + e0 * nrg * std::max(P.nred, 1) * 16;
  }
  const unsigned xgrid = (unsigned)((size_t)th * P.N[1] / sp.XROWS);
  const unsigned sgrid = (unsigned)((size_t)th * P.F * (P.N[0] / sp.TX));
  auto set = [](StreamArgsHost& b, const StreamOp& o) {
    b.m = o.m;
    b.draw0 = o.draw0;
    b.draw1 = o.draw1;
    b.n = o.n;
    b.t = o.t;
  };
  auto run = [&](const StreamOp& o, StreamArgsHost& b) {
    set(b, o);
    void* prm[] = {&b};
    switch (o.kind) {
      case StreamOp::INIT:
        xs_launch(h, XS_KERNEL_X_INIT, h.f_xinit, xgrid, 1, 1, 256, (unsigned)sp.xsmem, st, prm, "row pass");
        break;
      case StreamOp::ROW:
        xs_launch(h, XS_KERNEL_X_STEP, h.f_xnl, xgrid, 1, 1, 256, (unsigned)sp.xsmem, st, prm, "row pass");
        break;
      case StreamOp::FINAL:
        xs_launch(h, XS_KERNEL_X_FINAL, h.f_xfinal, xgrid, 1, 1, 256, (unsigned)sp.xsmem, st, prm, "row pass");
        break;
      case StreamOp::COL:
        xs_launch(h, XS_KERNEL_Y_PASS, h.f_spass, sgrid, 1, 1, 256, (unsigned)sp.ssmem, st, prm, "column pass");
        break;
      case StreamOp::OBS:
        launch_observe(h, prm, nrg, nb, st);
        if (P.nout_scalar)
          xs_launch(h, XS_KERNEL_SCALAR, h.f_scalar, (unsigned)nb, 1, 1, 256, 0, st, prm, "scalar observables");
        break;
    }
  };
  const std::vector<StreamOp> ops = stream_ops(P, nc, a.a_out != nullptr);
  const size_t L = ops.size();
  for (size_t i = 0; i <= L; ++i) {
    const StreamOp* o0 = i < L ? &ops[i] : nullptr;      // first half: op i
    const StreamOp* o1 = i >= 1 ? &ops[i - 1] : nullptr;  // second half: op i - 1
    if (o0 && o1 && ((o0->kind == StreamOp::ROW && o1->kind == StreamOp::COL) ||
                     (o0->kind == StreamOp::COL && o1->kind == StreamOp::ROW))) {
      const int hr = o0->kind == StreamOp::ROW ? 0 : 1;
      StreamArgsHost& R = half[hr];
      StreamArgsHost& C = half[1 - hr];
      set(R, hr == 0 ? *o0 : *o1);
      set(C, hr == 0 ? *o1 : *o0);
      void* prm[] = {&R, &C};
      xs_launch(h, XS_KERNEL_RC_PASS, h.f_rc, xgrid + sgrid, 1, 1, 256, (unsigned)std::max(sp.xsmem, sp.ssmem), st,
                prm, "fused row/column pass");
      continue;
    }
    if (o0) run(*o0, half[0]);
    if (o1) run(*o1, half[1]);
  }
}

// Streaming schedule of one xpath call on a 3D DST/DCT lattice (xs_stream3.cuh): the pass
// sequence of the 2D path (stream_ops), z-line passes in place of the column passes and plane
// passes in place of the row passes, on persistent grids.
void launch_stream3(xs_handle& h, int first_block, int nblocks, int nc, const void* a_in_dev, void* av_dev,
                    void* a_out_dev, cudaStream_t st) {
  const Problem& P = h.P;
  const StreamPlan& sp = h.sp;
  const int total = nblocks * P.E1;
  const size_t cxs = h.fp64 ? 16 : 8;
  h.d_field.ensure((size_t)total * P.NS * cxs);
  const int nz = P.N[2];
  if (P.nred) h.d_redpart.ensure((size_t)total * nz * P.nred * 16);
  StreamArgsHost a{};
  a.ntraj = total;
  a.ens1 = P.E1;
  a.block0 = first_block;
  a.seq = P.p.sequence;
  a.seed = (unsigned)(P.p.seed & 0xffffffffu);
  a.draw1 = -1;
  a.npoints = P.p.points[0];
  a.wscale = std::sqrt(P.nscale * P.noisefactor);
  a.vscale = std::sqrt(P.noisefactor);
  a.dtr = pass_dtr(P, nc);
  a.field = h.d_field.p;
  a.prop1 = ensure_prop(h, nc);
  a.prop2 = ensure_prop2(h, nc);
  a.a_in = a_in_dev;
  a.a_out = a_out_dev;
  a.av = av_dev;
  a.redpart = h.d_redpart.p;
  a.status = (int*)h.d_status.p;
  a.params = (const double*)h.d_params.p;
  a.mat = h.d_mat3.p;
  if (P.nout_site) {
    h.d_opart.ensure((size_t)kObsSplit * nblocks * P.nout_site * P.NS * 16);
    a.opart = h.d_opart.p;
  }
  void* params[] = {&a};
  const size_t nplanes = (size_t)total * nz, ntiles = (size_t)total * (P.N[0] * P.N[1] / sp.QT);
  const unsigned gp = (unsigned)std::min<size_t>(nplanes, (size_t)h.grid_p);
  const unsigned gz = (unsigned)std::min<size_t>(ntiles, (size_t)h.grid_z);
  // the initial field stays in x space until its first observation has been taken (the
  // transforms drop Dirichlet boundary values, which that observation still sees)
  bool xspace = false;
  for (const StreamOp& o : stream_ops(P, nc, a_out_dev != nullptr)) {
    a.m = o.m;
    a.draw0 = o.draw0;
    a.draw1 = o.draw1;
    a.n = o.n;
    a.t = o.t;
    if (xspace && (o.kind == StreamOp::ROW || o.kind == StreamOp::COL)) {
      a.xspace = 0;
      xs_launch(h, XS_KERNEL_X_INIT, h.f_ptok, gp, 1, 1, 256, (unsigned)sp.psmem3[0], st, params, "plane pass");
      xspace = false;
    }
    a.xspace = xspace ? 1 : 0;
    switch (o.kind) {
      case StreamOp::INIT: {
        const unsigned gi = (unsigned)std::min<size_t>(((size_t)total * P.NS + 255) / 256, (size_t)h.grid_p * 8);
        xs_launch(h, XS_KERNEL_X_INIT, h.f_pinit, gi, 1, 1, 256, 0, st, params, "initial field");
        xspace = true;
        break;
      }
      case StreamOp::ROW:
        if (h.tc3) {
          const void* mt = h.d_mat3tc.p;
          void* tparams[] = {&a, &mt};
          const unsigned gt = (unsigned)std::min<size_t>(nplanes, (size_t)h.grid_tc);
          xs_launch(h, XS_KERNEL_X_STEP, h.f_pnl_tc, gt, 1, 1, kTc3Threads, (unsigned)kTc3Smem, st, tparams,
                    "plane pass (tensor cores)");
        } else {
          xs_launch(h, XS_KERNEL_X_STEP, h.f_pnl, gp, 1, 1, 256, (unsigned)sp.psmem3[1], st, params, "plane pass");
        }
        break;
      case StreamOp::FINAL:
        xs_launch(h, XS_KERNEL_X_FINAL, h.f_pfinal, gp, 1, 1, 256, (unsigned)sp.psmem3[2], st, params, "plane pass");
        break;
      case StreamOp::COL:
        xs_launch(h, XS_KERNEL_Y_PASS, h.f_zpass, gz, 1, 1, 256, (unsigned)sp.zsmem3, st, params, "z-line pass");
        break;
      case StreamOp::OBS:
        xs_launch(h, XS_KERNEL_X_OBS, h.f_pobs, (unsigned)nz, (unsigned)nblocks, kObsSplit, 256, (unsigned)sp.osmem3, st,
                  params, "observation pass");
        if (P.nout_site) {
          int nsplit = kObsSplit;
          void* cprm[] = {params[0], &nsplit};
          const unsigned gx = (unsigned)(((size_t)P.nout_site * P.NS + 255) / 256);
          xs_launch(h, XS_KERNEL_X_OBS, h.f_xcomb, gx, (unsigned)nblocks, 1, 256, 0, st, cprm, "observation combine");
        }
        if (P.nout_scalar)
          xs_launch(h, XS_KERNEL_SCALAR, h.f_scalar, (unsigned)nblocks, 1, 1, 256, 0, st, params, "scalar observables");
        break;
    }
  }
}

// Streaming schedule of one xpath call (Simulator/xpath.m:29-86) for MP:
// column passes apply the pending half-step propagators, row passes do the
// midpoint step; observations need all half steps applied first.
void launch_stream(xs_handle& h, int first_block, int nblocks, int nc, const void* a_in_dev, void* av_dev,
                   void* a_out_dev, cudaStream_t st) {
  if (h.kind == 3) {
    launch_stream3(h, first_block, nblocks, nc, a_in_dev, av_dev, a_out_dev, st);
    return;
  }
  const Problem& P = h.P;
  const StreamPlan& sp = h.sp;
  const int total = nblocks * P.E1;
  const size_t cxs = h.fp64 ? 16 : 8;
  h.d_field.ensure((size_t)total * P.F * P.NS * cxs);
  const int nrg = P.N[1] / sp.OROWS;
  if (P.nred) h.d_redpart.ensure((size_t)total * nrg * P.nred * 16);
  StreamArgsHost a{};
  a.ntraj = total;
  a.ens1 = P.E1;
  a.block0 = first_block;
  a.seq = P.p.sequence;
  a.seed = (unsigned)(P.p.seed & 0xffffffffu);
  a.draw0 = 0;
  a.draw1 = -1;
  a.npoints = P.p.points[0];
  a.wscale = std::sqrt(P.nscale * P.noisefactor);
  a.vscale = std::sqrt(P.noisefactor);
  a.dtr = pass_dtr(P, nc);
  a.t = P.p.origins[0];
  a.field = h.d_field.p;
  a.prop1 = ensure_prop(h, nc);
  a.prop2 = ensure_prop2(h, nc);
  a.a_in = a_in_dev;
  a.a_out = a_out_dev;
  a.av = av_dev;
  a.redpart = h.d_redpart.p;
  a.status = (int*)h.d_status.p;
  a.params = (const double*)h.d_params.p;
  a.tw_x = h.d_twiddle.p;
  a.tw_y = (const char*)h.d_twiddle.p + (size_t)sp.RX * sp.RX * cxs;
  if (P.nout_site) {
    h.d_opart.ensure((size_t)kObsSplit * nblocks * P.nout_site * P.NS * 16);
    a.opart = h.d_opart.p;
  }
  void* params[] = {&a};
  const unsigned xgrid = (unsigned)((size_t)total * P.N[1] / sp.XROWS);
  const unsigned sgrid = (unsigned)((size_t)total * P.F * (P.N[0] / sp.TX));
  auto row = [&](int kind, CUfunction f) {
    xs_launch(h, kind, f, xgrid, 1, 1, 256, (unsigned)sp.xsmem, st, params, "row pass");
  };
  if (h.tma && (h.tmap_ptr != h.d_field.p || h.tmap_rows != (long long)total * P.F * P.N[1])) {
    // the field as a 2D tensor of reals: [rows = trajectories x components x NY][2 NX]
    const cuuint64_t dims[2] = {(cuuint64_t)2 * P.N[0], (cuuint64_t)total * P.F * P.N[1]};
    const cuuint64_t strides[1] = {(cuuint64_t)2 * P.N[0] * (cxs / 2)};
    const cuuint32_t box[2] = {(cuuint32_t)(2 * sp.TX), (cuuint32_t)P.N[1]};
    const cuuint32_t estr[2] = {1, 1};
    cu_check(driver().tmap_encode(&h.tmap, h.fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                                  h.d_field.p, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE),
             "cuTensorMapEncodeTiled");
    h.tmap_ptr = h.d_field.p;
    h.tmap_rows = (long long)total * P.F * P.N[1];
  }
  auto col = [&](int m) {
    a.m = m;
    if (h.tma) {
      void* tparams[] = {&a, &h.tmap};
      const unsigned g = (unsigned)std::min<long long>(sgrid, h.tma_grid);
      xs_launch(h, XS_KERNEL_Y_PASS, h.f_spass_tma, g, 1, 1, 256, (unsigned)sp.tsmem, st, tparams,
                "column pass (TMA)");
    } else {
      xs_launch(h, XS_KERNEL_Y_PASS, h.f_spass, sgrid, 1, 1, 256, (unsigned)sp.ssmem, st, params, "column pass");
    }
  };
  auto observe = [&](int n) {
    a.n = n;
    launch_observe(h, params, nrg, nblocks, st);
    if (P.nout_scalar)
      xs_launch(h, XS_KERNEL_SCALAR, h.f_scalar, (unsigned)nblocks, 1, 1, 256, 0, st, params, "scalar observables");
  };
  if (P.p.method == XS_METHOD_RK4) {
    // RK4 (Applications/SDE/RK4.m:7-42): row passes 1, 2, 3 on the two fields with column
    // passes P on both in between; pass 3 also does the next step's pass 1 unless the field
    // is observed in between
    h.d_field2.ensure((size_t)total * P.F * P.NS * cxs);
    a.field2 = h.d_field2.p;
    struct RkOp {
      bool obs;
      int n, d0, d1;
    };
    std::vector<RkOp> ops;
    {
      int draw = 0, prev = -1;
      const int npts = P.p.points[0], S = P.p.steps, checks = P.p.checks;
      for (int n = 0; n < npts; ++n)
        for (int step = 0; step < S; ++step) {
          if (n > 0 || step > 0 || npts == 1)
            for (int chk = 0; chk <= checks; ++chk) {
              ++draw;
              if (nc == 2 && checks && chk == 0) {
                prev = draw;
                continue;
              }
              ops.push_back({false, 0, draw, (nc == 2 && checks) ? prev : -1});
            }
          if (step == 0) ops.push_back({true, n, 0, -1});
        }
    }
    auto rk = [&](int i) {
      xs_launch(h, XS_KERNEL_X_STEP, h.f_xrk[i], xgrid, 1, 1, 256, (unsigned)sp.rksmem, st, params, "RK4 row pass");
    };
    auto col_both = [&]() {
      a.m = 1;
      xs_launch(h, XS_KERNEL_Y_PASS, h.f_spass, sgrid, 1, 1, 256, (unsigned)sp.ssmem, st, params, "column pass");
      StreamArgsHost b = a;
      b.field = a.field2;
      void* bp[] = {&b};
      xs_launch(h, XS_KERNEL_Y_PASS, h.f_spass, sgrid, 1, 1, 256, (unsigned)sp.ssmem, st, bp, "column pass");
    };
    row(XS_KERNEL_X_INIT, h.f_xinit);
    bool pass1_done = false;
    for (size_t i = 0; i < ops.size(); ++i) {
      if (ops[i].obs) {
        observe(ops[i].n);
        continue;
      }
      a.draw0 = ops[i].d0;
      a.draw1 = ops[i].d1;
      a.fuse = 0;
      if (!pass1_done) rk(0);
      col_both();
      rk(1);
      col_both();
      const bool next = i + 1 < ops.size() && !ops[i + 1].obs;
      a.fuse = next ? 1 : 0;
      if (next) {
        a.ndraw0 = ops[i + 1].d0;
        a.ndraw1 = ops[i + 1].d1;
      }
      rk(2);
      pass1_done = next;
      a.t += a.dtr;
    }
    if (a_out_dev) row(XS_KERNEL_X_FINAL, h.f_xfinal);
    return;
  }
  if (h.fuse && h.f_rc && !h.tma && nblocks >= 2 && nblocks % 2 == 0) {
    launch_stream_halves(h, a, nblocks, nc, av_dev, st);
    return;
  }
  row(XS_KERNEL_X_INIT, h.f_xinit);
  int pending = 0, draw = 0, prev_draw = -1;
  const int npts = P.p.points[0], S = P.p.steps, checks = P.p.checks;
  for (int n = 0; n < npts; ++n) {
    for (int step = 0; step < S; ++step) {
      if (n > 0 || step > 0 || npts == 1) {
        for (int chk = 0; chk <= checks; ++chk) {
          ++draw;
          if (nc == 2 && checks && chk == 0) {
            prev_draw = draw;
            continue;
          }
          col(pending + 1);
          a.draw0 = draw;
          a.draw1 = (nc == 2 && checks) ? prev_draw : -1;
          row(XS_KERNEL_X_STEP, h.f_xnl);
          a.t += a.dtr;
          pending = 1;
        }
      }
      if (step == 0) {
        if (pending) col(pending);
        pending = 0;
        observe(n);
      }
    }
  }
  if (a_out_dev) {
    if (pending) col(pending);
    row(XS_KERNEL_X_FINAL, h.f_xfinal);
  }
}

// device [b][n][k] -> host MATLAB av{o} [lines, time, space] per block per observable
void scatter_av(const Problem& P, const std::vector<double>& dev, int nblocks, double* out) {
  const size_t stride = av_stride(P);
  const int npts = P.p.points[0];
  size_t o_off = 0;
  size_t per_block = av_doubles_per_block(P);
  for (int b = 0; b < nblocks; ++b) {
    double* ob = out + (size_t)b * per_block;
    o_off = 0;
    for (auto& o : P.obs) {
      if (o.partial) {  // sum the block means over the reduced dimensions (Int.m:48-70, Ave.m)
        const size_t ns = obs_sites(P, o);
        std::vector<int> j0(3, 0), keep(3, 1);
        for (int d = 0; d < P.D; ++d)
          if (o.pw[d] > 0) {
            keep[d] = 0;
            if (o.plo[d] < o.phi[d])  // first point 1 + floor((lo - x(1)) / dx), 1-based, as Int.m
              j0[d] = std::max(0, (int)std::floor((o.plo[d] - P.p.origins[d + 1]) / P.dx[d + 1]));
          }
        std::vector<double> acc((size_t)2 * o.lines * ns);
        for (int n = 0; n < npts; ++n) {
          std::fill(acc.begin(), acc.end(), 0.0);
          for (size_t s = 0; s < P.NS; ++s) {
            const int i[3] = {(int)(s % P.N[0]), P.D > 1 ? (int)((s / P.N[0]) % P.N[1]) : 0,
                              P.D > 2 ? (int)(s / ((size_t)P.N[0] * P.N[1])) : 0};
            double w = 1;
            size_t r = 0, rs = 1;
            bool in = true;
            for (int d = 0; d < P.D; ++d) {
              if (keep[d]) {
                r += (size_t)i[d] * rs;
                rs *= (size_t)P.N[d];
                continue;
              }
              w *= o.pw[d];
              if (o.plo[d] < o.phi[d])
                in = in && i[d] >= j0[d] && P.p.origins[d + 1] + i[d] * P.dx[d + 1] <= o.phi[d];
            }
            if (!in) continue;
            for (int l = 0; l < o.lines; ++l) {
              const size_t k = (size_t)(o.out_off + l) * P.NS + s;
              const size_t src = (((size_t)b * npts + n) * stride + k) * 2;
              acc[2 * ((size_t)l + (size_t)o.lines * r)] += w * dev[src];
              acc[2 * ((size_t)l + (size_t)o.lines * r) + 1] += w * dev[src + 1];
            }
          }
          for (size_t r = 0; r < ns; ++r)
            for (int l = 0; l < o.lines; ++l) {
              const size_t dst = o_off + ((size_t)l + (size_t)o.lines * ((size_t)n + (size_t)npts * r)) * 2;
              ob[dst] = acc[2 * ((size_t)l + (size_t)o.lines * r)];
              ob[dst + 1] = acc[2 * ((size_t)l + (size_t)o.lines * r) + 1];
            }
        }
        o_off += (size_t)2 * o.lines * npts * ns;
        continue;
      }
      size_t ns = o.spatial ? P.NS : 1;
      for (int n = 0; n < npts; ++n)
        for (size_t s = 0; s < ns; ++s)
          for (int l = 0; l < o.lines; ++l) {
            size_t k = o.spatial ? (size_t)(o.out_off + l) * P.NS + s : (size_t)P.nout_site * P.NS + o.out_off + l;
            size_t src = (((size_t)b * npts + n) * stride + k) * 2;
            size_t dst = o_off + ((size_t)l + (size_t)o.lines * ((size_t)n + (size_t)npts * s)) * 2;
            ob[dst] = dev[src];
            ob[dst + 1] = dev[src + 1];
          }
      o_off += (size_t)2 * o.lines * npts * ns;
    }
  }
}

template <class F>
xs_status guard(F&& f) {
  try {
    return f();
  } catch (const XsError& e) {
    g_err = e.msg;
    return e.code;
  } catch (const xs::GrammarError& e) {
    g_err = std::string("grammar: ") + e.what();
    return XS_ERR_GRAMMAR;
  } catch (const std::bad_alloc&) {
    g_err = "host out of memory";
    return XS_ERR_ARG;
  } catch (const std::exception& e) {
    g_err = e.what();
    return XS_ERR_ARG;
  }
}

void create_impl(const xs_problem* prob, xs_handle* h) {
  setup_problem(prob, h->P);
  h->fp64 = prob->precision != XS_PREC_FP32;
  if (prob->path_kind < 0 || prob->path_kind > 2) raise(XS_ERR_ARG, "path_kind must be 0, 1 or 2");
  h->path_kind = prob->path_kind;
  build_source(*h);
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
XS_API const char* xs_version(void) { return "xspde_b200 0.1 (sm_100a, NVRTC)"; }

XS_API size_t xs_last_error(char* buf, size_t n) {
  if (buf && n) {
    size_t m = std::min(n - 1, g_err.size());
    memcpy(buf, g_err.data(), m);
    buf[m] = 0;
  }
  return g_err.size();
}

XS_API xs_status xs_create(const xs_problem* prob, xs_handle** out) {
  if (!out) return XS_ERR_ARG;
  *out = nullptr;
  return guard([&]() -> xs_status {
    auto h = std::make_unique<xs_handle>();
    create_impl(prob, h.get());
    *out = h.release();
    return XS_OK;
  });
}

XS_API void xs_destroy(xs_handle* h) { delete h; }

XS_API xs_status xs_compile_check(const xs_problem* prob, char* log, size_t n) {
  return guard([&]() -> xs_status {
    xs_handle h;
    create_impl(prob, &h);
    std::string lg;
    nvrtc_compile(h.source, h.kind == 3 ? "xs_stream3" : h.kind == 2 ? "xs_stream" : "xs_resident", &lg);
    if (log && n) {
      size_t m = std::min(n - 1, lg.size());
      memcpy(log, lg.data(), m);
      log[m] = 0;
    }
    return XS_OK;
  });
}

XS_API xs_status xs_observe_info(const xs_handle* h, int o, int* lines, int* spatial) {
  if (!h || o < 0 || o >= (int)h->P.obs.size()) {
    g_err = "bad handle or observable index";
    return XS_ERR_ARG;
  }
  if (lines) *lines = h->P.obs[o].lines;
  if (spatial) *spatial = h->P.obs[o].spatial ? 1 : 0;
  return XS_OK;
}

XS_API xs_status xs_observe_shape(const xs_handle* h, int o, int* dims) {
  if (!h || o < 0 || o >= (int)h->P.obs.size() || !dims) {
    g_err = "bad handle, observable index or output pointer";
    return XS_ERR_ARG;
  }
  const Problem& P = h->P;
  const ObsInfo& ob = P.obs[o];
  for (int d = 0; d < 3; ++d)
    dims[d] = (d < P.D && ob.spatial && !(ob.partial && ob.pw[d] > 0)) ? P.N[d] : 1;
  return XS_OK;
}

XS_API size_t xs_av_doubles_per_block(const xs_handle* h) { return h ? av_doubles_per_block(h->P) : 0; }

XS_API int xs_path_kind(const xs_handle* h) { return h ? h->kind : 0; }

namespace {
struct RawScope {  // the raw-trajectory pointer belongs to one xs_run_path_raw call
  xs_handle* h;
  ~RawScope() { h->raw_dev = nullptr; }
};

// xs_run_path on the streaming path with the host copies overlapped: the blocks
// run in groups (the trajectories of different blocks are independent); group g's
// initial field is copied in on a second stream while group g - 1 integrates, and
// group g's block means (and final field) are copied out while group g + 1
// integrates.  Each group is the same pass sequence as one call for its blocks, so
// the results equal those of a single call.
void run_stream_pipelined(xs_handle* h, int first_block, int nblocks, int nc, const double* a_in, double* av_out,
                          double* a_out) {
  const Problem& P = h->P;
  const int ng = std::min(nblocks, 4);
  if (!h->cstream) CUDA_CHECK(cudaStreamCreateWithFlags(&h->cstream, cudaStreamNonBlocking));
  while ((int)h->pipe_ev.size() < 2 * ng) {
    cudaEvent_t e;
    CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    h->pipe_ev.push_back(e);
  }
  const size_t ntraj = (size_t)nblocks * P.E1, per_traj = (size_t)P.F * P.NS * 16;
  const size_t stride = av_stride(P), per_block = av_doubles_per_block(P);
  const size_t avd = (size_t)nblocks * P.p.points[0] * stride * 2;
  h->d_ain.ensure(ntraj * per_traj);
  h->d_av.ensure(std::max<size_t>(avd, 1) * 8);
  h->d_avm.ensure(std::max<size_t>((size_t)nblocks * per_block, 1) * 8);
  if (a_out) h->d_aout.ensure(ntraj * per_traj);
  XsAvMap m{};
  m.nobs = (int)P.obs.size();
  m.npts = P.p.points[0];
  m.NS = P.NS;
  m.nout_site = P.nout_site;
  m.stride = (int)stride;
  m.per_block = (long long)(per_block / 2);
  long long off = 0;
  for (int o = 0; o < m.nobs; ++o) {
    m.lines[o] = P.obs[o].lines;
    m.spatial[o] = P.obs[o].spatial ? 1 : 0;
    m.out_off[o] = P.obs[o].out_off;
    m.o_off[o] = off;
    off += (long long)P.obs[o].lines * m.npts * (P.obs[o].spatial ? P.NS : 1);
  }
  CUDA_CHECK(cudaMemsetAsync(h->d_status.p, 0, sizeof(int), h->stream));
  auto grp = [&](int g, int& b0, int& nb) {
    b0 = (int)((long long)nblocks * g / ng);
    nb = (int)((long long)nblocks * (g + 1) / ng) - b0;
  };
  for (int g = 0; g < ng; ++g) {  // every copy in, in order, on the copy stream
    int b0, nb;
    grp(g, b0, nb);
    const size_t t0 = (size_t)b0 * P.E1;
    CUDA_CHECK(cudaMemcpyAsync((char*)h->d_ain.p + t0 * per_traj, a_in + t0 * per_traj / 8, (size_t)nb * P.E1 * per_traj,
                               cudaMemcpyHostToDevice, h->cstream));
    CUDA_CHECK(cudaEventRecord(h->pipe_ev[2 * g], h->cstream));
  }
  for (int g = 0; g < ng; ++g) {
    int b0, nb;
    grp(g, b0, nb);
    const size_t t0 = (size_t)b0 * P.E1;
    CUDA_CHECK(cudaStreamWaitEvent(h->stream, h->pipe_ev[2 * g], 0));
    double* avg = (double*)h->d_av.p + (size_t)b0 * P.p.points[0] * stride * 2;
    void* dout = a_out ? (char*)h->d_aout.p + t0 * per_traj : nullptr;
    launch_stream(*h, first_block + b0, nb, nc, (const char*)h->d_ain.p + t0 * per_traj, avg, dout, h->stream);
    double* avm = (double*)h->d_avm.p + (size_t)b0 * per_block;
    if (av_out && per_block) CUDA_CHECK((cudaError_t)xs_aot_av_matlab_launch(avg, avm, &m, nb, h->stream));
    CUDA_CHECK(cudaEventRecord(h->pipe_ev[2 * g + 1], h->stream));
    CUDA_CHECK(cudaStreamWaitEvent(h->cstream, h->pipe_ev[2 * g + 1], 0));
    if (av_out && per_block)
      CUDA_CHECK(cudaMemcpyAsync(av_out + (size_t)b0 * per_block, avm, (size_t)nb * per_block * 8,
                                 cudaMemcpyDeviceToHost, h->cstream));
    if (a_out)
      CUDA_CHECK(cudaMemcpyAsync(a_out + t0 * per_traj / 8, dout, (size_t)nb * P.E1 * per_traj, cudaMemcpyDeviceToHost,
                                 h->cstream));
  }
  int status = 0;
  CUDA_CHECK(cudaMemcpyAsync(&status, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CUDA_CHECK(cudaStreamSynchronize(h->stream));
  CUDA_CHECK(cudaStreamSynchronize(h->cstream));
  if (status & 2) raise(XS_ERR_SHAPE, "kernel refused a launch whose shared-memory layout or grid did not match");
  if (status & 1) raise(XS_ERR_NAN, "a trajectory became non-finite (NaN/Inf) during the path");
}

xs_status run_path_impl(xs_handle* h, int first_block, int nblocks, int nc, const double* a_in, double* av_out,
                        double* a_out, double* raw_out) {
  NvtxRange range("xs_run_path nc=%d blocks %d+%d", nc, first_block, nblocks);
  return guard([&]() -> xs_status {
    if (!h || nblocks < 1 || first_block < 0 || (nc != 1 && nc != 2)) raise(XS_ERR_ARG, "bad arguments to xs_run_path");
    if (nc == 2 && !h->P.p.checks) raise(XS_ERR_ARG, "coarse pass requested without checks");
    load_module(*h);
    const Problem& P = h->P;
    if (h->kind >= 2 && a_in && !raw_out && nblocks >= 2 && P.F == 1 && P.obs.size() <= 32 && !any_partial(P)) {
      run_stream_pipelined(h, first_block, nblocks, nc, a_in, av_out, a_out);
      return XS_OK;
    }
    RawScope raw_scope{h};
    size_t rbytes = 0;
    if (raw_out) {
      if (h->kind != 1) raise(XS_ERR_UNSUPPORTED, "raw trajectories are recorded by the resident path only");
      rbytes = (size_t)nblocks * P.E1 * P.p.points[0] * P.F * P.NS * 16;
      size_t free_b = 0, total_b = 0;
      CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
      if (rbytes > free_b + h->d_raw.bytes)
        raise(XS_ERR_SHAPE, "raw trajectories (" + std::to_string(rbytes >> 20) +
                                " MiB) exceed free device memory: run fewer ensemble blocks per call");
      h->d_raw.ensure(rbytes);
      h->raw_dev = h->d_raw.p;
    }
    const size_t ntraj = (size_t)nblocks * P.E1;
    const size_t fbytes = ntraj * P.F * P.NS * 16;
    const void* din = nullptr;
    void* dout = nullptr;
    if (a_in) {
      // host [F, space, ens] -> device [e][f][s] (identical when F == 1)
      h->d_ain.ensure(fbytes);
      if (P.F == 1) {
        CUDA_CHECK(cudaMemcpyAsync(h->d_ain.p, a_in, fbytes, cudaMemcpyHostToDevice, h->stream));
      } else {  // reorder on the device
        h->d_tmp.ensure(fbytes);
        CUDA_CHECK(cudaMemcpyAsync(h->d_tmp.p, a_in, fbytes, cudaMemcpyHostToDevice, h->stream));
        CUDA_CHECK((cudaError_t)xs_aot_reorder_launch(h->d_tmp.p, h->d_ain.p, P.F, P.NS, (long long)ntraj, 1,
                                                      h->stream));
      }
      din = h->d_ain.p;
    }
    if (a_out) {
      h->d_aout.ensure(fbytes);
      dout = h->d_aout.p;
    }
    const size_t stride = av_stride(P);
    const size_t avd = (size_t)nblocks * P.p.points[0] * stride * 2;
    h->d_av.ensure(std::max<size_t>(avd, 1) * 8);
    CUDA_CHECK(cudaMemsetAsync(h->d_status.p, 0, sizeof(int), h->stream));
    if (h->kind >= 2) launch_stream(*h, first_block, nblocks, nc, din, h->d_av.p, dout, h->stream);
    else launch_resident(*h, first_block, nblocks, nc, din, h->d_av.p, dout, h->stream);
    // block means into MATLAB's layout on the device, then one copy into the caller's buffer
    const size_t per_block = av_doubles_per_block(P);
    // means into MATLAB's order on the device (a plain permutation), or on the host when an
    // observable sums over reduced dimensions
    const bool dev_perm = P.obs.size() <= 32 && !any_partial(P);
    std::vector<double> av(dev_perm ? 0 : avd);
    if (av_out && per_block) {
      if (dev_perm) {
        XsAvMap m{};
        m.nobs = (int)P.obs.size();
        m.npts = P.p.points[0];
        m.NS = P.NS;
        m.nout_site = P.nout_site;
        m.stride = (int)stride;
        m.per_block = (long long)(per_block / 2);
        long long off = 0;
        for (int o = 0; o < m.nobs; ++o) {
          m.lines[o] = P.obs[o].lines;
          m.spatial[o] = P.obs[o].spatial ? 1 : 0;
          m.out_off[o] = P.obs[o].out_off;
          m.o_off[o] = off;
          off += (long long)P.obs[o].lines * m.npts * (P.obs[o].spatial ? P.NS : 1);
        }
        h->d_avm.ensure((size_t)nblocks * per_block * 8);
        CUDA_CHECK((cudaError_t)xs_aot_av_matlab_launch(h->d_av.p, h->d_avm.p, &m, nblocks, h->stream));
        CUDA_CHECK(cudaMemcpyAsync(av_out, h->d_avm.p, (size_t)nblocks * per_block * 8, cudaMemcpyDeviceToHost,
                                   h->stream));
      } else if (avd) {
        CUDA_CHECK(cudaMemcpyAsync(av.data(), h->d_av.p, avd * 8, cudaMemcpyDeviceToHost, h->stream));
      }
    }
    int status = 0;
    CUDA_CHECK(cudaMemcpyAsync(&status, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    if (raw_out) CUDA_CHECK(cudaMemcpyAsync(raw_out, h->d_raw.p, rbytes, cudaMemcpyDeviceToHost, h->stream));
    if (a_out) {
      if (P.F == 1) {
        CUDA_CHECK(cudaMemcpyAsync(a_out, dout, fbytes, cudaMemcpyDeviceToHost, h->stream));
        CUDA_CHECK(cudaStreamSynchronize(h->stream));
      } else {  // reorder on the device
        h->d_tmp.ensure(fbytes);
        CUDA_CHECK((cudaError_t)xs_aot_reorder_launch(dout, h->d_tmp.p, P.F, P.NS, (long long)ntraj, 0, h->stream));
        CUDA_CHECK(cudaMemcpyAsync(a_out, h->d_tmp.p, fbytes, cudaMemcpyDeviceToHost, h->stream));
      }
    }
    CUDA_CHECK(cudaStreamSynchronize(h->stream));
    if (av_out && !dev_perm) scatter_av(P, av, nblocks, av_out);
    if (status & 2) raise(XS_ERR_SHAPE, "kernel refused a launch whose shared-memory layout or grid did not match");
    if (status & 1) raise(XS_ERR_NAN, "a trajectory became non-finite (NaN/Inf) during the path");
    return XS_OK;
  });
}
}  // namespace

XS_API xs_status xs_run_path(xs_handle* h, int first_block, int nblocks, int nc, const double* a_in, double* av_out,
                             double* a_out) {
  return run_path_impl(h, first_block, nblocks, nc, a_in, av_out, a_out, nullptr);
}

XS_API xs_status xs_run_path_raw(xs_handle* h, int first_block, int nblocks, int nc, const double* a_in,
                                 double* av_out, double* a_out, double* raw_out) {
  return run_path_impl(h, first_block, nblocks, nc, a_in, av_out, a_out, raw_out);
}

XS_API xs_status xs_run_path_device(xs_handle* h, int first_block, int nblocks, int nc, const double* a_in_dev,
                                    double* av_dev, double* a_out_dev, void* stream) {
  NvtxRange range("xs_run_path_device nc=%d blocks %d+%d", nc, first_block, nblocks);
  return guard([&]() -> xs_status {
    if (!h || nblocks < 1 || first_block < 0 || (nc != 1 && nc != 2) || !av_dev)
      raise(XS_ERR_ARG, "bad arguments to xs_run_path_device");
    load_module(*h);
    cudaStream_t st = (cudaStream_t)stream;  // the caller's stream; NULL is the default stream
    CUDA_CHECK(cudaMemsetAsync(h->d_status.p, 0, sizeof(int), st));
    if (h->kind >= 2) launch_stream(*h, first_block, nblocks, nc, a_in_dev, av_dev, a_out_dev, st);
    else launch_resident(*h, first_block, nblocks, nc, a_in_dev, av_dev, a_out_dev, st);
    return XS_OK;
  });
}

XS_API xs_status xs_sync(xs_handle* h) {
  return guard([&]() -> xs_status {
    if (!h || !h->loaded) raise(XS_ERR_ARG, "handle has not run");
    CUDA_CHECK(cudaDeviceSynchronize());
    int status = 0;
    CUDA_CHECK(cudaMemcpy(&status, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (status & 2) raise(XS_ERR_SHAPE, "kernel refused a launch whose shared-memory layout or grid did not match");
    if (status & 1) raise(XS_ERR_NAN, "a trajectory became non-finite (NaN/Inf) during the path");
    return XS_OK;
  });
}

XS_API xs_status xs_set_boundary_values(xs_handle* h, int nc, int ntimes, const double* values) {
  return guard([&]() -> xs_status {
    if (!h || (nc != 1 && nc != 2) || ntimes < 1 || !values) raise(XS_ERR_ARG, "bad arguments to xs_set_boundary_values");
    const Problem& P = h->P;
    if (!P.bvals) raise(XS_ERR_ARG, "the problem was created without boundary_values");
    load_module(*h);
    const int slot = nc == 2 ? 1 : 0;
    const size_t n = (size_t)ntimes * P.D * P.F * 2;
    h->d_bval[slot].ensure(n * 16);
    CUDA_CHECK(cudaMemcpy(h->d_bval[slot].p, values, n * 16, cudaMemcpyHostToDevice));
    // da of the Neumann patch (xpropfactor.m:45-50): -(L(k1) - L(k0)) dt / pi^2 R^2 along each dimension
    std::vector<cd> da((size_t)std::max(P.D, 1) * P.F, cd(0, 0));
    if (P.has_linear) {
      const double dt = pass_dtr(P, nc) / P.p.ipsteps;
      const double fda = dt / (M_PI * M_PI);
      int sd = 1;
      for (int d = 0; d < P.D; ++d) {
        for (int f = 0; f < P.F; ++f) {
          const int c = P.Lc > 1 ? f : 0;
          if (P.N[d] > 1) {
            const cd L1 = P.L[(size_t)c * P.NS], L2 = P.L[(size_t)c * P.NS + sd];
            da[(size_t)d * P.F + f] = -(L2 - L1) * fda * P.p.ranges[d + 1] * P.p.ranges[d + 1];
          }
        }
        sd *= P.N[d];
      }
    }
    h->d_bda[slot].ensure(da.size() * 16);
    CUDA_CHECK(cudaMemcpy(h->d_bda[slot].p, da.data(), da.size() * 16, cudaMemcpyHostToDevice));
    h->bval_n[slot] = ntimes;
    return XS_OK;
  });
}

// Resident path with its observable partial sums in the library's fixed
// device scratch (xs_noalloc.cu) instead of handle-owned memory.  Uses only
// tables the handle already holds; allocates nothing.  Its two launches go
// straight to the driver, without the handle's timing events (creating those
// would allocate), and are not counted by xs_kernel_stats.
XS_API xs_status xs_run_path_device_noalloc(xs_handle* h, int first_block, int nblocks, int nc, double* av_dev,
                                            void* stream) {
  return guard([&]() -> xs_status {
    if (!h || nblocks < 1 || first_block < 0 || (nc != 1 && nc != 2) || !av_dev)
      raise(XS_ERR_ARG, "bad arguments to xs_run_path_device_noalloc");
    const Problem& P = h->P;
    if (h->kind != 1)
      raise(XS_ERR_UNSUPPORTED, "xs_run_path_device_noalloc covers problems on the resident path only");
    if (h->rp.gfield)
      raise(XS_ERR_UNSUPPORTED, "xs_run_path_device_noalloc needs the field in shared memory (it would allocate slices)");
    if (h->P.bvals) raise(XS_ERR_UNSUPPORTED, "xs_run_path_device_noalloc does not take boundary values");
    if (h->P.spec) raise(XS_ERR_UNSUPPORTED, "xs_run_path_device_noalloc does not record time spectra");
    if (h->P.NK || h->P.NKV) raise(XS_ERR_UNSUPPORTED, "xs_run_path_device_noalloc does not take k-filtered noises");
    if (h->P.NA) raise(XS_ERR_UNSUPPORTED, "xs_run_path_device_noalloc does not take auxiliary fields");
    if (nc == 2 && !P.p.checks) raise(XS_ERR_ARG, "coarse pass requested without checks");
    const int slot = nc == 2 ? 1 : 0;
    if (!h->loaded || !h->d_prop[slot].p || (P.has_linear && h->prop_dtr[slot] != pass_dtr(P, nc)))
      raise(XS_ERR_ARG,
            "handle not prepared for this check pass: call xs_run_path or xs_run_path_device once with the same "
            "nc first (that call allocates the handle's tables)");
    const int total = nblocks * P.E1;
    const int G = h->rp.G;
    const int nctas = total / G;
    const size_t stride = av_stride(P);
    const int npts = P.p.points[0];
    const size_t need = (size_t)npts * nctas * stride;
    if (need > XS_NOALLOC_SCRATCH_DOUBLE2)
      raise(XS_ERR_SHAPE, "xs_run_path_device_noalloc needs " + std::to_string(need) +
                              " complex FP64 scratch values for this launch; the fixed scratch holds " +
                              std::to_string((size_t)XS_NOALLOC_SCRATCH_DOUBLE2) + " (16 MiB): use fewer blocks per call");
    void* scratch = nullptr;
    cudaError_t e = xs_noalloc_scratch_address(&scratch);
    if (e != cudaSuccess) raise(XS_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    cudaStream_t st = (cudaStream_t)stream;  // the caller's stream; NULL is the default stream
    CUDA_CHECK(cudaMemsetAsync(h->d_status.p, 0, sizeof(int), st));
    PathArgsHost a{};
    a.ntraj = total;
    a.ens1 = P.E1;
    a.block0 = first_block;
    a.nc = nc;
    a.checks = P.p.checks;
    a.npoints = npts;
    a.steps = P.p.steps;
    a.seq = P.p.sequence;
    a.seed = (unsigned)(P.p.seed & 0xffffffffu);
    a.wscale = std::sqrt(P.nscale * P.noisefactor);
    a.vscale = std::sqrt(P.noisefactor);
    a.dtr = pass_dtr(P, nc);
    a.t0 = P.p.origins[0];
    a.prop = h->d_prop[slot].p;
    a.prop2 = h->d_prop2[slot].p;
    a.tmat = h->d_tmat.p;
    for (int i = 0; i < 4; ++i) a.tmat_off[i] = h->tmat_off[i];
    a.a_in = nullptr;
    a.a_out = nullptr;
    a.obs = scratch;
    a.status = (int*)h->d_status.p;
    a.params = (const double*)h->d_params.p;
    void* params[] = {&a};
    cu_check(driver().launch(h->f_resident, nctas, 1, 1, h->rp.threads, 1, 1, (unsigned)h->rp.smem, (CUstream)st,
                             params, nullptr),
             "launch xs_resident (no-alloc)");
    if (stride > 0) {
      const void* part = scratch;
      void* av = av_dev;
      int ctas_per_block = P.E1 / G;
      int strd = (int)stride;
      double inv = 1.0 / P.E1;
      int np = npts, nct = nctas;
      void* rparams[] = {&part, &av, &np, &nct, &ctas_per_block, &strd, &inv};
      cu_check(driver().launch(h->f_reduce, (unsigned)((stride + 127) / 128), (unsigned)npts, (unsigned)nblocks, 128,
                               1, 1, 0, (CUstream)st, rparams, nullptr),
               "launch xs_obs_reduce (no-alloc)");
    }
    return XS_OK;
  });
}

XS_API xs_status xs_noise_features(xs_handle* h, int first_block, int nblocks, const int* region, int first_draw,
                                   int draws_per_window, int windows, double decay, float* out_dev, void* stream) {
  return guard([&]() -> xs_status {
    if (!h || nblocks < 1 || first_block < 0 || !region || !out_dev || draws_per_window < 1 || windows < 1 ||
        first_draw < 1)
      raise(XS_ERR_ARG, "bad arguments to xs_noise_features");
    const Problem& P = h->P;
    if (P.D > 2 || P.NW < 1) raise(XS_ERR_UNSUPPORTED, "noise features need at most two space dimensions and noises");
    const int i1lo = region[0], i2lo = region[1], bw = region[2], bh = region[3], nbx = region[4], nby = region[5];
    if (bw < 1 || bh < 1 || nbx < 1 || nby < 1 || nbx > 16 || nby > 16 || i1lo < 0 || i2lo < 0 ||
        i1lo + nbx * bw > P.N[0] || i2lo + nby * bh > P.N[1])
      raise(XS_ERR_ARG, "feature region outside the lattice or more than 16x16 blocks");
    load_module(*h);
    struct {
      int ntraj, ens1, block0, seq;
      unsigned seed;
      int i1lo, i2lo, bw, bh, nbx, nby;
      int d0, dw, nt;
      float decay;
      float* out;
      int* status;
    } a{};
    a.ntraj = nblocks * P.E1;
    a.ens1 = P.E1;
    a.block0 = first_block;
    a.seed = (unsigned)(P.p.seed & 0xffffffffu);
    a.i1lo = i1lo;
    a.i2lo = i2lo;
    a.bw = bw;
    a.bh = bh;
    a.nbx = nbx;
    a.nby = nby;
    a.d0 = first_draw;
    a.dw = draws_per_window;
    a.nt = windows;
    a.decay = (float)decay;
    a.out = out_dev;
    a.status = (int*)h->d_status.p;
    void* params[] = {&a};
    cudaStream_t st = (cudaStream_t)stream;  // the caller's stream; NULL is the default stream
    cu_check(driver().launch(h->f_feat, (unsigned)(a.ntraj * windows), 1, 1, 256, 1, 1, 0, (CUstream)st, params,
                             nullptr),
             "launch xs_noise_features");
    return XS_OK;
  });
}

// ---- learned control variate network (device pointers, caller's stream) ----
XS_API size_t xs_mlp_sizes(int in, int hidden, int batch, size_t* nparams) {
  if (in < 1 || hidden < 1 || batch < 1) return 0;
  return xs_mlp_layout(in, hidden, batch, nparams);
}

XS_API xs_status xs_mlp_forward(int batch, int in, int hidden, const float* x, const float* params, float* work,
                                float* y, void* stream) {
  if (batch < 1 || in < 1 || hidden < 1 || !x || !params || !work) {
    g_err = "bad arguments to xs_mlp_forward";
    return XS_ERR_ARG;
  }
  int e = xs_mlp_forward_impl(batch, in, hidden, x, params, work, y, (cudaStream_t)stream, false);
  if (e) {
    g_err = std::string("xs_mlp_forward: ") + cudaGetErrorString((cudaError_t)e);
    return XS_ERR_CUDA;
  }
  if (xs_mlp_status((cudaStream_t)stream)) {
    g_err = "xs_mlp_forward: a tensor-core layer gave up waiting for its operands";
    return XS_ERR_TIMEOUT;
  }
  return XS_OK;
}

XS_API xs_status xs_mlp_train_grad(int batch, int in, int hidden, const float* x, const float* params, float* work,
                                   const float* target, float* grad, double* loss_dev, void* stream) {
  if (batch < 1 || in < 1 || hidden < 1 || !x || !params || !work || !target || !grad || !loss_dev) {
    g_err = "bad arguments to xs_mlp_train_grad";
    return XS_ERR_ARG;
  }
  int e = xs_mlp_forward_impl(batch, in, hidden, x, params, work, nullptr, (cudaStream_t)stream, true);
  if (!e) e = xs_mlp_backward_impl(batch, in, hidden, x, params, work, target, grad, loss_dev, (cudaStream_t)stream);
  if (e) {
    g_err = std::string("xs_mlp_train_grad: ") + cudaGetErrorString((cudaError_t)e);
    return XS_ERR_CUDA;
  }
  if (xs_mlp_status((cudaStream_t)stream)) {
    g_err = "xs_mlp_train_grad: a tensor-core layer gave up waiting for its operands";
    return XS_ERR_TIMEOUT;
  }
  return XS_OK;
}

XS_API xs_status xs_mlp_adam(size_t n, float* params, const float* grad, float* m, float* v, float lr, float beta1,
                             float beta2, float eps, int step, float weight_decay, void* stream) {
  if (!n || !params || !grad || !m || !v || step < 1) {
    g_err = "bad arguments to xs_mlp_adam";
    return XS_ERR_ARG;
  }
  int e = xs_mlp_adam_impl(n, params, grad, m, v, lr, beta1, beta2, eps, step, weight_decay, (cudaStream_t)stream);
  if (e) {
    g_err = std::string("xs_mlp_adam: ") + cudaGetErrorString((cudaError_t)e);
    return XS_ERR_CUDA;
  }
  return XS_OK;
}

XS_API xs_status xs_set_kernel_timing(xs_handle* h, int on) {
  if (!h) {
    g_err = "null handle";
    return XS_ERR_ARG;
  }
  h->timing = on != 0;
  return XS_OK;
}

XS_API xs_status xs_kernel_stats(xs_handle* h, int reset, double* ms_out, long long* launches_out) {
  return guard([&]() -> xs_status {
    if (!h) raise(XS_ERR_ARG, "null handle");
    if (!h->pending.empty()) {
      CUDA_CHECK(cudaStreamSynchronize(h->stream));
      CUDA_CHECK(cudaDeviceSynchronize());
      for (auto& p : h->pending) {
        float ms = 0;
        CUDA_CHECK(cudaEventElapsedTime(&ms, p.a, p.b));
        h->kms[p.kind] += ms;
        h->event_pool.push_back(p.a);
        h->event_pool.push_back(p.b);
      }
      h->pending.clear();
    }
    for (int k = 0; k < XS_KERNEL_KINDS; ++k) {
      if (ms_out) ms_out[k] = h->kms[k];
      if (launches_out) launches_out[k] = h->launches[k];
      if (reset) {
        h->kms[k] = 0;
        h->launches[k] = 0;
      }
    }
    return XS_OK;
  });
}

XS_API xs_status xs_block_moments(const double* av_dev, int nblocks, long long n, double scale, double* mom_dev,
                                  int accumulate, void* stream) {
  return guard([&]() -> xs_status {
    if (!av_dev || !mom_dev || nblocks < 1 || n < 0) raise(XS_ERR_ARG, "bad arguments to xs_block_moments");
    if (n == 0) return XS_OK;
    CUDA_CHECK((cudaError_t)xs_aot_block_moments_launch(av_dev, n, nblocks, scale, mom_dev, accumulate ? 1 : 0,
                                                        (cudaStream_t)stream));
    return XS_OK;
  });
}

namespace {
xs_status export_normals(xs_handle* h, bool random, int block, int draw, double scale, double* out) {
  return guard([&]() -> xs_status {
    if (!h || block < 0 || draw < 0 || !out) raise(XS_ERR_ARG, "bad arguments");
    load_module(*h);
    const Problem& P = h->P;
    const int nc = random ? P.NV : P.NW;
    const size_t n = (size_t)nc * P.NS * P.E1;
    if (n == 0) return XS_OK;
    h->d_w.ensure(n * 8);
    unsigned blk = (unsigned)block, dr = (unsigned)draw, seq = (unsigned)P.p.sequence,
             seed = (unsigned)(P.p.seed & 0xffffffffu);
    int ens1 = P.E1;
    void* dp = h->d_w.p;
    void* params[] = {&dp, &ens1, &blk, &dr, &seq, &seed, &scale};
    unsigned grid = (unsigned)std::min<size_t>((n / nc + 255) / 256, 148 * 16);
    xs_launch(*h, XS_KERNEL_RESIDENT, random ? h->f_random : h->f_noise, grid, 1, 1, 256, 0, h->stream, params,
              "noise export");
    h->launches[XS_KERNEL_RESIDENT]--;  // not a path launch
    CUDA_CHECK(cudaMemcpyAsync(out, h->d_w.p, n * 8, cudaMemcpyDeviceToHost, h->stream));
    CUDA_CHECK(cudaStreamSynchronize(h->stream));
    return XS_OK;
  });
}
}  // namespace

XS_API xs_status xs_noise(xs_handle* h, int block, int draw, double scale, double* w_out) {
  if (!h) {
    g_err = "null handle";
    return XS_ERR_ARG;
  }
  return export_normals(h, false, block, draw, std::sqrt(scale * h->P.noisefactor), w_out);  // xnoise.m:32
}

XS_API xs_status xs_random(xs_handle* h, int block, double* v_out) {
  if (!h) {
    g_err = "null handle";
    return XS_ERR_ARG;
  }
  return export_normals(h, true, block, 0, std::sqrt(h->P.noisefactor), v_out);  // xrandom.m:22
}

XS_API xs_status xs_step(xs_handle* h, double* a_inout, const double* w, double t, double dtr) {
  return guard([&]() -> xs_status {
    if (!h || !a_inout || !(dtr > 0)) raise(XS_ERR_ARG, "bad arguments to xs_step");
    if (h->kind != 1) raise(XS_ERR_UNSUPPORTED, "xs_step covers problems on the resident path only");
    if (h->P.bvals) raise(XS_ERR_UNSUPPORTED, "xs_step does not take boundary values");
    if (h->P.NK || h->P.NKV) raise(XS_ERR_UNSUPPORTED, "xs_step does not take k-filtered noises");
    if (h->P.NA) raise(XS_ERR_UNSUPPORTED, "xs_step does not take auxiliary fields");
    load_module(*h);
    const Problem& P = h->P;
    const size_t ntraj = (size_t)P.E1;
    const size_t fbytes = ntraj * P.F * P.NS * 16;
    // exp(L dtr/ipsteps) for this step (xpropfactor.m:28-39)
    if (P.has_linear && h->pstep_dtr != dtr) {
      std::vector<cd> pr(P.L.size());
      for (size_t i = 0; i < P.L.size(); ++i) pr[i] = std::exp(P.L[i] * (dtr / P.p.ipsteps));
      h->d_pstep.ensure(pr.size() * 16);
      CUDA_CHECK(cudaMemcpy(h->d_pstep.p, pr.data(), pr.size() * 16, cudaMemcpyHostToDevice));
      h->pstep_dtr = dtr;
    } else if (!P.has_linear) {
      h->d_pstep.ensure(16);
    }
    std::vector<double> tmp(ntraj * P.F * P.NS * 2);
    for (size_t e = 0; e < ntraj; ++e)
      for (int f = 0; f < P.F; ++f)
        for (int s = 0; s < P.NS; ++s) {
          size_t src = (f + (size_t)P.F * (s + (size_t)P.NS * e)) * 2, dst = ((e * P.F + f) * P.NS + s) * 2;
          tmp[dst] = a_inout[src];
          tmp[dst + 1] = a_inout[src + 1];
        }
    h->d_ain.ensure(fbytes);
    h->d_aout.ensure(fbytes);
    CUDA_CHECK(cudaMemcpyAsync(h->d_ain.p, tmp.data(), fbytes, cudaMemcpyHostToDevice, h->stream));
    const size_t wn = (size_t)P.NW * P.NS * ntraj;
    if (w && wn) {
      h->d_w.ensure(wn * 8);
      CUDA_CHECK(cudaMemcpyAsync(h->d_w.p, w, wn * 8, cudaMemcpyHostToDevice, h->stream));
    }
    h->d_obs.ensure(16);
    CUDA_CHECK(cudaMemsetAsync(h->d_status.p, 0, sizeof(int), h->stream));
    PathArgsHost a{};
    a.ntraj = (int)ntraj;
    a.ens1 = P.E1;
    a.nc = 1;
    a.npoints = 0;
    a.steps = 1;
    a.seed = (unsigned)(P.p.seed & 0xffffffffu);
    a.dtr = dtr;
    a.t0 = t;
    a.prop = h->d_pstep.p;
    a.prop2 = h->d_pstep.p;  // one whole step: no merged half steps
    a.tmat = h->d_tmat.p;
    for (int i = 0; i < 4; ++i) a.tmat_off[i] = h->tmat_off[i];
    a.a_in = h->d_ain.p;
    a.a_out = h->d_aout.p;
    a.obs = h->d_obs.p;
    a.status = (int*)h->d_status.p;
    a.single_step = 1;
    a.w_in = (w && wn) ? (const double*)h->d_w.p : nullptr;
    a.params = (const double*)h->d_params.p;
    void* params[] = {&a};
    const int grid = resident_grid(*h, h->f_resident, (int)(ntraj / h->rp.G));
    a.gfield = h->d_gfield.p;
    xs_launch(*h, XS_KERNEL_RESIDENT, h->f_resident, (unsigned)grid, 1, 1, h->rp.threads,
              (unsigned)h->rp.smem, h->stream, params, "launch xs_resident (step)");
    int status = 0;
    CUDA_CHECK(cudaMemcpyAsync(tmp.data(), h->d_aout.p, fbytes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_CHECK(cudaMemcpyAsync(&status, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_CHECK(cudaStreamSynchronize(h->stream));
    for (size_t e = 0; e < ntraj; ++e)
      for (int f = 0; f < P.F; ++f)
        for (int s = 0; s < P.NS; ++s) {
          size_t dst = (f + (size_t)P.F * (s + (size_t)P.NS * e)) * 2, src = ((e * P.F + f) * P.NS + s) * 2;
          a_inout[dst] = tmp[src];
          a_inout[dst + 1] = tmp[src + 1];
        }
    if (status & 2) raise(XS_ERR_SHAPE, "kernel refused a launch whose shared-memory layout or grid did not match");
    if (status & 1) raise(XS_ERR_NAN, "a trajectory became non-finite (NaN/Inf) during the step");
    return XS_OK;
  });
}

// ---------------------------------------------------------------------------
// Uneven batch: many independent problems in one CUDA-graph launch
// ---------------------------------------------------------------------------
namespace {

struct BatchItemHost {  // mirrors XsBatchItem
  int ntraj, steps, npoints, seq;
  unsigned seed;
  int block0, nunits;
  short nc, checks;
  double wscale, vscale, dtr, t0;
  const void* prop;
  void* part;
  void* av;
  const double* params;
  int* done;
  const void* prop2;
};
static_assert(sizeof(BatchItemHost) == 112, "XsBatchItem layout");

struct BatchArgsHost {  // mirrors XsBatchArgs
  const void* items;
  const void* units;
  int nunits, pad;
  int* next;
  int* status;
  const void* tmat;
  int tmat_off[4];
  void* gfield;
};
static_assert(sizeof(BatchArgsHost) == 72, "XsBatchArgs layout");

struct BatchVariant {
  std::string key;                 // generated source at a unit tile
  std::vector<int> items;
  std::unique_ptr<xs_handle> h;    // compiled at the chosen tile
  int G = 0, threads = 0, grid = 0, nunits = 0, gcd_traj = 0;
  bool tuned = false;
  double probe_us = 0;             // autotuner: probe microseconds per trajectory-step
  double work = 0;
  DevBuf d_items, d_units, d_next;
  cudaStream_t stream = nullptr;
  cudaEvent_t join = nullptr;
  ~BatchVariant() {
    if (join) cudaEventDestroy(join);
    if (stream) cudaStreamDestroy(stream);
  }
};

struct BatchEntry {
  std::unique_ptr<xs_handle> h;    // the item's problem; streaming items also run through it
  int variant = -1;                // resident variant, -1 = streaming path
  // check passes (xensemble.m:41-45): 1, or 2 with p.checks = 1 (pass 0 fine, nc = 1; pass 1
  // coarse, nc = 2 with twice the step and the mean of two fine draws)
  int passes = 1;
  size_t av_off = 0, param_off = 0;        // element offsets; pass q's means at av_off + q * av_pass
  size_t av_pass = 0;
  size_t part_off[2] = {0, 0}, prop_off[2] = {0, 0};
  int done_off = 0;                        // unit counter of pass q: d_done[done_off + q]
  int nunits = 0;
  double work = 0;                 // trajectory-steps x sites
};

int ntraj_of(const Problem& P) { return P.p.ensembles[0]; }


std::vector<cd> prop_table(const Problem& P, double dtr) {
  std::vector<cd> pr(P.L.size());
  const double dt = dtr / P.p.ipsteps;  // xpropfactor.m:28
  for (size_t i = 0; i < P.L.size(); ++i) pr[i] = std::exp(P.L[i] * dt);
  return pr;
}

// Tile chosen by the autotuner, cached per variant source and device.
std::string tile_cache_path() { return cache_dir() + "/batch_tiles.txt"; }

std::string tile_key(const std::string& src) {
  cudaDeviceProp prop{};
  int dev = 0;
  cudaGetDevice(&dev);
  cudaGetDeviceProperties(&prop, dev);
  char b[64];
  snprintf(b, sizeof b, "%016llx_%d", (unsigned long long)fnv1a(src + prop.name), prop.multiProcessorCount);
  return b;
}

bool tile_lookup(const std::string& key, int& G, int& threads) {
  std::ifstream f(tile_cache_path());
  std::string k;
  int g, t;
  while (f >> k >> g >> t)
    if (k == key) {
      G = g;
      threads = t;
      return true;
    }
  return false;
}

void tile_store(const std::string& key, int G, int threads) {
  mkdirs(cache_dir());
  std::ofstream f(tile_cache_path(), std::ios::app);
  f << key << " " << G << " " << threads << "\n";
}

}  // namespace

struct xs_batch {
  std::vector<std::unique_ptr<BatchVariant>> variants;
  std::vector<std::unique_ptr<BatchEntry>> items;
  DevBuf d_av, d_part, d_prop, d_params, d_done, d_status;
  size_t av_total = 0;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_join;
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool prepared = false;
  int launches_per_run = 0;
  ~xs_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto e : side_join) cudaEventDestroy(e);
    for (auto s : side) cudaStreamDestroy(s);
    if (fork) cudaEventDestroy(fork);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

void batch_drop_graph(xs_batch& b) {
  if (b.exec) cudaGraphExecDestroy(b.exec);
  if (b.graph) cudaGraphDestroy(b.graph);
  b.exec = nullptr;
  b.graph = nullptr;
  b.prepared = false;
}

// Candidate tiles of a variant: G trajectories per CTA (a power of two that
// divides every item's trajectory count and fits shared memory), threads.
std::vector<std::pair<int, int>> tile_candidates(const BatchVariant& v, const xs_handle& proto) {
  const Problem& P = proto.P;
  const int narr = method_arrays(P);
  if (resident_smem(proto, 1, narr) > 200 * 1024)  // field in device memory: one trajectory per CTA
    return {{1, 256}, {1, 512}, {1, 1024}};
  std::vector<int> Gs;  // divisors of every item's trajectory count, ascending
  for (int G = 1; G <= 4096 && G <= v.gcd_traj; ++G) {
    if (v.gcd_traj % G) continue;
    if (resident_smem(proto, G, narr) > 200 * 1024) break;
    if ((size_t)G * P.NS > 16384 && G > 1) break;
    Gs.push_back(G);
  }
  if (Gs.empty()) raise(XS_ERR_UNSUPPORTED, "no trajectory tile of this variant fits shared memory");
  std::vector<std::pair<int, int>> out;
  const int nG = (int)Gs.size();
  for (int i = std::max(0, nG - 3); i < nG; ++i) {
    const int G = Gs[i];
    const int items = G * P.NS * P.F;
    for (int t : {128, 256, 512})
      if (t <= std::max(128, (items + 31) / 32 * 32)) out.push_back({G, t});
  }
  return out;
}

std::unique_ptr<xs_handle> variant_handle(const xs_problem& raw, const Problem& P, bool fp64, int G, int threads) {
  auto h = std::make_unique<xs_handle>();
  h->P = P;  // grid, expressions and L already set up
  h->fp64 = fp64;
  h->path_kind = 1;
  h->force_G = G;
  h->force_threads = threads;
  (void)raw;
  build_source(*h);
  return h;
}

// Items table and longest-first unit queue of a variant at its tile.
void variant_tables(xs_batch& b, BatchVariant& v, int steps_cap, int points_cap, DevBuf& d_items, DevBuf& d_units,
                    void* part_base) {
  std::vector<BatchItemHost> its;
  std::vector<std::pair<double, std::pair<int, int>>> units;
  size_t part = 0;
  for (size_t k = 0; k < v.items.size(); ++k) {
    BatchEntry& e = *b.items[v.items[k]];
    const Problem& P = e.h->P;
    for (int q = 0; q < e.passes; ++q) {  // one table row per check pass
      BatchItemHost it{};
      it.ntraj = ntraj_of(P);
      it.steps = steps_cap > 0 ? std::min(P.p.steps, steps_cap) : P.p.steps;
      it.npoints = points_cap > 0 ? std::min(P.p.points[0], points_cap) : P.p.points[0];
      it.seq = P.p.sequence;
      it.seed = (unsigned)(P.p.seed & 0xffffffffu);
      it.block0 = 0;
      it.nunits = it.ntraj / v.G;
      it.nc = (short)(q + 1);
      it.checks = (short)(e.passes - 1);
      it.wscale = std::sqrt(P.nscale * P.noisefactor);  // xnoise.m:32
      it.vscale = std::sqrt(P.noisefactor);              // xrandom.m:22
      it.dtr = pass_dtr(P, q + 1);
      it.t0 = P.p.origins[0];
      it.prop = (const char*)b.d_prop.p + e.prop_off[q] * 16;
      it.prop2 = (const char*)b.d_prop.p + (e.prop_off[q] + (P.has_linear ? P.L.size() : 1)) * 16;
      const size_t stride = av_stride(P);
      if (part_base) {
        it.part = (char*)part_base + part * 16;
        part += (size_t)it.npoints * it.nunits * stride;
      } else {
        it.part = (char*)b.d_part.p + e.part_off[q] * 16;
      }
      it.av = (char*)b.d_av.p + (e.av_off + q * e.av_pass) * 16;
      it.params = P.runtime_defaults.empty() ? (const double*)b.d_params.p
                                             : (const double*)((const char*)b.d_params.p + e.param_off * 8);
      it.done = (int*)b.d_done.p + e.done_off + q;
      const int row = (int)its.size();
      its.push_back(it);
      // the fine pass of a checked item takes two steps per coarse step
      const double cost = (double)it.steps * it.npoints * (e.passes > 1 && q == 0 ? 2 : 1);
      for (int u = 0; u < it.nunits; ++u) units.push_back({cost, {row, u}});
    }
  }
  std::stable_sort(units.begin(), units.end(), [](const auto& a, const auto& c) { return a.first > c.first; });
  std::vector<int> flat;
  for (auto& u : units) {
    flat.push_back(u.second.first);
    flat.push_back(u.second.second);
  }
  d_items.ensure(its.size() * sizeof(BatchItemHost));
  CUDA_CHECK(cudaMemcpy(d_items.p, its.data(), its.size() * sizeof(BatchItemHost), cudaMemcpyHostToDevice));
  d_units.ensure(std::max<size_t>(flat.size(), 2) * sizeof(int));
  CUDA_CHECK(cudaMemcpy(d_units.p, flat.data(), flat.size() * sizeof(int), cudaMemcpyHostToDevice));
  v.nunits = (int)units.size();
}

void variant_launch(xs_batch& b, BatchVariant& v, const DevBuf& d_items, const DevBuf& d_units, cudaStream_t st) {
  xs_handle& h = *v.h;
  BatchArgsHost a{};
  a.items = d_items.p;
  a.units = d_units.p;
  a.nunits = v.nunits;
  a.next = (int*)v.d_next.p;
  a.status = (int*)b.d_status.p;
  a.tmat = h.d_tmat.p;
  for (int i = 0; i < 4; ++i) a.tmat_off[i] = h.tmat_off[i];
  a.gfield = h.d_gfield.p;
  void* params[] = {&a};
  cu_check(driver().launch(h.f_batch, (unsigned)v.grid, 1, 1, (unsigned)h.rp.threads, 1, 1, (unsigned)h.rp.smem,
                           (CUstream)st, params, nullptr),
           "launch xs_batch");
}

int variant_grid(BatchVariant& v) {
  if (v.h->rp.gfield) return resident_grid(*v.h, v.h->f_batch, v.nunits);
  int dev = 0, sms = 0, occ = 0;
  CUDA_CHECK(cudaGetDevice(&dev));
  CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  cu_check(driver().occupancy(&occ, v.h->f_batch, v.h->rp.threads, v.h->rp.smem), "occupancy");
  if (occ < 1) raise(XS_ERR_UNSUPPORTED, "batch tile cannot be resident on an SM");
  return std::max(1, std::min(v.nunits, sms * occ));
}

// Device buffers shared by all items: propagators, runtime scalars, means,
// partial sums, unit counters.
int batch_counters(const xs_batch& b);

void batch_buffers(xs_batch& b) {
  size_t prop = 0, par = 0, av = 0, part = 0;
  int done = 0;
  for (auto& ep : b.items) {
    BatchEntry& e = *ep;
    const Problem& P = e.h->P;
    const size_t stride = av_stride(P);
    e.av_off = av;
    e.av_pass = (size_t)P.p.points[0] * stride;
    av += e.passes * e.av_pass;
    e.done_off = done;
    done += e.passes;
    if (e.variant < 0) continue;
    const BatchVariant& v = *b.variants[e.variant];
    e.nunits = ntraj_of(P) / std::max(v.G, 1);
    e.param_off = par;
    par += P.runtime_defaults.size();
    for (int q = 0; q < e.passes; ++q) {
      e.prop_off[q] = prop;  // exp(L dtr/ipsteps), then exp(2 L dtr/ipsteps), dtr of pass q
      prop += 2 * (P.has_linear ? P.L.size() : 1);
      e.part_off[q] = part;
      part += (size_t)P.p.points[0] * e.nunits * stride;
    }
  }
  b.av_total = av;
  b.d_av.ensure(std::max<size_t>(av, 1) * 16);
  b.d_part.ensure(std::max<size_t>(part, 1) * 16);
  b.d_prop.ensure(std::max<size_t>(prop, 1) * 16);
  b.d_params.ensure(std::max<size_t>(par, 1) * 8);
  b.d_done.ensure(std::max<size_t>(done, 1) * sizeof(int));
  b.d_status.ensure(sizeof(int));
  std::vector<cd> hp(std::max<size_t>(prop, 1));
  std::vector<double> hpar(std::max<size_t>(par, 1));
  for (auto& ep : b.items) {
    BatchEntry& e = *ep;
    if (e.variant < 0) continue;
    const Problem& P = e.h->P;
    if (P.has_linear)
      for (int q = 0; q < e.passes; ++q) {
        const double dtr = pass_dtr(P, q + 1);
        auto pr = prop_table(P, dtr);
        std::copy(pr.begin(), pr.end(), hp.begin() + e.prop_off[q]);
        auto pr2 = prop_table(P, 2 * dtr);
        std::copy(pr2.begin(), pr2.end(), hp.begin() + e.prop_off[q] + pr.size());
      }
    std::copy(P.runtime_defaults.begin(), P.runtime_defaults.end(), hpar.begin() + e.param_off);
  }
  CUDA_CHECK(cudaMemcpy(b.d_prop.p, hp.data(), hp.size() * 16, cudaMemcpyHostToDevice));
  CUDA_CHECK(cudaMemcpy(b.d_params.p, hpar.data(), hpar.size() * 8, cudaMemcpyHostToDevice));
  CUDA_CHECK(cudaMemset(b.d_done.p, 0, std::max(done, 1) * sizeof(int)));
  CUDA_CHECK(cudaMemset(b.d_status.p, 0, sizeof(int)));
}

// unit counters of all items and passes (d_done)
int batch_counters(const xs_batch& b) {
  int n = 0;
  for (auto& ep : b.items) n += ep->passes;
  return std::max(n, 1);
}

void compile_all(std::vector<xs_handle*>& hs) {
  std::vector<std::string> errs(hs.size());
  std::vector<std::thread> th;
  const unsigned ncpu = std::max(1u, std::thread::hardware_concurrency());
  std::atomic<size_t> next{0};
  for (unsigned t = 0; t < std::min<unsigned>(ncpu, (unsigned)hs.size()); ++t)
    th.emplace_back([&]() {
      for (size_t i = next++; i < hs.size(); i = next++) {
        try {
          nvrtc_compile(hs[i]->source, "xs_resident", nullptr);
        } catch (const XsError& e) {
          errs[i] = e.msg;
        } catch (const std::exception& e) {
          errs[i] = e.what();
        }
      }
    });
  for (auto& t : th) t.join();
  for (auto& e : errs)
    if (!e.empty()) raise(XS_ERR_NVRTC, e);
}

// Choose each resident variant's tile.  mode 0: the largest tile that still
// gives every SM work; mode 1: time every candidate on a short probe (the
// variant's own items with steps and output points capped) and keep the
// fastest per trajectory-step; the choice is cached per source and device.
void batch_tune(xs_batch& b, int mode) {
  ensure_device();
  batch_drop_graph(b);
  int dev = 0, sms = 0;
  CUDA_CHECK(cudaGetDevice(&dev));
  CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (!b.stream) CUDA_CHECK(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
  for (auto& vp : b.variants) {
    BatchVariant& v = *vp;
    const BatchEntry& proto = *b.items[v.items[0]];
    auto cands = tile_candidates(v, *proto.h);
    const std::string tkey = tile_key(v.key);
    int G = 0, T = 0;
    bool cached = mode == 1 && tile_lookup(tkey, G, T);
    if (cached) {
      bool ok = false;
      for (auto& c : cands) ok = ok || (c.first == G && c.second == T);
      cached = ok;
    }
    if (!cached && mode == 0) {
      // largest G whose unit count still covers the SMs, 256 threads
      long long total = 0;
      for (int i : v.items) total += ntraj_of(b.items[i]->h->P);
      G = cands.front().first;
      for (auto& c : cands)
        if (total / c.first >= sms) G = std::max(G, c.first);
      T = 0;
      for (auto& c : cands)
        if (c.first == G && (T == 0 || std::abs(c.second - 256) < std::abs(T - 256))) T = c.second;
    }
    if (!cached && mode == 1) {
      std::vector<std::unique_ptr<xs_handle>> hs;
      std::vector<xs_handle*> raw;
      for (auto& c : cands) {
        hs.push_back(variant_handle(proto.h->P.p, proto.h->P, proto.h->fp64, c.first, c.second));
        raw.push_back(hs.back().get());
      }
      compile_all(raw);
      double best = 1e300;
      for (size_t ci = 0; ci < cands.size(); ++ci) {
        v.G = cands[ci].first;
        v.h = std::move(hs[ci]);
        load_module(*v.h);
        batch_buffers(b);
        DevBuf d_items, d_units, d_part;
        size_t part = 0;
        double ts = 0;
        for (int i : v.items) {
          const Problem& P = b.items[i]->h->P;
          const int np = b.items[i]->passes;
          part += np * (size_t)std::min(P.p.points[0], 1) * (ntraj_of(P) / v.G) * av_stride(P);
          ts += (double)ntraj_of(P) * std::min(P.p.steps, 8) * (np > 1 ? 3 : 1);
        }
        d_part.ensure(std::max<size_t>(part, 1) * 16);
        variant_tables(b, v, 8, 1, d_items, d_units, d_part.p);
        v.d_next.ensure(sizeof(int));
        v.grid = variant_grid(v);
        cudaEvent_t e0, e1;
        CUDA_CHECK(cudaEventCreate(&e0));
        CUDA_CHECK(cudaEventCreate(&e1));
        float ms = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
          CUDA_CHECK(cudaMemsetAsync(v.d_next.p, 0, sizeof(int), b.stream));
          CUDA_CHECK(cudaMemsetAsync(b.d_done.p, 0, batch_counters(b) * sizeof(int), b.stream));
          CUDA_CHECK(cudaEventRecord(e0, b.stream));
          variant_launch(b, v, d_items, d_units, b.stream);
          CUDA_CHECK(cudaEventRecord(e1, b.stream));
          CUDA_CHECK(cudaEventSynchronize(e1));
          float m = 0;
          CUDA_CHECK(cudaEventElapsedTime(&m, e0, e1));
          ms = std::min(ms, m);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        int st = 0;
        CUDA_CHECK(cudaMemcpy(&st, b.d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (st & 2) raise(XS_ERR_SHAPE, "batch probe refused its launch layout");
        const double us = 1e3 * ms / ts;
        if (us < best) {
          best = us;
          G = cands[ci].first;
          T = cands[ci].second;
        }
        hs[ci] = std::move(v.h);
      }
      v.probe_us = best;
      tile_store(tkey, G, T);
    }
    v.G = G;
    v.threads = T;
    v.h = variant_handle(proto.h->P.p, proto.h->P, proto.h->fp64, G, T);
    v.tuned = true;
  }
}

void batch_prepare(xs_batch& b) {
  if (b.prepared) return;
  for (auto& vp : b.variants)
    if (!vp->tuned) {
      batch_tune(b, 0);
      break;
    }
  ensure_device();
  if (!b.stream) CUDA_CHECK(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
  std::vector<xs_handle*> raw;
  for (auto& vp : b.variants) raw.push_back(vp->h.get());
  for (auto& ep : b.items)
    if (ep->variant < 0) raw.push_back(ep->h.get());
  {
    std::vector<xs_handle*> res, str;
    for (auto* h : raw) (h->kind >= 2 ? str : res).push_back(h);
    compile_all(res);
    std::vector<std::string> errs(str.size());
    std::vector<std::thread> th;
    for (size_t i = 0; i < str.size(); ++i)
      th.emplace_back([&, i]() {
        try {
          nvrtc_compile(str[i]->source, "xs_stream", nullptr);
        } catch (const XsError& e) {
          errs[i] = e.msg;
        }
      });
    for (auto& t : th) t.join();
    for (auto& e : errs)
      if (!e.empty()) raise(XS_ERR_NVRTC, e);
  }
  for (auto* h : raw) load_module(*h);
  batch_buffers(b);
  for (auto& vp : b.variants) {
    BatchVariant& v = *vp;
    variant_tables(b, v, 0, 0, v.d_items, v.d_units, nullptr);
    v.d_next.ensure(sizeof(int));
    v.grid = variant_grid(v);
    if (!v.stream) CUDA_CHECK(cudaStreamCreateWithFlags(&v.stream, cudaStreamNonBlocking));
    if (!v.join) CUDA_CHECK(cudaEventCreateWithFlags(&v.join, cudaEventDisableTiming));
  }
  // streaming items: buffers and propagators before capture (no uploads inside it)
  std::vector<int> sitems;
  for (size_t i = 0; i < b.items.size(); ++i)
    if (b.items[i]->variant < 0) {
      xs_handle& h = *b.items[i]->h;
      const Problem& P = h.P;
      h.d_field.ensure((size_t)P.E1 * P.F * P.NS * (h.fp64 ? 16 : 8));
      const int parts = h.kind == 3 ? P.N[2] : P.N[1] / h.sp.OROWS;  // reduction parts per trajectory
      if (P.nred) h.d_redpart.ensure((size_t)P.E1 * parts * P.nred * 16);
      if (P.nout_site) h.d_opart.ensure((size_t)kObsSplit * P.nout_site * P.NS * 16);
      for (int q = 1; q <= b.items[i]->passes; ++q) {
        ensure_prop(h, q);
        ensure_prop2(h, q);
      }
      sitems.push_back((int)i);
    }
  std::sort(sitems.begin(), sitems.end(), [&](int x, int y) { return b.items[x]->work > b.items[y]->work; });
  const int nside = (int)std::min<size_t>(sitems.size(), 4);
  while ((int)b.side.size() < nside) {
    cudaStream_t s;
    cudaEvent_t e;
    CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b.side.push_back(s);
    b.side_join.push_back(e);
  }
  if (!b.fork) CUDA_CHECK(cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming));
  CUDA_CHECK(cudaDeviceSynchronize());
  // capture: counters reset, then every variant and streaming chain forked from one event
  std::vector<size_t> order(b.variants.size());
  std::iota(order.begin(), order.end(), 0);
  for (auto& vp : b.variants) {
    vp->work = 0;
    for (int i : vp->items) vp->work += b.items[i]->work;
  }
  std::sort(order.begin(), order.end(), [&](size_t x, size_t y) { return b.variants[x]->work > b.variants[y]->work; });
  int launches = 0;
  CUDA_CHECK(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeRelaxed));
  try {
    CUDA_CHECK(cudaMemsetAsync(b.d_done.p, 0, batch_counters(b) * sizeof(int), b.stream));
    CUDA_CHECK(cudaMemsetAsync(b.d_status.p, 0, sizeof(int), b.stream));
    for (auto& vp : b.variants) CUDA_CHECK(cudaMemsetAsync(vp->d_next.p, 0, sizeof(int), b.stream));
    for (int i : sitems) CUDA_CHECK(cudaMemsetAsync(b.items[i]->h->d_status.p, 0, sizeof(int), b.stream));
    CUDA_CHECK(cudaEventRecord(b.fork, b.stream));
    for (size_t k : order) {
      BatchVariant& v = *b.variants[k];
      CUDA_CHECK(cudaStreamWaitEvent(v.stream, b.fork, 0));
      variant_launch(b, v, v.d_items, v.d_units, v.stream);
      ++launches;
      CUDA_CHECK(cudaEventRecord(v.join, v.stream));
    }
    for (int s = 0; s < nside; ++s) CUDA_CHECK(cudaStreamWaitEvent(b.side[s], b.fork, 0));
    for (size_t q = 0; q < sitems.size(); ++q) {
      BatchEntry& e = *b.items[sitems[q]];
      xs_handle& h = *e.h;
      const long long before = std::accumulate(std::begin(h.launches), std::end(h.launches), 0LL);
      for (int pass = 0; pass < e.passes; ++pass)
        launch_stream(h, 0, 1, pass + 1, nullptr, (char*)b.d_av.p + (e.av_off + pass * e.av_pass) * 16, nullptr,
                      b.side[q % nside]);
      launches += (int)(std::accumulate(std::begin(h.launches), std::end(h.launches), 0LL) - before);
    }
    for (int s = 0; s < nside; ++s) {
      CUDA_CHECK(cudaEventRecord(b.side_join[s], b.side[s]));
      CUDA_CHECK(cudaStreamWaitEvent(b.stream, b.side_join[s], 0));
    }
    for (auto& vp : b.variants) CUDA_CHECK(cudaStreamWaitEvent(b.stream, vp->join, 0));
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(b.stream, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  CUDA_CHECK(cudaStreamEndCapture(b.stream, &b.graph));
  CUDA_CHECK(cudaGraphInstantiate(&b.exec, b.graph, 0));
  b.launches_per_run = launches;
  b.prepared = true;
}

}  // namespace

XS_API xs_status xs_batch_create(const xs_problem* items, int nitems, xs_batch** out) {
  if (!out) return XS_ERR_ARG;
  *out = nullptr;
  return guard([&]() -> xs_status {
    if (!items || nitems < 1) raise(XS_ERR_ARG, "empty batch");
    auto b = std::make_unique<xs_batch>();
    std::map<std::string, int> vmap;
    for (int i = 0; i < nitems; ++i) {
      auto e = std::make_unique<BatchEntry>();
      e->h = std::make_unique<xs_handle>();
      xs_handle& h = *e->h;
      try {
        setup_problem(&items[i], h.P);
        h.fp64 = items[i].precision != XS_PREC_FP32;
        if (items[i].path_kind < 0 || items[i].path_kind > 2) raise(XS_ERR_ARG, "path_kind must be 0, 1 or 2");
        h.path_kind = items[i].path_kind;
        if (items[i].checks < 0 || items[i].checks > 1) raise(XS_ERR_UNSUPPORTED, "batch items take checks = 0 or 1");
        if (items[i].boundary_values) raise(XS_ERR_UNSUPPORTED, "batch items take no boundary values");
        if (h.P.spec) raise(XS_ERR_UNSUPPORTED, "batch items take no time-spectrum observables");
        if (h.P.NK || h.P.NKV) raise(XS_ERR_UNSUPPORTED, "batch items take no k-filtered noises");
        if (h.P.NA) raise(XS_ERR_UNSUPPORTED, "batch items take no auxiliary fields");
        if (items[i].ensembles[1] != 1 || items[i].ensembles[2] != 1)
          raise(XS_ERR_UNSUPPORTED, "a batch item is one ensemble block (ensembles(2) = ensembles(3) = 1)");
        h.force_G = 1;
        build_source(h);
      } catch (XsError& err) {
        err.msg = "batch item " + std::to_string(i) + ": " + err.msg;
        throw;
      }
      const Problem& P = h.P;
      e->passes = P.p.checks ? 2 : 1;
      e->work = (double)ntraj_of(P) * P.p.steps * std::max(1, P.p.points[0] - 1) * P.NS * (P.p.checks ? 3 : 1);
      if (h.kind == 1) {
        auto it = vmap.find(h.source);
        if (it == vmap.end()) {
          auto v = std::make_unique<BatchVariant>();
          v->key = h.source;
          it = vmap.emplace(h.source, (int)b->variants.size()).first;
          b->variants.push_back(std::move(v));
        }
        BatchVariant& v = *b->variants[it->second];
        e->variant = it->second;
        v.items.push_back(i);
        v.gcd_traj = std::gcd(v.gcd_traj, ntraj_of(P));
      } else {
        h.force_G = 0;
      }
      b->items.push_back(std::move(e));
    }
    *out = b.release();
    return XS_OK;
  });
}

XS_API void xs_batch_destroy(xs_batch* b) { delete b; }

XS_API xs_status xs_batch_tune(xs_batch* b, int mode) {
  return guard([&]() -> xs_status {
    if (!b || mode < 0 || mode > 1) raise(XS_ERR_ARG, "bad arguments to xs_batch_tune");
    batch_tune(*b, mode);
    return XS_OK;
  });
}

XS_API xs_status xs_batch_run(xs_batch* b, void* stream) {
  NvtxRange range("xs_batch_run");
  return guard([&]() -> xs_status {
    if (!b) raise(XS_ERR_ARG, "null batch");
    batch_prepare(*b);
    CUDA_CHECK(cudaGraphLaunch(b->exec, stream ? (cudaStream_t)stream : b->stream));
    return XS_OK;
  });
}

XS_API xs_status xs_batch_sync(xs_batch* b) {
  return guard([&]() -> xs_status {
    if (!b) raise(XS_ERR_ARG, "null batch");
    CUDA_CHECK(cudaDeviceSynchronize());
    int st = 0;
    if (b->d_status.p) CUDA_CHECK(cudaMemcpy(&st, b->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
    for (auto& ep : b->items)
      if (ep->variant < 0 && ep->h->d_status.p) {
        int s2 = 0;
        CUDA_CHECK(cudaMemcpy(&s2, ep->h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
        st |= s2;
      }
    if (st & 2) raise(XS_ERR_SHAPE, "kernel refused a launch whose shared-memory layout or grid did not match");
    if (st & 1) raise(XS_ERR_NAN, "a trajectory became non-finite (NaN/Inf)");
    return XS_OK;
  });
}

XS_API size_t xs_batch_av_doubles(const xs_batch* b, int item) {
  if (!b || item < 0 || item >= (int)b->items.size()) return 0;
  return b->items[item]->passes * av_doubles_per_block(b->items[item]->h->P);
}

XS_API xs_status xs_batch_results(xs_batch* b, int item, double* av_out) {
  return guard([&]() -> xs_status {
    if (!b || item < 0 || item >= (int)b->items.size() || !av_out) raise(XS_ERR_ARG, "bad arguments to xs_batch_results");
    if (!b->prepared) raise(XS_ERR_ARG, "xs_batch_run has not been called");
    const BatchEntry& e = *b->items[item];
    const Problem& P = e.h->P;
    const size_t n = (size_t)P.p.points[0] * av_stride(P) * 2;
    std::vector<double> dev(std::max<size_t>(n, 1));
    CUDA_CHECK(cudaStreamSynchronize(b->stream));
    for (int q = 0; q < e.passes; ++q) {  // fine pass, then (checks = 1) the coarse pass
      if (n)
        CUDA_CHECK(cudaMemcpy(dev.data(), (const char*)b->d_av.p + (e.av_off + q * e.av_pass) * 16, n * 8,
                              cudaMemcpyDeviceToHost));
      scatter_av(P, dev, 1, av_out + q * av_doubles_per_block(P));
    }
    return XS_OK;
  });
}

XS_API xs_status xs_batch_info(const xs_batch* b, int item, int* info, int ninfo) {
  return guard([&]() -> xs_status {
    if (!b || !info || ninfo < 1) raise(XS_ERR_ARG, "bad arguments to xs_batch_info");
    if (item < 0) {  // batch summary: items, variants, streaming items, launches per run
      int nst = 0;
      for (auto& ep : b->items) nst += ep->variant < 0;
      const int v[4] = {(int)b->items.size(), (int)b->variants.size(), nst, b->launches_per_run};
      for (int k = 0; k < ninfo && k < 4; ++k) info[k] = v[k];
      return XS_OK;
    }
    if (item >= (int)b->items.size()) raise(XS_ERR_ARG, "item index out of range");
    const BatchEntry& e = *b->items[item];
    int v[6] = {e.variant, e.variant < 0 ? 2 : 1, 0, 0, 0, 0};
    if (e.variant >= 0) {
      const BatchVariant& bv = *b->variants[e.variant];
      v[2] = bv.G;
      v[3] = bv.threads;
      v[4] = bv.grid;
      v[5] = e.nunits;
    }
    for (int k = 0; k < ninfo && k < 6; ++k) info[k] = v[k];
    return XS_OK;
  });
}
