// MATLAB anonymous-function subset -> AST -> CUDA device code / FP64 host evaluation.
//
// xSPDE users write the drift (p.deriv), initial condition (p.initial),
// observables (p.observe) and linear operator (p.linear) as MATLAB anonymous
// functions, e.g. "@(a,w,p) 1i*a.*conj(a).*a + 0.01*w(1,:)".  The reference
// evaluates them as MATLAB code (Applications/SDE/MP.m:16, Simulator/xdata.m:30,
// Applications/SPDE/xpropfactor.m:38).  Here the same text is parsed once:
// pointwise functions become device code inside the fused kernel; the linear
// operator is evaluated in FP64 on the host to build exp(L dt).  Anything
// outside the grammar is rejected with a message -- there is no CPU fallback.
#pragma once
#include <complex>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace xs {

struct GrammarError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

enum class NK { Num, Imag, Var, Field, Index, Call, Bin, Un, Concat, Colon, CellIndex };

struct Node {
  NK kind;
  double num = 0;            // Num / Imag
  std::string name;          // Var / Field (p.<name>) / Call (function) / Bin / Un operator
  std::vector<std::shared_ptr<Node>> kids;
  std::vector<std::vector<std::shared_ptr<Node>>> rows;  // Concat
};
using NodeP = std::shared_ptr<Node>;

struct AnonFn {
  std::vector<std::string> params;  // "~" for ignored
  NodeP body;
  std::string text;
};

AnonFn parse_anon(const std::string& text);

// Roles of the anonymous function's arguments.
enum class Role { Field, Noise, Random, Params, Ignored, Aux, KNoise, KRandom };

struct Scalars {
  std::map<std::string, double> values;  // p.<name> constants
};

// Context for code generation of a pointwise function.
struct GenCtx {
  std::vector<Role> roles;   // per positional argument
  int nfield = 1;            // components of the field a
  int nnoise = 0;            // components of w
  int nrand = 0;             // components of v
  int nknoise = 0;           // components of the k-filtered noise (complex, zk[])
  int nkrand = 0;            // components of the k-filtered randoms (complex, vk[])
  int naux = 0;              // components of the auxiliary cell (complex, xa[]; observe only)
  int ndim = 0;              // space dimensions
  bool allow_reduce = false; // Int/Ave allowed (observe)
  bool kgrid = false;        // p.kx/ky/kz available as site values (observe): xs_kt<d>[i<d>]
  const Scalars* scalars = nullptr;
  const std::vector<std::string>* runtime = nullptr;  // p.<name> read at run time as prm[k]
  std::vector<double> dx, dk, origins, ranges;  // index 0 = time
  double dt = 0;
};

// Reduction slot discovered in an observe function: Int/Ave of a pointwise integrand.
struct Reduction {
  bool ave = false;                  // Ave (mean) instead of Int (sum*dx)
  std::vector<int> dims;             // space dims (1-based, 1 = x) reduced
  std::vector<double> weight;        // per reduced dim multiplier (dx or dk or 1/N)
  std::vector<double> lo, hi;        // bounds per dim (lo >= hi: all points)
  int lines = 1;                     // components of the integrand
  std::string integrand_code;        // device statements writing r[0..lines)
};

struct Generated {
  int len = 1;                       // components of the result
  bool is_complex = true;   // the result has an imaginary part (else out[i].im = 0)
  std::string code;                  // device statements; result in out[0..len)
  std::vector<Reduction> reductions; // observe only
  bool uses_k = false;               // needs k-space field (not supported: error)
  bool stencil = false;              // D1/D2 finite differences: reads neighbouring sites of the field
  bool spatial = true;               // result depends on the lattice site
};

// Generate device code for a pointwise function.  Variables available in the
// emitted code: `a` (const cx*), `w` (const real*), `v` (const real*),
// `x`,`y`,`z` (real site coordinates), `t` (real time), output array `out`.
// For observe functions with Int/Ave, reduced values are read from `red`.
Generated generate(const AnonFn& fn, const GenCtx& ctx);

// Additive split of a drift D(a, ...) = dep(a, ...) + inv(...) along the terms of its outermost
// sum (per component of a top-level [e1; e2; ...]): `inv` collects the terms that do not read the
// field a.  The midpoint iterations of MP evaluate a = a0 + h D(a) several times with the same
// noise; they compute `start`: out = c0 + h inv once per site (with c0 = a0), then `step`:
// out = c0 + h dep(a) in each iteration.  In the emitted code h is a real scalar `h` and c0 a
// complex array `c0`; h is pushed through sums and into one scalar factor of each product (with
// literal factors folded into it) so that the updates contract into fused multiply-adds.  Both
// have len components (complex).  Returns false when either part would be empty (no gain).
bool generate_split(const AnonFn& fn, const GenCtx& ctx, Generated& start, Generated& step);

// Host FP64 evaluation of the linear operator on the propagation grid:
// returns L per (component, site) with component count 1 or F.
struct GridInfo {
  int ndim = 0;
  std::vector<int> n;                                   // points per space dim
  std::vector<std::vector<std::vector<double>>> k;      // [field][dim][i] k grid (propagation order)
  std::vector<std::vector<double>> x;                   // [dim][i] coordinates
  int nfield = 1;
};
std::vector<std::complex<double>> eval_linear(const AnonFn& fn, const GridInfo& g, const Scalars& sc,
                                              int* ncomp_out);

}  // namespace xs
