/* xspde_path_mex.c -- MATLAB MEX binding of the B200 path to xSPDE's p.path hook.
 *
 *   [a, av, raw] = xspde_path_mex(a, nc, p)
 *
 * is a drop-in for the reference's default path function (Simulator/xpath.m:1,
 * set at Simulator/xpreferences.m:62 and called once per ensemble block, check
 * pass and sequence at Simulator/xensemble.m:79):
 *
 *   p.path = @(a, nc, p) xspde_path_mex(a, nc, p);
 *
 * Inputs and outputs are those of xpath: `a` is the cell array of field cells
 * (a{1} = [fields, space..., ens1] complex), `nc` the check index (1 fine,
 * 2 coarse), `p` the parameter struct after xpreferences; `av` is the cell of
 * block means av{o} with the dimensions p.d.av{o} = [lines, points(1), space]
 * (Simulator/xpreferences.m:340) and `raw` the cell raw{1} =
 * [fields, points(1), space..., ens1] when p.rawdata is set (xpath.m:73-78).
 *
 * The struct fields are copied into an xs_problem (include/xspde_b200.h) once
 * per distinct problem and the compiled handle is kept for the MATLAB session
 * (up to XSM_MAX_HANDLES problems; clear xspde_path_mex frees them):
 *   p.dimensions, p.fields{1}, p.noises{1}, p.inrandoms{1}, p.knoises{1},
 *   p.krandoms{1}, p.auxfields{1}, p.points{1}, p.ranges, p.origins,
 *   p.steps(1), p.checks(1), p.ensembles, p.method (func2str: MP, RK4, Euler,
 *   RK2, Implicit), p.iterations, p.ipsteps, p.seed, p.boundaries{1,d},
 *   p.deriv{1}, p.initial{1}, p.linear{1}, p.define{1}, p.observe{n} and
 *   p.transforms{n} (function handles as their func2str text), every real
 *   scalar field as a named constant p.<name>, p.nfilter{1} / p.rfilter{1}
 *   evaluated here on the k lattice, and p.boundfun evaluated here at every
 *   half step of the pass when the problem has non-periodic boundaries and a
 *   boundfun other than the default.  Optional extra fields that xSPDE
 *   ignores: p.precision = 'fp32' for the FP32-field mode (default FP64, the
 *   reference's precision) and p.sequence (0-based index of the input in a
 *   sequence, so each sequence draws its own noise as the Python host does).
 *
 * Ensemble block: xensemble seeds MATLAB's generator with
 * nsp = p.seed + npar + (j-1)*p.ensembles(3) before each path
 * (Simulator/xensemble.m:26,31); the binding reads that seed back through
 * rng() and uses block = nsp - p.seed - 1 = (npar-1) + (j-1)*ensembles(3) as the
 * Philox block key, so the noise of a block does not depend on which process
 * or in which order it runs (Octave seeds through randn('state'), where the
 * field p.block must be set instead).
 *
 * Errors come back as MATLAB errors with the library's message.  MATLAB is not
 * available where this repository is built, so this file is compiled and run
 * against a stand-in of the MEX API in the repository's tests.
 *
 * Build: mex -R2018a xspde_path_mex.c -I<repo>/include -L<repo>/xspde_matlab_b200 -lxspde_b200
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"
#include "xspde_b200.h"

#define XSM_MAX_HANDLES 16
#define XSM_MAX_OBS 64
#define XSM_MAX_PARAMS 256

typedef struct {
  char* sig;      /* text signature of the problem */
  xs_handle* h;
  int nobs;
  int bvals;      /* boundary values from p.boundfun */
  int bv_done[2]; /* boundary values set for check pass 1 / 2 */
} xsm_entry;

static xsm_entry g_handles[XSM_MAX_HANDLES];
static int g_nhandles = 0;

static void xsm_free_all(void) {
  for (int i = 0; i < g_nhandles; ++i) {
    xs_destroy(g_handles[i].h);
    free(g_handles[i].sig);
  }
  g_nhandles = 0;
}

static void xsm_fail(const char* id, const char* what) {
  char msg[2048];
  xs_last_error(msg, sizeof msg);
  mexErrMsgIdAndTxt(id, "%s: %s", what, msg);
}

/* ---- small helpers over the struct p ----------------------------------------------- */

static const mxArray* xsm_field(const mxArray* p, const char* name) { return mxGetField(p, 0, name); }

/* first cell of a cell field, or the field itself */
static const mxArray* xsm_cell1(const mxArray* f) {
  if (f && mxIsCell(f)) return mxGetNumberOfElements(f) ? mxGetCell(f, 0) : NULL;
  return f;
}

static double xsm_scalar(const mxArray* p, const char* name, double dflt) {
  const mxArray* f = xsm_cell1(xsm_field(p, name));
  if (!f || !mxIsNumeric(f) || mxIsEmpty(f)) return dflt;
  return mxGetScalar(f);
}

/* element k of a numeric vector field (first cell for cells) */
static double xsm_elem(const mxArray* f, size_t k, double dflt) {
  f = xsm_cell1(f);
  if (!f || !mxIsNumeric(f) || k >= mxGetNumberOfElements(f)) return dflt;
  return mxGetDoubles(f) ? mxGetDoubles(f)[k] : dflt;
}

/* func2str of a function handle (first cell for cells); NULL for a numeric or empty value.
 * The caller frees the result with mxFree. */
static char* xsm_fnstr(const mxArray* f) {
  f = xsm_cell1(f);
  if (!f || !mxIsClass(f, "function_handle")) return NULL;
  mxArray* in = (mxArray*)f;
  mxArray* out = NULL;
  if (mexCallMATLAB(1, &out, 1, &in, "func2str") != 0 || !out) return NULL;
  char* s = mxArrayToString(out);
  mxDestroyArray(out);
  return s;
}

static void xsm_sig_add(char** sig, size_t* len, const char* s) {
  const size_t n = strlen(s);
  *sig = (char*)realloc(*sig, *len + n + 2);
  memcpy(*sig + *len, s, n);
  (*sig)[*len + n] = '\x1f';
  (*sig)[*len + n + 1] = 0;
  *len += n + 1;
}

static void xsm_sig_num(char** sig, size_t* len, double v) {
  char b[64];
  snprintf(b, sizeof b, "%.17g", v);
  xsm_sig_add(sig, len, b);
}

/* complex copy of a numeric array as interleaved (re, im) doubles */
static mxArray* xsm_complex_copy(const mxArray* a) {
  mxArray* c = mxDuplicateArray(a);
  if (!mxIsComplex(c) && !mxMakeArrayComplex(c)) mexErrMsgIdAndTxt("xspde:path", "cannot make the field complex");
  return c;
}

/* ---- the problem ------------------------------------------------------------------ */

typedef struct {
  xs_problem pr;
  int bnd[(XS_MAXDIM - 1) * 64 * 2];
  char* texts[XSM_MAX_OBS + 8];
  int ntexts;
  const char* obs[XSM_MAX_OBS];
  int transforms[XSM_MAX_OBS * 4];
  const char* pnames[XSM_MAX_PARAMS];
  double pvals[XSM_MAX_PARAMS];
  double* nfilter;
  double* rfilter;
  int has_transforms;
  int bvals;
} xsm_problem;

static char* xsm_keep(xsm_problem* q, char* s) {
  if (s && q->ntexts < (int)(sizeof q->texts / sizeof q->texts[0])) q->texts[q->ntexts++] = s;
  return s;
}

static void xsm_release(xsm_problem* q) {
  for (int i = 0; i < q->ntexts; ++i) mxFree(q->texts[i]);
  free(q->nfilter);
  free(q->rfilter);
}

/* p.nfilter{1}(ones([n, space]), p) (Simulator/xnoise.m:42): the factor of each k-space
 * value, the k lattice in the propagation (FFT) order of p.kx, p.ky, p.kz */
static double* xsm_filter(const mxArray* p, const char* name, int ncomp) {
  const mxArray* fn = xsm_cell1(xsm_field(p, name));
  if (!fn || !mxIsClass(fn, "function_handle") || ncomp < 1) return NULL;
  const mxArray* pts = xsm_cell1(xsm_field(p, "points"));
  const int nd = (int)xsm_scalar(p, "dimensions", 1);
  mwSize dims[XS_MAXDIM] = {(mwSize)ncomp, 1, 1, 1};
  size_t nspace = 1;
  for (int d = 1; d < nd; ++d) {
    dims[d] = (mwSize)xsm_elem(pts, (size_t)d, 1);
    nspace *= dims[d];
  }
  mxArray* ones = mxCreateNumericArray((mwSize)(nd > 1 ? nd : 2), dims, mxDOUBLE_CLASS, mxREAL);
  double* o = mxGetDoubles(ones);
  for (size_t i = 0; i < (size_t)ncomp * nspace; ++i) o[i] = 1.0;
  mxArray* in[3] = {(mxArray*)fn, ones, (mxArray*)p};
  mxArray* out = NULL;
  if (mexCallMATLAB(1, &out, 3, in, "feval") != 0 || !out)
    mexErrMsgIdAndTxt("xspde:filter", "evaluating p.%s failed", name);
  mxArray* c = xsm_complex_copy(out);
  const size_t n = (size_t)ncomp * nspace;
  if (mxGetNumberOfElements(c) != n) mexErrMsgIdAndTxt("xspde:filter", "p.%s returned the wrong size", name);
  double* t = (double*)malloc(n * 2 * sizeof(double));
  memcpy(t, mxGetComplexDoubles(c), n * 2 * sizeof(double));
  mxDestroyArray(c);
  mxDestroyArray(out);
  mxDestroyArray(ones);
  return t;
}

static int xsm_method(const mxArray* p) {
  char* m = xsm_fnstr(xsm_field(p, "method"));
  int r = -1;
  if (m) {
    const char* b = strrchr(m, '.');
    b = b ? b + 1 : m;
    if (!strcmp(b, "MP")) r = XS_METHOD_MP;
    else if (!strcmp(b, "RK4")) r = XS_METHOD_RK4;
    else if (!strcmp(b, "Euler")) r = XS_METHOD_EULER;
    else if (!strcmp(b, "RK2")) r = XS_METHOD_RK2;
    else if (!strcmp(b, "Implicit")) r = XS_METHOD_IMPLICIT;
    mxFree(m);
  }
  if (r < 0) mexErrMsgIdAndTxt("xspde:method", "p.method must be MP, RK4, Euler, RK2 or Implicit on the device");
  return r;
}

/* Fill q from p; *sig receives the text signature that keys the handle cache. */
static void xsm_problem_from(const mxArray* p, xsm_problem* q, char** sig) {
  size_t slen = 0;
  memset(q, 0, sizeof *q);
  xs_problem* pr = &q->pr;
  const int nd = (int)xsm_scalar(p, "dimensions", 1);
  if (nd < 1 || nd > XS_MAXDIM) mexErrMsgIdAndTxt("xspde:shape", "p.dimensions must be 1..%d", XS_MAXDIM);
  pr->dimensions = nd;
  pr->fields = (int)xsm_scalar(p, "fields", 1);
  pr->noises = (int)xsm_scalar(p, "noises", 0);
  pr->inrandoms = (int)xsm_scalar(p, "inrandoms", 0);
  pr->knoises = (int)xsm_scalar(p, "knoises", 0);
  pr->krandoms = (int)xsm_scalar(p, "krandoms", 0);
  pr->auxfields = (int)xsm_scalar(p, "auxfields", 0);
  const mxArray* pts = xsm_field(p, "points");
  for (int d = 0; d < nd; ++d) {
    pr->points[d] = (int)xsm_elem(pts, (size_t)d, 1);
    pr->ranges[d] = xsm_elem(xsm_field(p, "ranges"), (size_t)d, 10.0);
    pr->origins[d] = xsm_elem(xsm_field(p, "origins"), (size_t)d, 0.0);
  }
  pr->steps = (int)xsm_elem(xsm_field(p, "steps"), 0, 1);
  pr->checks = (int)xsm_elem(xsm_field(p, "checks"), 0, 0);
  for (int k = 0; k < 3; ++k) pr->ensembles[k] = (int)xsm_elem(xsm_field(p, "ensembles"), (size_t)k, 1);
  pr->method = xsm_method(p);
  pr->iterations = (int)xsm_scalar(p, "iterations", 4);
  pr->ipsteps = (int)xsm_scalar(p, "ipsteps", pr->method >= XS_METHOD_EULER ? 1 : 2);
  pr->seed = (unsigned long long)xsm_scalar(p, "seed", 0);
  pr->sequence = (int)xsm_scalar(p, "sequence", 0);
  {
    const mxArray* pc = xsm_field(p, "precision");
    char* s = (pc && mxIsChar(pc)) ? mxArrayToString(pc) : NULL;
    pr->precision = (s && !strcmp(s, "fp32")) ? XS_PREC_FP32 : XS_PREC_FP64;
    if (s) mxFree(s);
  }
  /* p.boundaries{1,d}: [fields, 2] per space dimension (Applications/SPDE/spdpreferences.m:15,53-54) */
  const mxArray* bc = xsm_field(p, "boundaries");
  int any = 0;
  if (bc && mxIsCell(bc) && nd > 1) {
    const size_t rows = mxGetM(bc);
    if (pr->fields > 64) mexErrMsgIdAndTxt("xspde:shape", "at most 64 field components with boundaries");
    for (int d = 1; d < nd; ++d) {
      const mxArray* b = (size_t)d * rows < mxGetNumberOfElements(bc) ? mxGetCell(bc, (mwIndex)(d * rows)) : NULL;
      for (int f = 0; f < pr->fields; ++f)
        for (int e = 0; e < 2; ++e) {
          int v = 0;
          if (b && mxIsNumeric(b) && !mxIsEmpty(b)) v = (int)mxGetDoubles(b)[f + (size_t)mxGetM(b) * e];
          q->bnd[((d - 1) * pr->fields + f) * 2 + e] = v;
          any |= v != 0;
          xsm_sig_num(sig, &slen, v);
        }
    }
  }
  pr->boundaries = any ? q->bnd : NULL;
  /* function handles as text */
  pr->deriv = xsm_keep(q, xsm_fnstr(xsm_field(p, "deriv")));
  pr->initial = xsm_keep(q, xsm_fnstr(xsm_field(p, "initial")));
  pr->linear = xsm_keep(q, xsm_fnstr(xsm_field(p, "linear")));
  pr->define = pr->auxfields ? xsm_keep(q, xsm_fnstr(xsm_field(p, "define"))) : NULL;
  const mxArray* ob = xsm_field(p, "observe");
  const mxArray* tr = xsm_field(p, "transforms");
  int nobs = 0;
  if (ob && mxIsCell(ob)) {
    nobs = (int)mxGetNumberOfElements(ob);
    if (nobs > XSM_MAX_OBS) mexErrMsgIdAndTxt("xspde:shape", "at most %d observe functions", XSM_MAX_OBS);
    for (int n = 0; n < nobs; ++n) {
      char* s = xsm_fnstr(mxGetCell(ob, (mwIndex)n));
      if (s && strncmp(s, "@(", 2) != 0) {  /* a named function: only xSPDE's default xobserve is known */
        const int dflt = !strcmp(s, "xobserve");
        mxFree(s);
        if (!dflt) mexErrMsgIdAndTxt("xspde:grammar", "p.observe{%d} must be an anonymous function", n + 1);
        s = NULL;
      }
      q->obs[n] = s ? xsm_keep(q, s) : "@(a,p) a";
      for (int k = 0; k < 4; ++k) {
        const mxArray* tn = (tr && mxIsCell(tr) && (size_t)n < mxGetNumberOfElements(tr)) ? mxGetCell(tr, (mwIndex)n) : NULL;
        const int v = (int)xsm_elem(tn, (size_t)k, 0);
        q->transforms[n * 4 + k] = v;
        q->has_transforms |= v != 0;
        xsm_sig_num(sig, &slen, v);
      }
      xsm_sig_add(sig, &slen, q->obs[n]);
    }
  }
  pr->nobserve = nobs;
  pr->observe = q->obs;
  pr->transforms = q->has_transforms ? q->transforms : NULL;
  /* every real scalar field: the named constants p.<name> */
  const int nf = mxGetNumberOfFields(p);
  int np = 0;
  for (int i = 0; i < nf && np < XSM_MAX_PARAMS; ++i) {
    const mxArray* f = mxGetFieldByNumber(p, 0, i);
    if (!f || !mxIsDouble(f) || mxIsComplex(f) || mxGetNumberOfElements(f) != 1) continue;
    q->pnames[np] = mxGetFieldNameByNumber(p, i);
    q->pvals[np] = mxGetScalar(f);
    xsm_sig_add(sig, &slen, q->pnames[np]);
    xsm_sig_num(sig, &slen, q->pvals[np]);
    ++np;
  }
  pr->nparams = np;
  pr->param_names = q->pnames;
  pr->param_values = q->pvals;
  /* k-space filters */
  q->nfilter = pr->knoises ? xsm_filter(p, "nfilter", pr->knoises) : NULL;
  q->rfilter = pr->krandoms ? xsm_filter(p, "rfilter", pr->krandoms) : NULL;
  pr->nfilter = q->nfilter;
  pr->rfilter = q->rfilter;
  /* boundary values from a user p.boundfun (the default xboundfun gives zeros) */
  char* bf = any ? xsm_fnstr(xsm_field(p, "boundfun")) : NULL;
  q->bvals = bf && strcmp(bf, "xboundfun") != 0;
  if (bf) mxFree(bf);
  pr->boundary_values = q->bvals;
  /* the rest of the signature: everything the compiled kernels depend on */
  const char* texts[] = {pr->deriv ? pr->deriv : "", pr->initial ? pr->initial : "", pr->linear ? pr->linear : "",
                         pr->define ? pr->define : ""};
  for (int i = 0; i < 4; ++i) xsm_sig_add(sig, &slen, texts[i]);
  const double nums[] = {nd, pr->fields, pr->noises, pr->inrandoms, pr->knoises, pr->krandoms, pr->auxfields,
                         pr->points[0], pr->points[1], pr->points[2], pr->points[3], pr->ranges[0], pr->ranges[1],
                         pr->ranges[2], pr->ranges[3], pr->origins[0], pr->origins[1], pr->origins[2],
                         pr->origins[3], pr->steps, pr->checks, pr->ensembles[0], pr->ensembles[1],
                         pr->ensembles[2], pr->method, pr->iterations, pr->ipsteps, pr->precision,
                         (double)pr->seed, pr->sequence, q->bvals};
  for (size_t i = 0; i < sizeof nums / sizeof nums[0]; ++i) xsm_sig_num(sig, &slen, nums[i]);
  if (q->nfilter)
    for (size_t i = 0; i < 2 * (size_t)pr->knoises; ++i) xsm_sig_num(sig, &slen, q->nfilter[i]);
}

static xsm_entry* xsm_handle_for(const mxArray* p) {
  xsm_problem q;
  char* sig = NULL;
  xsm_problem_from(p, &q, &sig);
  for (int i = 0; i < g_nhandles; ++i)
    if (!strcmp(g_handles[i].sig, sig)) {
      free(sig);
      xsm_release(&q);
      return &g_handles[i];
    }
  if (g_nhandles == XSM_MAX_HANDLES) {  /* forget the oldest problem */
    xs_destroy(g_handles[0].h);
    free(g_handles[0].sig);
    memmove(g_handles, g_handles + 1, (XSM_MAX_HANDLES - 1) * sizeof g_handles[0]);
    --g_nhandles;
  }
  xs_handle* h = NULL;
  const xs_status st = xs_create(&q.pr, &h);
  const int nobs = q.pr.nobserve ? q.pr.nobserve : 1;
  const int bvals = q.bvals;
  xsm_release(&q);
  if (st != XS_OK) {
    free(sig);
    xsm_fail("xspde:create", "xs_create");
  }
  xsm_entry* e = &g_handles[g_nhandles++];
  e->sig = sig;
  e->h = h;
  e->nobs = nobs;
  e->bvals = bvals;
  e->bv_done[0] = e->bv_done[1] = 0;
  return e;
}

/* p.boundfun(a, 1, d, p) at t = origins(1) + k dtr/2 for every half step of check pass nc
 * (the times xprop/xsetbound query, Applications/SDE/MP.m:11-26), spatially constant values
 * b{i, end} taken from their first element; sent to the device once per pass. */
static void xsm_boundary_values(xsm_entry* e, const mxArray* a, int nc, const mxArray* p) {
  const int slot = nc == 2 ? 1 : 0;
  if (!e->bvals || e->bv_done[slot]) return;
  const int nd = (int)xsm_scalar(p, "dimensions", 1), F = (int)xsm_scalar(p, "fields", 1);
  const int P1 = (int)xsm_elem(xsm_field(p, "points"), 0, 1), S = (int)xsm_elem(xsm_field(p, "steps"), 0, 1);
  const int checks = (int)xsm_elem(xsm_field(p, "checks"), 0, 0);
  const double dt = xsm_scalar(p, "dt", 0), t0 = xsm_elem(xsm_field(p, "origins"), 0, 0);
  const int fine = checks && nc != 2;
  const double dtr = fine ? dt / (2 * S) : dt / S;
  const int nsteps = (P1 * S - 1) * (fine ? 2 : 1), ntimes = 2 * nsteps + 3;
  double* tab = (double*)calloc((size_t)ntimes * (nd - 1) * F * 2 * 2, sizeof(double));
  mxArray* q = mxDuplicateArray(p);
  const mxArray* fn = xsm_field(p, "boundfun");
  for (int k = 0; k < ntimes; ++k) {
    mxArray* tv = mxCreateDoubleScalar(t0 + k * dtr / 2);
    mxSetField(q, 0, "t", tv);
    for (int d = 1; d < nd; ++d) {
      mxArray* in[5] = {(mxArray*)fn, (mxArray*)a, mxCreateDoubleScalar(1), mxCreateDoubleScalar(d + 1), q};
      mxArray* out = NULL;
      if (mexCallMATLAB(1, &out, 5, in, "feval") != 0 || !out || !mxIsCell(out))
        mexErrMsgIdAndTxt("xspde:boundfun", "p.boundfun must return a cell of boundary values");
      for (int f = 0; f < F; ++f)
        for (int b = 0; b < 2; ++b) {
          const size_t r = mxGetM(out) > (size_t)f ? (size_t)f : 0;
          const mxArray* v = mxGetCell(out, (mwIndex)(r + mxGetM(out) * (size_t)b));
          double re = 0, im = 0;
          if (v && mxIsNumeric(v) && !mxIsEmpty(v)) {
            mxArray* c = xsm_complex_copy(v);
            re = mxGetComplexDoubles(c)[0].real;
            im = mxGetComplexDoubles(c)[0].imag;
            mxDestroyArray(c);
          }
          double* dst = tab + ((((size_t)k * (nd - 1) + (d - 1)) * F + f) * 2 + b) * 2;
          dst[0] = re;
          dst[1] = im;
        }
      mxDestroyArray(out);
      mxDestroyArray(in[2]);
      mxDestroyArray(in[3]);
    }
  }
  mxDestroyArray(q);
  const xs_status st = xs_set_boundary_values(e->h, nc, ntimes, tab);
  free(tab);
  if (st != XS_OK) xsm_fail("xspde:boundfun", "xs_set_boundary_values");
  e->bv_done[slot] = 1;
}

static int xsm_block(const mxArray* p) {
  const mxArray* b = xsm_field(p, "block");
  if (b && mxIsNumeric(b) && !mxIsEmpty(b)) return (int)mxGetScalar(b);
  mxArray* s = NULL;
  if (mexCallMATLAB(1, &s, 0, NULL, "rng") != 0 || !s || !mxIsStruct(s))
    mexErrMsgIdAndTxt("xspde:block", "cannot read the generator's seed (set p.block)");
  const mxArray* seed = mxGetField(s, 0, "Seed");
  const double nsp = seed ? mxGetScalar(seed) : 0;
  mxDestroyArray(s);
  const int block = (int)(nsp - xsm_scalar(p, "seed", 0) - 1);
  if (block < 0) mexErrMsgIdAndTxt("xspde:block", "generator seed below p.seed + 1 (set p.block)");
  return block;
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  mexAtExit(xsm_free_all);
  if (nrhs != 3 || !mxIsCell(prhs[0]) || !mxIsStruct(prhs[2]))
    mexErrMsgIdAndTxt("xspde:args", "usage: [a, av, raw] = xspde_path_mex(a, nc, p)");
  const mxArray* p = prhs[2];
  const int nc = (int)mxGetScalar(prhs[1]);
  if (nc != 1 && nc != 2) mexErrMsgIdAndTxt("xspde:args", "nc must be 1 or 2");
  xsm_entry* e = xsm_handle_for(p);
  const mxArray* a1 = mxGetCell(prhs[0], 0);
  if (!a1 || !mxIsDouble(a1)) mexErrMsgIdAndTxt("xspde:args", "a{1} must be a double array");
  xsm_boundary_values(e, prhs[0], nc, p);
  const int block = xsm_block(p);
  /* a{1} in, final field out: [fields, space..., ens1] complex, interleaved */
  mxArray* ain = xsm_complex_copy(a1);
  mxArray* aout = xsm_complex_copy(a1);
  const size_t per_block = xs_av_doubles_per_block(e->h);
  double* av = (double*)mxMalloc((per_block ? per_block : 2) * sizeof(double));
  const int rawdata = (int)xsm_scalar(p, "rawdata", 0);
  mxArray* raw = NULL;
  if (nlhs > 2 && rawdata) {  /* raw{1}: [fields, points(1), space..., ens1] (xpreferences.m:148) */
    const int nd = (int)xsm_scalar(p, "dimensions", 1);
    mwSize dims[XS_MAXDIM + 2];
    const mxArray* pts = xsm_field(p, "points");
    int k = 0;
    dims[k++] = (mwSize)xsm_scalar(p, "fields", 1);
    dims[k++] = (mwSize)xsm_elem(pts, 0, 1);
    for (int d = 1; d < nd; ++d) dims[k++] = (mwSize)xsm_elem(pts, (size_t)d, 1);
    dims[k++] = (mwSize)xsm_elem(xsm_field(p, "ensembles"), 0, 1);
    raw = mxCreateNumericArray((mwSize)k, dims, mxDOUBLE_CLASS, mxCOMPLEX);
  }
  const xs_status st = xs_run_path_raw(e->h, block, 1, nc, (const double*)mxGetComplexDoubles(ain), av,
                                       (double*)mxGetComplexDoubles(aout),
                                       raw ? (double*)mxGetComplexDoubles(raw) : NULL);
  mxDestroyArray(ain);
  if (st != XS_OK) {
    mxDestroyArray(aout);
    if (raw) mxDestroyArray(raw);
    mxFree(av);
    xsm_fail("xspde:path", "xs_run_path");
  }
  /* outputs: a (cell of field cells), av{o} with the dimensions p.d.av{o}, raw */
  const mwSize na = (mwSize)mxGetNumberOfElements(prhs[0]);
  plhs[0] = mxCreateCellMatrix(1, na);
  mxSetCell(plhs[0], 0, aout);
  for (mwSize c = 1; c < na; ++c) mxSetCell(plhs[0], c, mxDuplicateArray(mxGetCell(prhs[0], c)));
  if (nlhs > 1) {
    const mxArray* d = xsm_field(p, "d");
    const mxArray* dav = d ? mxGetField(d, 0, "av") : NULL;
    plhs[1] = mxCreateCellMatrix(1, (mwSize)e->nobs);
    size_t off = 0;
    for (int o = 0; o < e->nobs; ++o) {
      int lines = 0, spatial = 0;
      if (xs_observe_info(e->h, o, &lines, &spatial) != XS_OK) xsm_fail("xspde:path", "xs_observe_info");
      const mxArray* pts = xsm_field(p, "points");
      size_t n = (size_t)lines * (size_t)xsm_elem(pts, 0, 1);
      if (spatial) {  /* the lattice, with the dimensions a partial Int/Ave reduces of size 1 */
        int shp[3] = {1, 1, 1};
        if (xs_observe_shape(e->h, o, shp) != XS_OK) xsm_fail("xspde:path", "xs_observe_shape");
        for (int dd = 1; dd < (int)xsm_scalar(p, "dimensions", 1) && dd <= 3; ++dd) n *= (size_t)shp[dd - 1];
      }
      const mxArray* dims = (dav && mxIsCell(dav) && (size_t)o < mxGetNumberOfElements(dav)) ? mxGetCell(dav, (mwIndex)o) : NULL;
      mxArray* out;
      if (dims && mxIsNumeric(dims) && mxGetNumberOfElements(dims) >= 2) {
        const size_t nd = mxGetNumberOfElements(dims);
        mwSize dv[8];
        size_t prod = 1;
        for (size_t k = 0; k < nd && k < 8; ++k) {
          dv[k] = (mwSize)mxGetDoubles(dims)[k];
          prod *= dv[k];
        }
        out = prod == n ? mxCreateNumericArray((mwSize)(nd < 8 ? nd : 8), dv, mxDOUBLE_CLASS, mxCOMPLEX)
                        : mxCreateNumericMatrix((mwSize)n, 1, mxDOUBLE_CLASS, mxCOMPLEX);
      } else {
        out = mxCreateNumericMatrix((mwSize)n, 1, mxDOUBLE_CLASS, mxCOMPLEX);
      }
      memcpy(mxGetComplexDoubles(out), av + 2 * off, n * 2 * sizeof(double));
      off += n;
      mxSetCell(plhs[1], (mwIndex)o, out);
    }
  }
  mxFree(av);
  if (nlhs > 2) {
    plhs[2] = mxCreateCellMatrix(1, 1);
    if (raw) mxSetCell(plhs[2], 0, raw);
  } else if (raw) {
    mxDestroyArray(raw);
  }
}
