/* Host stand-in for the MATLAB MEX runtime (see mex.h beside this file): just
 * enough of mxArray -- double arrays (real or interleaved complex), cells,
 * 1x1 structs, char arrays and function handles that remember their text --
 * for the tests to run xspde_path_mex.c without MATLAB.  mexCallMATLAB knows
 * func2str (the handle's text) and rng (a struct whose Seed is
 * fake_mex_rng_seed); an error raised with mexErrMsgIdAndTxt prints the message
 * and exits with status 3. */
#define _POSIX_C_SOURCE 200809L
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
  mxClassID cls;
  int complex;
  mwSize nd;
  mwSize dims[8];
  double* data;      /* numeric: n (real) or 2n (complex, interleaved) doubles */
  mxArray** cells;   /* cell: n entries; struct: nfields values */
  char** names;      /* struct: field names */
  int nfields;
  char* text;        /* char array or function-handle text */
};

double fake_mex_rng_seed = 0;

static size_t numel(const mxArray* a) {
  size_t n = 1;
  for (mwSize i = 0; i < a->nd; ++i) n *= a->dims[i];
  return n;
}

static mxArray* alloc(mxClassID c) {
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = c;
  a->nd = 2;
  a->dims[0] = a->dims[1] = 1;
  return a;
}

mxArray* fake_struct(void) { return alloc(mxSTRUCT_CLASS); }
mxArray* fake_handle(const char* text) {
  mxArray* a = alloc(mxFUNCTION_CLASS);
  a->text = strdup(text);
  return a;
}
mxArray* fake_string(const char* text) {
  mxArray* a = alloc(mxCHAR_CLASS);
  a->text = strdup(text);
  a->dims[1] = strlen(text);
  return a;
}
mxArray* fake_row(int n, const double* v) {
  mxArray* a = mxCreateNumericMatrix(1, (mwSize)n, mxDOUBLE_CLASS, mxREAL);
  memcpy(a->data, v, (size_t)n * sizeof(double));
  return a;
}
mxArray* fake_cell1(mxArray* v) {
  mxArray* c = mxCreateCellMatrix(1, 1);
  mxSetCell(c, 0, v);
  return c;
}

mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name) {
  (void)i;
  if (!s || s->cls != mxSTRUCT_CLASS) return NULL;
  for (int k = 0; k < s->nfields; ++k)
    if (!strcmp(s->names[k], name)) return s->cells[k];
  return NULL;
}
void mxSetField(mxArray* s, mwIndex i, const char* name, mxArray* v) {
  (void)i;
  for (int k = 0; k < s->nfields; ++k)
    if (!strcmp(s->names[k], name)) {
      if (s->cells[k]) mxDestroyArray(s->cells[k]);
      s->cells[k] = v;
      return;
    }
  s->names = (char**)realloc(s->names, (size_t)(s->nfields + 1) * sizeof(char*));
  s->cells = (mxArray**)realloc(s->cells, (size_t)(s->nfields + 1) * sizeof(mxArray*));
  s->names[s->nfields] = strdup(name);
  s->cells[s->nfields] = v;
  ++s->nfields;
}
int mxGetNumberOfFields(const mxArray* s) { return s->nfields; }
mxArray* mxGetFieldByNumber(const mxArray* s, mwIndex i, int k) { (void)i; return s->cells[k]; }
const char* mxGetFieldNameByNumber(const mxArray* s, int k) { return s->names[k]; }
mxArray* mxGetCell(const mxArray* c, mwIndex i) { return i < numel(c) ? c->cells[i] : NULL; }
void mxSetCell(mxArray* c, mwIndex i, mxArray* v) { c->cells[i] = v; }
bool mxIsCell(const mxArray* a) { return a && a->cls == mxCELL_CLASS; }
bool mxIsStruct(const mxArray* a) { return a && a->cls == mxSTRUCT_CLASS; }
bool mxIsChar(const mxArray* a) { return a && a->cls == mxCHAR_CLASS; }
bool mxIsNumeric(const mxArray* a) { return a && a->cls == mxDOUBLE_CLASS; }
bool mxIsDouble(const mxArray* a) { return a && a->cls == mxDOUBLE_CLASS; }
bool mxIsComplex(const mxArray* a) { return a && a->complex; }
bool mxIsEmpty(const mxArray* a) { return numel(a) == 0; }
bool mxIsClass(const mxArray* a, const char* name) {
  if (!a) return false;
  if (!strcmp(name, "function_handle")) return a->cls == mxFUNCTION_CLASS;
  if (!strcmp(name, "cell")) return a->cls == mxCELL_CLASS;
  if (!strcmp(name, "double")) return a->cls == mxDOUBLE_CLASS;
  return false;
}
size_t mxGetNumberOfElements(const mxArray* a) { return a->cls == mxSTRUCT_CLASS ? 1 : numel(a); }
size_t mxGetM(const mxArray* a) { return a->dims[0]; }
double mxGetScalar(const mxArray* a) { return (a->cls == mxDOUBLE_CLASS && numel(a)) ? a->data[0] : 0.0; }
mxDouble* mxGetDoubles(const mxArray* a) { return (a->cls == mxDOUBLE_CLASS && !a->complex) ? a->data : NULL; }
mxComplexDouble* mxGetComplexDoubles(const mxArray* a) {
  return (a->cls == mxDOUBLE_CLASS && a->complex) ? (mxComplexDouble*)a->data : NULL;
}
int mxMakeArrayComplex(mxArray* a) {
  if (a->complex) return 1;
  const size_t n = numel(a);
  double* d = (double*)calloc(2 * (n ? n : 1), sizeof(double));
  for (size_t i = 0; i < n; ++i) d[2 * i] = a->data[i];
  free(a->data);
  a->data = d;
  a->complex = 1;
  return 1;
}
mxArray* mxDuplicateArray(const mxArray* a) {
  mxArray* b = (mxArray*)calloc(1, sizeof(mxArray));
  *b = *a;
  if (a->text) b->text = strdup(a->text);
  if (a->data) {
    const size_t n = numel(a) * (a->complex ? 2 : 1);
    b->data = (double*)malloc((n ? n : 1) * sizeof(double));
    memcpy(b->data, a->data, n * sizeof(double));
  }
  const int nc = a->cls == mxCELL_CLASS ? (int)numel(a) : (a->cls == mxSTRUCT_CLASS ? a->nfields : 0);
  if (nc) {
    b->cells = (mxArray**)calloc((size_t)nc, sizeof(mxArray*));
    for (int i = 0; i < nc; ++i) b->cells[i] = a->cells[i] ? mxDuplicateArray(a->cells[i]) : NULL;
  }
  if (a->cls == mxSTRUCT_CLASS && nc) {
    b->names = (char**)calloc((size_t)nc, sizeof(char*));
    for (int i = 0; i < nc; ++i) b->names[i] = strdup(a->names[i]);
  }
  return b;
}
void mxDestroyArray(mxArray* a) {
  if (!a) return;
  const int nc = a->cls == mxCELL_CLASS ? (int)numel(a) : (a->cls == mxSTRUCT_CLASS ? a->nfields : 0);
  for (int i = 0; i < nc; ++i) mxDestroyArray(a->cells[i]);
  if (a->names)
    for (int i = 0; i < a->nfields; ++i) free(a->names[i]);
  free(a->names);
  free(a->cells);
  free(a->data);
  free(a->text);
  free(a);
}
mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID c, mxComplexity x) {
  mxArray* a = alloc(c);
  a->nd = nd;
  for (mwSize i = 0; i < nd && i < 8; ++i) a->dims[i] = dims[i];
  a->complex = x == mxCOMPLEX;
  const size_t n = numel(a) * (a->complex ? 2 : 1);
  a->data = (double*)calloc(n ? n : 1, sizeof(double));
  return a;
}
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x) {
  const mwSize d[2] = {m, n};
  return mxCreateNumericArray(2, d, c, x);
}
mxArray* mxCreateDoubleScalar(double v) {
  mxArray* a = mxCreateNumericMatrix(1, 1, mxDOUBLE_CLASS, mxREAL);
  a->data[0] = v;
  return a;
}
mxArray* mxCreateCellMatrix(mwSize m, mwSize n) {
  mxArray* a = alloc(mxCELL_CLASS);
  a->dims[0] = m;
  a->dims[1] = n;
  const size_t cnt = (size_t)m * (size_t)n;
  a->cells = (mxArray**)calloc(cnt > 0 ? cnt : 1, sizeof(mxArray*));
  return a;
}
char* mxArrayToString(const mxArray* a) { return a->text ? strdup(a->text) : NULL; }
void* mxMalloc(size_t n) { return malloc(n); }
void mxFree(void* p) { free(p); }
int mexCallMATLAB(int nlhs, mxArray* plhs[], int nrhs, mxArray* prhs[], const char* name) {
  (void)nlhs;
  if (!strcmp(name, "func2str") && nrhs == 1 && prhs[0]->cls == mxFUNCTION_CLASS) {
    plhs[0] = fake_string(prhs[0]->text);
    return 0;
  }
  if (!strcmp(name, "rng") && nrhs == 0) {
    plhs[0] = fake_struct();
    mxSetField(plhs[0], 0, "Seed", mxCreateDoubleScalar(fake_mex_rng_seed));
    return 0;
  }
  return 1;
}
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, "%s: ", id);
  vfprintf(stderr, fmt, ap);
  fprintf(stderr, "\n");
  va_end(ap);
  exit(3);
}
int mexAtExit(void (*fn)(void)) {
  (void)fn;
  return 0;
}
