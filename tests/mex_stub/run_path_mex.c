/* Test driver for the MEX binding: builds the parameter struct that xSPDE's
 * xpreferences would hand to p.path for a small 1D stochastic NLS problem
 * (cells for fields, noises, points, deriv, initial, linear, observe,
 * boundaries; d.av; a named scalar p.g used by the drift), sets the
 * generator seed the way xensemble does (nsp = p.seed + npar + (j-1)
 * ensembles(3)), calls mexFunction and writes the outputs.
 *
 *   run_path_mex <a_in.bin> <block> <nc> <out.bin>
 *
 * a_in.bin: the initial field a{1} = [1, 32, 4] complex, interleaved doubles.
 * out.bin: av{1}, av{2} ([1, 5, 32] complex each), the final field a{1}, raw{1}
 * ([1, 5, 32, 4] complex), all interleaved doubles, plus 8 int64 holding the
 * dimensions of av{1} and raw{1} as the binding created them. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

extern double fake_mex_rng_seed;
mxArray* fake_struct(void);
mxArray* fake_handle(const char* text);
mxArray* fake_string(const char* text);
mxArray* fake_row(int n, const double* v);
mxArray* fake_cell1(mxArray* v);

static mxArray* field_cell(mxArray* v) { return fake_cell1(v); }

int main(int argc, char** argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: run_path_mex a_in.bin block nc out.bin\n");
    return 2;
  }
  const int block = atoi(argv[2]), nc = atoi(argv[3]);
  const int NX = 32, P1 = 5, E1 = 4;
  mxArray* p = fake_struct();
  mxSetField(p, 0, "dimensions", mxCreateDoubleScalar(2));
  mxSetField(p, 0, "fields", field_cell(mxCreateDoubleScalar(1)));
  mxSetField(p, 0, "noises", field_cell(mxCreateDoubleScalar(2)));
  mxSetField(p, 0, "inrandoms", field_cell(mxCreateDoubleScalar(2)));
  mxSetField(p, 0, "knoises", field_cell(mxCreateNumericMatrix(0, 0, mxDOUBLE_CLASS, mxREAL)));
  const double pts[2] = {P1, NX}, rng[2] = {0.5, 10.0}, org[2] = {0.0, -5.0}, st[2] = {2, 1}, ck[2] = {1, 0};
  const double ens[3] = {E1, 2, 1};
  mxSetField(p, 0, "points", field_cell(fake_row(2, pts)));
  mxSetField(p, 0, "ranges", fake_row(2, rng));
  mxSetField(p, 0, "origins", fake_row(2, org));
  mxSetField(p, 0, "steps", fake_row(2, st));
  mxSetField(p, 0, "checks", fake_row(2, ck));
  mxSetField(p, 0, "ensembles", fake_row(3, ens));
  mxSetField(p, 0, "method", fake_handle("MP"));
  mxSetField(p, 0, "iterations", mxCreateDoubleScalar(4));
  mxSetField(p, 0, "ipsteps", mxCreateDoubleScalar(2));
  mxSetField(p, 0, "seed", mxCreateDoubleScalar(7));
  mxSetField(p, 0, "dt", mxCreateDoubleScalar(0.125));
  mxSetField(p, 0, "rawdata", mxCreateDoubleScalar(1));
  mxSetField(p, 0, "g", mxCreateDoubleScalar(0.01));
  mxSetField(p, 0, "deriv", field_cell(fake_handle("@(a,w,p) 1i*a.*conj(a).*a + p.g*(w(1,:)+1i*w(2,:))/sqrt(2)")));
  mxSetField(p, 0, "initial", field_cell(fake_handle("@(v,p) exp(-p.x.^2)")));
  mxSetField(p, 0, "linear", field_cell(fake_handle("@(p) 1i*p.Dx.^2")));
  mxArray* obs = mxCreateCellMatrix(1, 2);
  mxSetCell(obs, 0, fake_handle("@(a,p) a.*conj(a)"));
  mxSetCell(obs, 1, fake_handle("@(a,p) real(a)"));
  mxSetField(p, 0, "observe", obs);
  mxArray* tr = mxCreateCellMatrix(1, 2);
  const double z4[4] = {0, 0, 0, 0};
  mxSetCell(tr, 0, fake_row(4, z4));
  mxSetCell(tr, 1, fake_row(4, z4));
  mxSetField(p, 0, "transforms", tr);
  mxArray* bnd = mxCreateCellMatrix(2, 2);  /* p.boundaries{nc+1, nd}: periodic */
  const double z2[2] = {0, 0};
  mxSetCell(bnd, 2, fake_row(2, z2));
  mxSetField(p, 0, "boundaries", bnd);
  mxSetField(p, 0, "boundfun", fake_handle("xboundfun"));
  mxArray* d = fake_struct();
  mxArray* dav = mxCreateCellMatrix(1, 2);
  const double avd[3] = {1, P1, NX};
  mxSetCell(dav, 0, fake_row(3, avd));
  mxSetCell(dav, 1, fake_row(3, avd));
  mxSetField(d, 0, "av", dav);
  mxSetField(p, 0, "d", d);
  /* a{1}: [1, NX, E1] complex from the file */
  const mwSize adims[3] = {1, (mwSize)NX, (mwSize)E1};
  mxArray* a1 = mxCreateNumericArray(3, adims, mxDOUBLE_CLASS, mxCOMPLEX);
  FILE* f = fopen(argv[1], "rb");
  if (!f || fread(mxGetComplexDoubles(a1), sizeof(double), 2 * NX * E1, f) != (size_t)(2 * NX * E1)) return 2;
  fclose(f);
  mxArray* a = fake_cell1(a1);
  /* xensemble: rng(nsp) with nsp = p.seed + npar + (j-1)*ensembles(3) */
  fake_mex_rng_seed = 7 + 1 + block;
  mxArray* ncv = mxCreateDoubleScalar(nc);
  mxArray* plhs[3] = {NULL, NULL, NULL};
  const mxArray* prhs[3] = {a, ncv, p};
  mexFunction(3, plhs, 3, prhs);
  FILE* o = fopen(argv[4], "wb");
  for (int k = 0; k < 2; ++k) {
    const mxArray* av = mxGetCell(plhs[1], (mwIndex)k);
    fwrite(mxGetComplexDoubles(av), sizeof(double), 2 * mxGetNumberOfElements(av), o);
  }
  const mxArray* af = mxGetCell(plhs[0], 0);
  fwrite(mxGetComplexDoubles(af), sizeof(double), 2 * mxGetNumberOfElements(af), o);
  const mxArray* raw = mxGetCell(plhs[2], 0);
  fwrite(mxGetComplexDoubles(raw), sizeof(double), 2 * mxGetNumberOfElements(raw), o);
  long long dims[8] = {0};
  const mxArray* av0 = mxGetCell(plhs[1], 0);
  dims[0] = (long long)mxGetM(av0);
  dims[1] = (long long)mxGetNumberOfElements(av0);
  dims[2] = (long long)mxGetM(raw);
  dims[3] = (long long)mxGetNumberOfElements(raw);
  fwrite(dims, sizeof(long long), 8, o);
  fclose(o);
  return 0;
}
