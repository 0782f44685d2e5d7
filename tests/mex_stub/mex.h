/* Stand-in for MATLAB's mex.h (R2018a interleaved-complex API), for the tests:
 * declares the part of the MEX/mx API that xspde_matlab_b200/mex/xspde_path_mex.c
 * uses.  fake_mex.c implements it on the host so that the binding can be
 * compiled and run without MATLAB. */
#ifndef XS_TEST_MEX_H
#define XS_TEST_MEX_H
#include <stddef.h>
#include <stdbool.h>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef enum { mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxCHAR_CLASS, mxDOUBLE_CLASS,
               mxFUNCTION_CLASS } mxClassID;
typedef struct { double real, imag; } mxComplexDouble;
typedef double mxDouble;

mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name);
void mxSetField(mxArray* s, mwIndex i, const char* name, mxArray* v);
int mxGetNumberOfFields(const mxArray* s);
mxArray* mxGetFieldByNumber(const mxArray* s, mwIndex i, int k);
const char* mxGetFieldNameByNumber(const mxArray* s, int k);
mxArray* mxGetCell(const mxArray* c, mwIndex i);
void mxSetCell(mxArray* c, mwIndex i, mxArray* v);
bool mxIsCell(const mxArray* a);
bool mxIsStruct(const mxArray* a);
bool mxIsChar(const mxArray* a);
bool mxIsNumeric(const mxArray* a);
bool mxIsDouble(const mxArray* a);
bool mxIsComplex(const mxArray* a);
bool mxIsEmpty(const mxArray* a);
bool mxIsClass(const mxArray* a, const char* name);
size_t mxGetNumberOfElements(const mxArray* a);
size_t mxGetM(const mxArray* a);
double mxGetScalar(const mxArray* a);
mxDouble* mxGetDoubles(const mxArray* a);
mxComplexDouble* mxGetComplexDoubles(const mxArray* a);
int mxMakeArrayComplex(mxArray* a);
mxArray* mxDuplicateArray(const mxArray* a);
void mxDestroyArray(mxArray* a);
mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID c, mxComplexity x);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x);
mxArray* mxCreateDoubleScalar(double v);
mxArray* mxCreateCellMatrix(mwSize m, mwSize n);
char* mxArrayToString(const mxArray* a);
void* mxMalloc(size_t n);
void mxFree(void* p);
int mexCallMATLAB(int nlhs, mxArray* plhs[], int nrhs, mxArray* prhs[], const char* name);
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);
#endif
