/*
 * mex.h -- a stand-in for MATLAB's MEX API, owned by the test harness.
 *
 * MATLAB and Octave are not installed where these tests run, so the MEX
 * gateway (matlab/rgf_mex.c) is compiled against this header and
 * tests/mexstub/mexstub.c, which implement the subset of the R2018a
 * interleaved-complex API the gateway uses over plain C structs.  Semantics
 * follow MATLAB's documentation: column-major data, complex arrays stored as
 * interleaved {real, imag} pairs, mexErrMsgIdAndTxt does not return.
 */
#ifndef RGF_TEST_MEX_H
#define RGF_TEST_MEX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef struct mxArray_tag mxArray;
typedef struct {
  double real, imag;
} mxComplexDouble;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef enum { mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxCHAR_CLASS, mxDOUBLE_CLASS = 6 } mxClassID;

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) __attribute__((noreturn));
void mexWarnMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));

void* mxMalloc(size_t n);
void* mxCalloc(size_t n, size_t size);

int mxIsNumeric(const mxArray* a);
int mxIsDouble(const mxArray* a);
int mxIsComplex(const mxArray* a);
int mxIsChar(const mxArray* a);
int mxIsCell(const mxArray* a);
int mxIsStruct(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
double mxGetScalar(const mxArray* a);
double* mxGetDoubles(const mxArray* a);
mxComplexDouble* mxGetComplexDoubles(const mxArray* a);
int mxMakeArrayComplex(mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize len);
mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name);
void mxSetField(mxArray* s, mwIndex i, const char* name, mxArray* value);
mxArray* mxGetCell(const mxArray* c, mwIndex i);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray* mxCreateDoubleScalar(double v);
mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID cls, mxComplexity c);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names);
mxArray* mxDuplicateArray(const mxArray* a);
void mxDestroyArray(mxArray* a);

#ifdef __cplusplus
}
#endif
#endif
