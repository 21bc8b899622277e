/* Minimal stand-in for MATLAB's mex.h (test infrastructure only): the types
 * and functions of the interleaved-complex MEX API that
 * elastodynamicebem_b200/mex/ebem_mex.c uses, implemented over plain host
 * arrays by mex_stub.c so that the gateway compiles and runs without MATLAB. */
#ifndef EBEM_TEST_MEX_STUB_H
#define EBEM_TEST_MEX_STUB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef struct mxArray_tag mxArray;
typedef enum { mxUNKNOWN_CLASS = 0, mxCHAR_CLASS = 4, mxDOUBLE_CLASS = 6 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

double* mxGetDoubles(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
double mxGetScalar(const mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize len);
int mxIsChar(const mxArray* a);
int mxIsDouble(const mxArray* a);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity c);
mxArray* mxCreateDoubleScalar(double v);
void mxDestroyArray(mxArray* a);
void* mxMalloc(size_t n);
void mxFree(void* p);
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

#ifdef __cplusplus
}
#endif

#endif
