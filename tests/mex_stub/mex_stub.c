/* Implementation of the mex.h stand-in (test infrastructure only).  Arrays
 * are column-major double (or char) buffers; mexErrMsgIdAndTxt unwinds to
 * stub_call with longjmp, as MATLAB unwinds a failing MEX call; arrays
 * created during a failing call are freed, as MATLAB frees them.  The
 * stub_* functions are what the Python tests call through ctypes. */
#include "mex.h"

#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

struct mxArray_tag {
    mxClassID cls;
    mwSize ndim;
    mwSize dims[4];
    double* data;
    char* str;
};

static jmp_buf g_jmp;
static char g_err_id[128], g_err_msg[2048];
static void (*g_exit_fn)(void) = NULL;
#define MAX_LIVE 4096
static mxArray* g_live[MAX_LIVE];     /* arrays created during the current call */
static int g_nlive = 0;
static int g_in_call = 0;

static void track(mxArray* a) {
    if (g_in_call && g_nlive < MAX_LIVE) g_live[g_nlive++] = a;
}

static void untrack(mxArray* a) {
    for (int i = 0; i < g_nlive; i++)
        if (g_live[i] == a) { g_live[i] = g_live[--g_nlive]; return; }
}

double* mxGetDoubles(const mxArray* a) { return a->data; }
size_t mxGetM(const mxArray* a) { return a->dims[0]; }
size_t mxGetN(const mxArray* a) {
    size_t n = 1;
    for (mwSize k = 1; k < a->ndim; k++) n *= a->dims[k];
    return n;
}
size_t mxGetNumberOfElements(const mxArray* a) { return mxGetM(a) * mxGetN(a); }
double mxGetScalar(const mxArray* a) { return a->data ? a->data[0] : 0.0; }
int mxIsChar(const mxArray* a) { return a->cls == mxCHAR_CLASS; }
int mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }

int mxGetString(const mxArray* a, char* buf, mwSize len) {
    if (a->cls != mxCHAR_CLASS || !a->str) return 1;
    size_t n = strlen(a->str);
    if (n + 1 > len) return 1;
    memcpy(buf, a->str, n + 1);
    return 0;
}

mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity c) {
    (void)c;
    mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
    size_t n = 1;
    a->cls = cls;
    a->ndim = ndim < 2 ? 2 : ndim;
    a->dims[0] = a->dims[1] = 1;
    for (mwSize k = 0; k < ndim && k < 4; k++) { a->dims[k] = dims[k]; n *= dims[k]; }
    a->data = (double*)calloc(n ? n : 1, sizeof(double));
    track(a);
    return a;
}

mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
    mwSize d[2] = {m, n};
    return mxCreateNumericArray(2, d, mxDOUBLE_CLASS, c);
}

mxArray* mxCreateDoubleScalar(double v) {
    mxArray* a = mxCreateDoubleMatrix(1, 1, mxREAL);
    a->data[0] = v;
    return a;
}

void mxDestroyArray(mxArray* a) {
    if (!a) return;
    untrack(a);
    free(a->data);
    free(a->str);
    free(a);
}

void* mxMalloc(size_t n) { return malloc(n ? n : 1); }
void mxFree(void* p) { free(p); }

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
    va_list ap;
    snprintf(g_err_id, sizeof g_err_id, "%s", id);
    va_start(ap, fmt);
    vsnprintf(g_err_msg, sizeof g_err_msg, fmt, ap);
    va_end(ap);
    longjmp(g_jmp, 1);
}

int mexAtExit(void (*fn)(void)) {
    g_exit_fn = fn;
    return 0;
}

/* ---- test-side API ---- */

mxArray* stub_double(mwSize m, mwSize n, mwSize p, const double* data) {
    mwSize d[3] = {m, n, p};
    int was = g_in_call;
    g_in_call = 0;
    mxArray* a = mxCreateNumericArray(p > 1 ? 3 : 2, d, mxDOUBLE_CLASS, mxREAL);
    g_in_call = was;
    if (data) memcpy(a->data, data, sizeof(double) * m * n * (p ? p : 1));
    return a;
}

mxArray* stub_string(const char* s) {
    mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
    a->cls = mxCHAR_CLASS;
    a->ndim = 2;
    a->dims[0] = 1;
    a->dims[1] = strlen(s);
    a->str = (char*)malloc(strlen(s) + 1);
    memcpy(a->str, s, strlen(s) + 1);
    return a;
}

size_t stub_numel(const mxArray* a) { return mxGetNumberOfElements(a); }
size_t stub_dim(const mxArray* a, int k) { return k < (int)a->ndim ? a->dims[k] : 1; }
const double* stub_data(const mxArray* a) { return a->data; }
void stub_free(mxArray* a) { mxDestroyArray(a); }
const char* stub_error_id(void) { return g_err_id; }
const char* stub_error_msg(void) { return g_err_msg; }
int stub_run_at_exit(void) {
    if (!g_exit_fn) return 0;
    g_exit_fn();
    return 1;
}

/* Calls mexFunction; 0 on success, 1 when it raised an error (message via
 * stub_error_msg).  Outputs of a failing call are released. */
int stub_call(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    g_err_id[0] = g_err_msg[0] = '\0';
    for (int k = 0; k < nlhs; k++) plhs[k] = NULL;
    g_nlive = 0;
    g_in_call = 1;
    if (setjmp(g_jmp)) {
        g_in_call = 0;
        while (g_nlive > 0) mxDestroyArray(g_live[g_nlive - 1]);
        for (int k = 0; k < nlhs; k++) plhs[k] = NULL;
        return 1;
    }
    mexFunction(nlhs, plhs, nrhs, prhs);
    g_in_call = 0;
    g_nlive = 0;           /* outputs now belong to the caller */
    return 0;
}
