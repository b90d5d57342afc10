/*
 * mexstub.c -- the test harness's implementation of tests/mexstub/mex.h, and
 * a driver API (stub_*) through which pytest builds MATLAB values, calls the
 * gateway's mexFunction and reads the results back.
 *
 * Test infrastructure only: it lets the MEX gateway matlab/rgf_mex.c run
 * without MATLAB.  Built with the gateway into tests/mexstub/libmexstub.so by
 * rgf_b200/build.py.
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

#define STUB_API __attribute__((visibility("default")))

enum { K_DOUBLE, K_CHAR, K_CELL, K_STRUCT };

struct mxArray_tag {
  int kind;
  int cplx;
  mwSize ndim;
  mwSize dims[8];
  size_t numel;
  double* re;          /* real double data (mxREAL)                  */
  mxComplexDouble* cx; /* interleaved complex data (mxCOMPLEX)       */
  char* str;           /* char data, numel characters + NUL          */
  mxArray** cells;     /* cell elements (numel)                      */
  int nfields;         /* 1x1 struct: field names and values         */
  char** fnames;
  mxArray** fvals;
};

/* ---- error, warning and allocation bookkeeping of one mexFunction call ---- */
static jmp_buf g_jmp;
static int g_in_call = 0;
static char g_err_id[128], g_err_msg[1024];
static char g_warn[16][512];
static int g_nwarn = 0;
static void (*g_atexit)(void) = NULL;
static void** g_allocs = NULL;
static size_t g_nallocs = 0, g_capallocs = 0;

static void track(void* p) {
  if (g_nallocs == g_capallocs) {
    g_capallocs = g_capallocs ? 2 * g_capallocs : 64;
    g_allocs = (void**)realloc(g_allocs, sizeof(void*) * g_capallocs);
  }
  g_allocs[g_nallocs++] = p;
}

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  va_list ap;
  snprintf(g_err_id, sizeof(g_err_id), "%s", id ? id : "");
  va_start(ap, fmt);
  vsnprintf(g_err_msg, sizeof(g_err_msg), fmt, ap);
  va_end(ap);
  if (g_in_call) longjmp(g_jmp, 1);
  fprintf(stderr, "mexErrMsgIdAndTxt outside a call: %s: %s\n", g_err_id, g_err_msg);
  abort();
}

void mexWarnMsgIdAndTxt(const char* id, const char* fmt, ...) {
  if (g_nwarn >= 16) return;
  char msg[400];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof(msg), fmt, ap);
  va_end(ap);
  snprintf(g_warn[g_nwarn++], sizeof(g_warn[0]), "%s: %s", id ? id : "", msg);
}

int mexAtExit(void (*fn)(void)) {
  g_atexit = fn;
  return 0;
}

void* mxMalloc(size_t n) {
  void* p = malloc(n ? n : 1);
  track(p);
  return p;
}

void* mxCalloc(size_t n, size_t size) {
  void* p = calloc(n ? n : 1, size ? size : 1);
  track(p);
  return p;
}

/* ---- arrays --------------------------------------------------------------- */
static mxArray* new_array(int kind, mwSize nd, const mwSize* dims) {
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->kind = kind;
  a->ndim = nd < 2 ? 2 : nd;
  a->dims[0] = a->dims[1] = 1;
  a->numel = 1;
  for (mwSize i = 0; i < nd && i < 8; i++) a->dims[i] = dims[i];
  for (mwSize i = 0; i < a->ndim; i++) a->numel *= a->dims[i];
  return a;
}

int mxIsNumeric(const mxArray* a) { return a && a->kind == K_DOUBLE; }
int mxIsDouble(const mxArray* a) { return a && a->kind == K_DOUBLE; }
int mxIsComplex(const mxArray* a) { return a && a->kind == K_DOUBLE && a->cplx; }
int mxIsChar(const mxArray* a) { return a && a->kind == K_CHAR; }
int mxIsCell(const mxArray* a) { return a && a->kind == K_CELL; }
int mxIsStruct(const mxArray* a) { return a && a->kind == K_STRUCT; }
size_t mxGetNumberOfElements(const mxArray* a) { return a->numel; }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a->ndim; }
const mwSize* mxGetDimensions(const mxArray* a) { return a->dims; }
size_t mxGetM(const mxArray* a) { return a->dims[0]; }
size_t mxGetN(const mxArray* a) { return a->numel / (a->dims[0] ? a->dims[0] : 1); }
double* mxGetDoubles(const mxArray* a) { return (a->kind == K_DOUBLE && !a->cplx) ? a->re : NULL; }
mxComplexDouble* mxGetComplexDoubles(const mxArray* a) { return (a->kind == K_DOUBLE && a->cplx) ? a->cx : NULL; }

double mxGetScalar(const mxArray* a) {
  if (a->kind != K_DOUBLE || a->numel == 0) return 0.0;
  return a->cplx ? a->cx[0].real : a->re[0];
}

int mxMakeArrayComplex(mxArray* a) {
  if (a->kind != K_DOUBLE) return 0;
  if (a->cplx) return 1;
  a->cx = (mxComplexDouble*)calloc(a->numel ? a->numel : 1, sizeof(mxComplexDouble));
  for (size_t i = 0; i < a->numel; i++) a->cx[i].real = a->re[i];
  free(a->re);
  a->re = NULL;
  a->cplx = 1;
  return 1;
}

int mxGetString(const mxArray* a, char* buf, mwSize len) {
  if (!a || a->kind != K_CHAR || len == 0) return 1;
  const size_t n = a->numel;
  const size_t k = n < len - 1 ? n : len - 1;
  memcpy(buf, a->str, k);
  buf[k] = 0;
  return n > len - 1 ? 1 : 0;
}

mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name) {
  if (!s || s->kind != K_STRUCT || i != 0) return NULL;
  for (int f = 0; f < s->nfields; f++)
    if (!strcmp(s->fnames[f], name)) return s->fvals[f];
  return NULL;
}

void mxSetField(mxArray* s, mwIndex i, const char* name, mxArray* value) {
  if (!s || s->kind != K_STRUCT || i != 0) return;
  for (int f = 0; f < s->nfields; f++)
    if (!strcmp(s->fnames[f], name)) {
      if (s->fvals[f]) mxDestroyArray(s->fvals[f]);
      s->fvals[f] = value;
      return;
    }
}

mxArray* mxGetCell(const mxArray* c, mwIndex i) {
  if (!c || c->kind != K_CELL || i >= c->numel) return NULL;
  return c->cells[i];
}

mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID cls, mxComplexity c) {
  (void)cls;
  mxArray* a = new_array(K_DOUBLE, nd, dims);
  a->cplx = c == mxCOMPLEX;
  if (a->cplx) a->cx = (mxComplexDouble*)calloc(a->numel ? a->numel : 1, sizeof(mxComplexDouble));
  else a->re = (double*)calloc(a->numel ? a->numel : 1, sizeof(double));
  return a;
}

mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
  const mwSize d[2] = {m, n};
  return mxCreateNumericArray(2, d, mxDOUBLE_CLASS, c);
}

mxArray* mxCreateDoubleScalar(double v) {
  mxArray* a = mxCreateDoubleMatrix(1, 1, mxREAL);
  a->re[0] = v;
  return a;
}

mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names) {
  const mwSize d[2] = {m, n};
  mxArray* a = new_array(K_STRUCT, 2, d);
  a->nfields = nfields;
  a->fnames = (char**)calloc(nfields ? nfields : 1, sizeof(char*));
  a->fvals = (mxArray**)calloc(nfields ? nfields : 1, sizeof(mxArray*));
  for (int f = 0; f < nfields; f++) a->fnames[f] = strdup(names[f]);
  return a;
}

mxArray* mxDuplicateArray(const mxArray* a) {
  if (!a) return NULL;
  mxArray* b = new_array(a->kind, a->ndim, a->dims);
  b->cplx = a->cplx;
  const size_t n = a->numel ? a->numel : 1;
  if (a->re) {
    b->re = (double*)malloc(sizeof(double) * n);
    memcpy(b->re, a->re, sizeof(double) * n);
  }
  if (a->cx) {
    b->cx = (mxComplexDouble*)malloc(sizeof(mxComplexDouble) * n);
    memcpy(b->cx, a->cx, sizeof(mxComplexDouble) * n);
  }
  if (a->str) b->str = strdup(a->str);
  if (a->cells) {
    b->cells = (mxArray**)calloc(n, sizeof(mxArray*));
    for (size_t i = 0; i < a->numel; i++) b->cells[i] = mxDuplicateArray(a->cells[i]);
  }
  if (a->kind == K_STRUCT) {
    b->nfields = a->nfields;
    b->fnames = (char**)calloc(a->nfields ? a->nfields : 1, sizeof(char*));
    b->fvals = (mxArray**)calloc(a->nfields ? a->nfields : 1, sizeof(mxArray*));
    for (int f = 0; f < a->nfields; f++) {
      b->fnames[f] = strdup(a->fnames[f]);
      b->fvals[f] = mxDuplicateArray(a->fvals[f]);
    }
  }
  return b;
}

void mxDestroyArray(mxArray* a) {
  if (!a) return;
  free(a->re);
  free(a->cx);
  free(a->str);
  if (a->cells) {
    for (size_t i = 0; i < a->numel; i++) mxDestroyArray(a->cells[i]);
    free(a->cells);
  }
  for (int f = 0; f < a->nfields; f++) {
    free(a->fnames[f]);
    mxDestroyArray(a->fvals[f]);
  }
  free(a->fnames);
  free(a->fvals);
  free(a);
}

/* ---- driver API for the tests ---------------------------------------------- */
STUB_API mxArray* stub_double(mwSize nd, const mwSize* dims, const double* re, const double* im) {
  mxArray* a = mxCreateNumericArray(nd, dims, mxDOUBLE_CLASS, im ? mxCOMPLEX : mxREAL);
  for (size_t i = 0; i < a->numel; i++) {
    if (im) {
      a->cx[i].real = re[i];
      a->cx[i].imag = im[i];
    } else {
      a->re[i] = re[i];
    }
  }
  return a;
}

STUB_API mxArray* stub_char(const char* s) {
  const mwSize d[2] = {1, strlen(s)};
  mxArray* a = new_array(K_CHAR, 2, d);
  a->str = strdup(s);
  return a;
}

STUB_API mxArray* stub_cell(mwSize n, mxArray** elems) {
  const mwSize d[2] = {1, n};
  mxArray* a = new_array(K_CELL, 2, d);
  a->cells = (mxArray**)calloc(n ? n : 1, sizeof(mxArray*));
  for (mwSize i = 0; i < n; i++) a->cells[i] = elems[i];
  return a;
}

STUB_API mxArray* stub_struct(int nfields, const char** names, mxArray** vals) {
  mxArray* a = mxCreateStructMatrix(1, 1, nfields, names);
  for (int f = 0; f < nfields; f++) a->fvals[f] = vals[f];
  return a;
}

/* kind: 0 double, 1 char, 2 cell, 3 struct; returns ndim, fills dims (<= 8) */
STUB_API int stub_info(const mxArray* a, mwSize* dims, int* kind, int* cplx) {
  for (mwSize i = 0; i < a->ndim; i++) dims[i] = a->dims[i];
  *kind = a->kind;
  *cplx = a->cplx;
  return (int)a->ndim;
}

/* copies numel values out (im may be NULL; zeros for a real array) */
STUB_API void stub_read(const mxArray* a, double* re, double* im) {
  for (size_t i = 0; i < a->numel; i++) {
    re[i] = a->cplx ? a->cx[i].real : a->re[i];
    if (im) im[i] = a->cplx ? a->cx[i].imag : 0.0;
  }
}

STUB_API mxArray* stub_field(const mxArray* s, const char* name) { return mxGetField(s, 0, name); }
STUB_API void stub_destroy(mxArray* a) { mxDestroyArray(a); }
STUB_API const char* stub_err_id(void) { return g_err_id; }
STUB_API const char* stub_err_msg(void) { return g_err_msg; }
STUB_API int stub_nwarnings(void) { return g_nwarn; }
STUB_API const char* stub_warning(int i) { return (i >= 0 && i < g_nwarn) ? g_warn[i] : ""; }

/* runs mexFunction; returns 0, or 1 after mexErrMsgIdAndTxt (stub_err_id /
 * stub_err_msg).  mxMalloc'ed memory is freed afterwards, as MATLAB does. */
STUB_API int stub_call(int nlhs, mxArray** plhs, int nrhs, const mxArray** prhs) {
  int rc = 0;
  g_err_id[0] = g_err_msg[0] = 0;
  g_nwarn = 0;
  for (int i = 0; i < nlhs; i++) plhs[i] = NULL;
  g_in_call = 1;
  if (setjmp(g_jmp) == 0) {
    mexFunction(nlhs, plhs, nrhs, prhs);
  } else {
    rc = 1;
  }
  g_in_call = 0;
  for (size_t i = 0; i < g_nallocs; i++) free(g_allocs[i]);
  g_nallocs = 0;
  return rc;
}

/* MATLAB's clear mex: the gateway's exit handler */
STUB_API void stub_clear(void) {
  if (g_atexit) g_atexit();
  g_atexit = NULL;
}
