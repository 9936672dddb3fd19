/*
 * Test infrastructure only: a minimal in-process stand-in for the MATLAB C
 * API calls that faceted-hypersara_b200/mex/fhs_mex.c makes, so that the
 * gateway's argument checks can run on a machine without MATLAB.
 * mexErrMsgIdAndTxt records the error identifier and longjmps back to the
 * caller of run_gateway().  Arrays are plain heap blocks; nothing is freed
 * (one short-lived test process).
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
  mxClassID cls;
  int cplx;
  mwSize ndim;
  mwSize dims[4];
  size_t numel;
  void* data;
  char* str;
  /* struct: one field per entry */
  int nfield;
  const char* fname[8];
  mxArray* fval[8];
};

static jmp_buf g_jmp;
static char g_err_id[64];
static char g_err_msg[256];

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err_msg, sizeof g_err_msg, fmt, ap);
  va_end(ap);
  snprintf(g_err_id, sizeof g_err_id, "%s", id);
  longjmp(g_jmp, 1);
}

static mxArray* make(mxClassID cls, int cplx, mwSize ndim, const mwSize* dims) {
  mxArray* a = calloc(1, sizeof *a);
  a->cls = cls;
  a->cplx = cplx;
  a->ndim = ndim < 2 ? 2 : ndim;
  a->numel = 1;
  for (mwSize k = 0; k < a->ndim; ++k) {
    a->dims[k] = k < ndim ? dims[k] : 1;
    a->numel *= a->dims[k];
  }
  size_t es = cls == mxDOUBLE_CLASS ? (cplx ? 16 : 8) : 8;
  a->data = calloc(a->numel ? a->numel : 1, es);
  return a;
}

mxClassID mxGetClassID(const mxArray* a) { return a->cls; }
size_t mxGetNumberOfElements(const mxArray* a) { return a->numel; }
size_t mxGetM(const mxArray* a) { return a->dims[0]; }
size_t mxGetN(const mxArray* a) { return a->numel / (a->dims[0] ? a->dims[0] : 1); }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a->ndim; }
const mwSize* mxGetDimensions(const mxArray* a) { return a->dims; }
void* mxGetData(const mxArray* a) { return a->data; }
double* mxGetDoubles(const mxArray* a) { return (double*)a->data; }
mxComplexDouble* mxGetComplexDoubles(const mxArray* a) { return (mxComplexDouble*)a->data; }
double mxGetScalar(const mxArray* a) {
  if (a->cls == mxDOUBLE_CLASS) return ((double*)a->data)[0];
  return (double)((unsigned long long*)a->data)[0];
}
int mxGetString(const mxArray* a, char* buf, mwSize len) {
  if (!a->str || strlen(a->str) + 1 > len) return 1;
  memcpy(buf, a->str, strlen(a->str) + 1);
  return 0;
}
bool mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
bool mxIsComplex(const mxArray* a) { return a->cplx != 0; }
bool mxIsStruct(const mxArray* a) { return a->cls == mxSTRUCT_CLASS; }
bool mxIsChar(const mxArray* a) { return a->cls == mxCHAR_CLASS; }
bool mxIsEmpty(const mxArray* a) { return a->numel == 0; }
mxArray* mxGetField(const mxArray* a, size_t index, const char* name) {
  (void)index;
  for (int k = 0; k < a->nfield; ++k)
    if (!strcmp(a->fname[k], name)) return a->fval[k];
  return NULL;
}
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
  const mwSize d[2] = {m, n};
  return make(mxDOUBLE_CLASS, c == mxCOMPLEX, 2, d);
}
mxArray* mxCreateDoubleScalar(double v) {
  mxArray* a = mxCreateDoubleMatrix(1, 1, mxREAL);
  ((double*)a->data)[0] = v;
  return a;
}
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID id, mxComplexity c) {
  const mwSize d[2] = {m, n};
  return make(id, c == mxCOMPLEX, 2, d);
}
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID id, mxComplexity c) {
  return make(id, c == mxCOMPLEX, ndim, dims);
}
mxArray* mxDuplicateArray(const mxArray* a) {
  mxArray* b = make(a->cls, a->cplx, a->ndim, a->dims);
  memcpy(b->data, a->data, a->numel * (a->cplx ? 16 : 8));
  return b;
}
void mxDestroyArray(mxArray* a) { (void)a; }

/* ------------------------------------------------------------ test side */
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

mxArray* fake_char(const char* s) {
  mxArray* a = make(mxCHAR_CLASS, 0, 0, NULL);
  a->str = malloc(strlen(s) + 1);
  memcpy(a->str, s, strlen(s) + 1);
  return a;
}
mxArray* fake_handle(unsigned long long h) {
  mxArray* a = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
  ((unsigned long long*)a->data)[0] = h;
  return a;
}
mxArray* fake_real(size_t n) { return mxCreateDoubleMatrix(n, 1, mxREAL); }
mxArray* fake_cplx(size_t n) { return mxCreateDoubleMatrix(n, 1, mxCOMPLEX); }
mxArray* fake_cube(mwSize a, mwSize b, mwSize c) {
  const mwSize d[3] = {a, b, c};
  return make(mxDOUBLE_CLASS, 0, 3, d);
}
mxArray* fake_struct(int n, const char** names, mxArray** vals) {
  mxArray* a = make(mxSTRUCT_CLASS, 0, 0, NULL);
  a->nfield = n;
  for (int k = 0; k < n; ++k) {
    a->fname[k] = names[k];
    a->fval[k] = vals[k];
  }
  return a;
}

/* Runs the gateway; returns "" on success or the error identifier. */
const char* run_gateway(int nlhs, int nrhs, const mxArray** prhs) {
  static mxArray* plhs[8];
  g_err_id[0] = 0;
  if (setjmp(g_jmp) == 0) mexFunction(nlhs, plhs, nrhs, prhs);
  return g_err_id;
}
const char* last_message(void) { return g_err_msg; }
