/*
 * Test infrastructure only: declarations of the MATLAB C API (R2018a
 * interleaved-complex interface) functions that faceted-hypersara_b200/mex/
 * fhs_mex.c calls, so that the gateway can be compiled for a syntax and type
 * check where MATLAB's own mex.h is absent.  Nothing is defined or linked.
 */
#ifndef FHS_TEST_MEX_STUB_H
#define FHS_TEST_MEX_STUB_H
#include <stdbool.h>
#include <stddef.h>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;
typedef enum {
  mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
  mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
  mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS
} mxClassID;
typedef struct { double real, imag; } mxComplexDouble;

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
mxClassID mxGetClassID(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
void* mxGetData(const mxArray* a);
double* mxGetDoubles(const mxArray* a);
mxComplexDouble* mxGetComplexDoubles(const mxArray* a);
double mxGetScalar(const mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize len);
bool mxIsDouble(const mxArray* a);
bool mxIsComplex(const mxArray* a);
bool mxIsStruct(const mxArray* a);
bool mxIsChar(const mxArray* a);
bool mxIsEmpty(const mxArray* a);
mxArray* mxGetField(const mxArray* a, size_t index, const char* name);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray* mxCreateDoubleScalar(double v);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID id, mxComplexity c);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID id, mxComplexity c);
mxArray* mxDuplicateArray(const mxArray* a);
void mxDestroyArray(mxArray* a);
#endif
