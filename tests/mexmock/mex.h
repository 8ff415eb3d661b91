/*
 * mex.h — a minimal stand-in for MATLAB's MEX/matrix API, TEST INFRASTRUCTURE
 * ONLY.  MATLAB and Octave are not available where the tests run, so the MEX
 * gateways under gbm3d_b200/mex/ are compiled against this header and
 * mexmock.c, and driven from Python through the mm_* harness functions.  Only
 * the part of the API the gateways use is provided, with MATLAB's documented
 * semantics (column-major numeric arrays, cell and 1x1 struct arrays, char
 * strings, mexErrMsgIdAndTxt unwinding to the caller).
 */
#ifndef MEXMOCK_MEX_H
#define MEXMOCK_MEX_H
#include <stddef.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum {
  mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
  mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
  mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS, mxFUNCTION_CLASS
} mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;
typedef struct mxArray_tag mxArray;

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
int mexCallMATLAB(int nlhs, mxArray* plhs[], int nrhs, mxArray* prhs[], const char* name);

bool mxIsStruct(const mxArray* a);
bool mxIsCell(const mxArray* a);
bool mxIsChar(const mxArray* a);
bool mxIsNumeric(const mxArray* a);
bool mxIsLogical(const mxArray* a);
bool mxIsDouble(const mxArray* a);
bool mxIsSingle(const mxArray* a);
bool mxIsUint32(const mxArray* a);
bool mxIsComplex(const mxArray* a);
bool mxIsSparse(const mxArray* a);
bool mxIsEmpty(const mxArray* a);
mxClassID mxGetClassID(const mxArray* a);
mxArray* mxGetField(const mxArray* a, mwIndex i, const char* name);
mxArray* mxGetCell(const mxArray* a, mwIndex i);
void mxSetCell(mxArray* a, mwIndex i, mxArray* v);
double mxGetScalar(const mxArray* a);
void* mxGetData(const mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize len);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
mxArray* mxCreateCellMatrix(mwSize m, mwSize n);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x);
mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID c, mxComplexity x);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity x);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names);
void mxSetField(mxArray* a, mwIndex i, const char* name, mxArray* v);
void mxDestroyArray(mxArray* a);
void* mxMalloc(size_t n);
void mxFree(void* p);

#ifdef __cplusplus
}
#endif
#endif
