/*
 * mexmock.c — implementation of tests/mexmock/mex.h plus the mm_* harness
 * that Python uses to build arguments, call a gateway's mexFunction and read
 * its outputs.  TEST INFRASTRUCTURE ONLY (see mex.h).
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

enum { MM_GPUARRAY = 100 };  /* an opaque object that only gather() unwraps */

struct mxArray_tag {
  int cls;
  mwSize nd;
  mwSize dims[8];
  void* data;          /* numeric / char payload */
  mxArray** cells;     /* cell elements, or struct field values */
  char** fnames;       /* struct field names */
  int nfields;
  mxArray* wrapped;    /* MM_GPUARRAY payload */
};

static jmp_buf* mm_env = NULL;
static char mm_id[128], mm_msg[1024];
static void (*mm_atexit[16])(void);
static int mm_natexit = 0;

static size_t esize(int cls) {
  switch (cls) {
    case mxDOUBLE_CLASS: case mxINT64_CLASS: case mxUINT64_CLASS: return 8;
    case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
    case mxINT16_CLASS: case mxUINT16_CLASS: case mxCHAR_CLASS: return 2;
    case mxINT8_CLASS: case mxUINT8_CLASS: case mxLOGICAL_CLASS: return 1;
    default: return 0;
  }
}

static size_t numel(const mxArray* a) {
  size_t n = 1;
  for (mwSize i = 0; i < a->nd; ++i) n *= a->dims[i];
  return n;
}

static mxArray* make(int cls, mwSize nd, const mwSize* dims) {
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = cls;
  a->nd = nd < 2 ? 2 : nd;
  a->dims[0] = a->dims[1] = 1;
  for (mwSize i = 0; i < nd && i < 8; ++i) a->dims[i] = dims[i];
  while (a->nd > 2 && a->dims[a->nd - 1] == 1) --a->nd;  /* MATLAB drops trailing singletons */
  const size_t n = numel(a);
  if (cls == mxCELL_CLASS) a->cells = (mxArray**)calloc(n ? n : 1, sizeof(mxArray*));
  else if (esize(cls)) a->data = calloc(n ? n : 1, esize(cls));
  return a;
}

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  snprintf(mm_id, sizeof(mm_id), "%s", id);
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(mm_msg, sizeof(mm_msg), fmt, ap);
  va_end(ap);
  if (mm_env) longjmp(*mm_env, 1);
  fprintf(stderr, "mexErrMsgIdAndTxt outside a call: %s %s\n", mm_id, mm_msg);
  abort();
}

int mexAtExit(void (*fn)(void)) {
  for (int i = 0; i < mm_natexit; ++i)
    if (mm_atexit[i] == fn) return 0;
  if (mm_natexit < 16) mm_atexit[mm_natexit++] = fn;
  return 0;
}

static mxArray* copy_of(const mxArray* a);

int mexCallMATLAB(int nlhs, mxArray* plhs[], int nrhs, mxArray* prhs[], const char* name) {
  if (strcmp(name, "gather") == 0 && nlhs == 1 && nrhs == 1) {
    plhs[0] = copy_of(prhs[0]->cls == MM_GPUARRAY ? prhs[0]->wrapped : prhs[0]);
    return 0;
  }
  return 1;
}

bool mxIsStruct(const mxArray* a) { return a && a->cls == mxSTRUCT_CLASS; }
bool mxIsCell(const mxArray* a) { return a && a->cls == mxCELL_CLASS; }
bool mxIsChar(const mxArray* a) { return a && a->cls == mxCHAR_CLASS; }
bool mxIsLogical(const mxArray* a) { return a && a->cls == mxLOGICAL_CLASS; }
bool mxIsNumeric(const mxArray* a) { return a && a->cls >= mxDOUBLE_CLASS && a->cls <= mxUINT64_CLASS; }
bool mxIsDouble(const mxArray* a) { return a && a->cls == mxDOUBLE_CLASS; }
bool mxIsSingle(const mxArray* a) { return a && a->cls == mxSINGLE_CLASS; }
bool mxIsUint32(const mxArray* a) { return a && a->cls == mxUINT32_CLASS; }
bool mxIsComplex(const mxArray* a) { (void)a; return false; }
bool mxIsSparse(const mxArray* a) { (void)a; return false; }
bool mxIsEmpty(const mxArray* a) { return numel(a) == 0; }
mxClassID mxGetClassID(const mxArray* a) { return a->cls == MM_GPUARRAY ? mxUNKNOWN_CLASS : (mxClassID)a->cls; }

mxArray* mxGetField(const mxArray* a, mwIndex i, const char* name) {
  if (!mxIsStruct(a) || i != 0) return NULL;
  for (int f = 0; f < a->nfields; ++f)
    if (strcmp(a->fnames[f], name) == 0) return a->cells[f];
  return NULL;
}

mxArray* mxGetCell(const mxArray* a, mwIndex i) { return mxIsCell(a) && i < numel(a) ? a->cells[i] : NULL; }
void mxSetCell(mxArray* a, mwIndex i, mxArray* v) {
  if (mxIsCell(a) && i < numel(a)) a->cells[i] = v;
}

double mxGetScalar(const mxArray* a) {
  if (!a->data || numel(a) == 0) return 0.0;
  switch (a->cls) {
    case mxDOUBLE_CLASS: return ((double*)a->data)[0];
    case mxSINGLE_CLASS: return ((float*)a->data)[0];
    case mxINT32_CLASS: return ((int32_t*)a->data)[0];
    case mxUINT32_CLASS: return ((uint32_t*)a->data)[0];
    case mxLOGICAL_CLASS: case mxUINT8_CLASS: return ((uint8_t*)a->data)[0];
    case mxINT64_CLASS: return (double)((int64_t*)a->data)[0];
    default: return 0.0;
  }
}

void* mxGetData(const mxArray* a) { return a->data; }

int mxGetString(const mxArray* a, char* buf, mwSize len) {
  if (!mxIsChar(a) || len == 0) return 1;
  const size_t n = numel(a);
  const uint16_t* s = (const uint16_t*)a->data;
  size_t i = 0;
  for (; i < n && i + 1 < len; ++i) buf[i] = (char)s[i];
  buf[i] = 0;
  return i < n ? 1 : 0;
}

size_t mxGetM(const mxArray* a) { return a->dims[0]; }
size_t mxGetN(const mxArray* a) {
  size_t n = 1;
  for (mwSize i = 1; i < a->nd; ++i) n *= a->dims[i];
  return n;
}
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a->nd; }
const mwSize* mxGetDimensions(const mxArray* a) { return a->dims; }
size_t mxGetNumberOfElements(const mxArray* a) { return numel(a); }

mxArray* mxCreateCellMatrix(mwSize m, mwSize n) {
  mwSize d[2] = {m, n};
  return make(mxCELL_CLASS, 2, d);
}
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x) {
  (void)x;
  mwSize d[2] = {m, n};
  return make(c, 2, d);
}
mxArray* mxCreateNumericArray(mwSize nd, const mwSize* dims, mxClassID c, mxComplexity x) {
  (void)x;
  return make(c, nd, dims);
}
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity x) { return mxCreateNumericMatrix(m, n, mxDOUBLE_CLASS, x); }

/* 1 x 1 structs only (all the gateways create) */
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names) {
  mwSize d[2] = {m, n};
  mxArray* a = make(mxSTRUCT_CLASS, 2, d);
  a->cells = (mxArray**)calloc(64, sizeof(mxArray*));
  a->fnames = (char**)calloc(64, sizeof(char*));
  for (int f = 0; f < nfields && f < 64; ++f) a->fnames[f] = strdup(names[f]);
  a->nfields = nfields;
  return a;
}
void mxSetField(mxArray* a, mwIndex i, const char* name, mxArray* v) {
  if (!mxIsStruct(a) || i != 0) return;
  for (int f = 0; f < a->nfields; ++f)
    if (strcmp(a->fnames[f], name) == 0) {
      mxDestroyArray(a->cells[f]);
      a->cells[f] = v;
      return;
    }
}

void mxDestroyArray(mxArray* a) {
  if (!a) return;
  if (a->cls == mxCELL_CLASS || a->cls == mxSTRUCT_CLASS) {
    const size_t n = a->cls == mxCELL_CLASS ? numel(a) : (size_t)a->nfields;
    for (size_t i = 0; i < n; ++i) mxDestroyArray(a->cells[i]);
    free(a->cells);
  }
  for (int f = 0; f < a->nfields; ++f) free(a->fnames[f]);
  free(a->fnames);
  if (a->wrapped) mxDestroyArray(a->wrapped);
  free(a->data);
  free(a);
}

void* mxMalloc(size_t n) { return malloc(n ? n : 1); }
void mxFree(void* p) { free(p); }

static mxArray* copy_of(const mxArray* a) {
  mxArray* b = make(a->cls, a->nd, a->dims);
  if (a->data) memcpy(b->data, a->data, numel(a) * esize(a->cls));
  return b;
}

/* ---- harness ------------------------------------------------------------------ */

mxArray* mm_numeric(int cls, int nd, const size_t* dims, const void* data) {
  mxArray* a = make(cls, (mwSize)nd, dims);
  if (data && esize(cls)) memcpy(a->data, data, numel(a) * esize(cls));
  return a;
}
mxArray* mm_cell(size_t m, size_t n) { return mxCreateCellMatrix(m, n); }
void mm_set_cell(mxArray* c, size_t i, mxArray* v) { mxSetCell(c, i, v); }
mxArray* mm_struct(void) {
  mwSize d[2] = {1, 1};
  mxArray* a = make(mxSTRUCT_CLASS, 2, d);
  a->cells = (mxArray**)calloc(64, sizeof(mxArray*));
  a->fnames = (char**)calloc(64, sizeof(char*));
  return a;
}
int mm_set_field(mxArray* s, const char* name, mxArray* v) {
  if (!mxIsStruct(s) || s->nfields >= 64) return 1;
  s->fnames[s->nfields] = strdup(name);
  s->cells[s->nfields++] = v;
  return 0;
}
mxArray* mm_string(const char* str) {
  const size_t n = strlen(str);
  mwSize d[2] = {1, n};
  mxArray* a = make(mxCHAR_CLASS, 2, d);
  for (size_t i = 0; i < n; ++i) ((uint16_t*)a->data)[i] = (uint16_t)(unsigned char)str[i];
  return a;
}
mxArray* mm_gpuarray(mxArray* inner) {
  mwSize d[2] = {1, 1};
  mxArray* a = make(mxUNKNOWN_CLASS, 2, d);
  a->cls = MM_GPUARRAY;
  a->wrapped = inner;
  return a;
}

typedef void (*mexfn)(int, mxArray**, int, const mxArray**);

int mm_call(mexfn fn, int nlhs, mxArray** plhs, int nrhs, const mxArray** prhs) {
  jmp_buf env;
  mm_id[0] = mm_msg[0] = 0;
  for (int i = 0; i < nlhs; ++i) plhs[i] = NULL;
  mm_env = &env;
  if (setjmp(env)) {
    mm_env = NULL;
    return 1;
  }
  fn(nlhs, plhs, nrhs, prhs);
  mm_env = NULL;
  return 0;
}
const char* mm_err_id(void) { return mm_id; }
const char* mm_err_msg(void) { return mm_msg; }
void mm_run_atexit(void) {
  for (int i = mm_natexit - 1; i >= 0; --i) mm_atexit[i]();
  mm_natexit = 0;
}
int mm_class(const mxArray* a) { return a->cls; }
int mm_ndim(const mxArray* a) { return (int)a->nd; }
size_t mm_dim(const mxArray* a, int k) { return k < (int)a->nd ? a->dims[k] : 1; }
size_t mm_numel(const mxArray* a) { return numel(a); }
void* mm_data(const mxArray* a) { return a->data; }
mxArray* mm_get_cell(const mxArray* a, size_t i) { return mxGetCell(a, i); }
int mm_nfields(const mxArray* a) { return mxIsStruct(a) ? a->nfields : 0; }
const char* mm_field_name(const mxArray* a, int f) { return a->fnames[f]; }
mxArray* mm_field_value(const mxArray* a, int f) { return a->cells[f]; }
void mm_destroy(mxArray* a) { mxDestroyArray(a); }
