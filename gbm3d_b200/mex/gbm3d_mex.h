/*
 * gbm3d_mex.h — shared helpers of the MEX gateways that shadow the reference's
 * hot-path .m files (source/matchBlocksCPU.m, denoiseAndAggregateGPU.m,
 * matchBlocksWie.m, denoiseAndAggregateWieFast.m, denoiseAndAggregateWie.m,
 * matchBlocksGPU.m) with libgbm3d calls.  Each gateway is one C file with a
 * mexFunction; build them with build_mex.m (MATLAB) or the commands in it
 * (Octave: mkoctfile --mex).
 *
 * Only the classic matrix API is used (mxGetData, mxGetField, mxGetCell,
 * mxCreate*), which MATLAB (with or without -R2018a) and Octave both provide.
 * Arrays are read in place: MATLAB's column-major layout is the library's.
 */
#ifndef GBM3D_MEX_H
#define GBM3D_MEX_H

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "gbm3d.h"
#include "mex.h"

/* One library context per MATLAB process (parfor workers are processes),
 * created on first use and destroyed when the MEX file is cleared. */
static gbm3d_ctx* gm_context_ = NULL;

static void gm_release(void) {
  if (gm_context_) gbm3d_ctx_destroy(gm_context_);
  gm_context_ = NULL;
}

static gbm3d_ctx* gm_ctx(void) {
  if (!gm_context_) {
    if (gbm3d_ctx_create(0, &gm_context_) != GBM3D_OK)
      mexErrMsgIdAndTxt("gbm3d:cuda", "libgbm3d: no usable CUDA device (there is no CPU fallback)");
    mexAtExit(gm_release);
  }
  return gm_context_;
}

static void gm_check(int rc, const char* fn) {
  if (rc != GBM3D_OK) {
    char id[96];
    snprintf(id, sizeof(id), "gbm3d:%s", fn);
    mexErrMsgIdAndTxt(id, "%s", gbm3d_last_error(gm_context_));
  }
}

/* ---- option struct (utilities/setBM3Dopts.m / checkBM3Dopts.m field names) ---- */

static const mxArray* gm_field(const mxArray* o, const char* name) {
  return (o && mxIsStruct(o)) ? mxGetField(o, 0, name) : NULL;
}

static int gm_int_field(const mxArray* o, const char* name, int dflt) {
  const mxArray* v = gm_field(o, name);
  if (!v || mxIsEmpty(v)) return dflt;
  if (!mxIsNumeric(v) && !mxIsLogical(v)) mexErrMsgIdAndTxt("gbm3d:opts", "opts.%s must be numeric", name);
  return (int)mxGetScalar(v);
}

static void gm_spins(const mxArray* o, const char* name, int* n, int* dst) {
  const mxArray* v = gm_field(o, name);
  if (!v) return;
  const size_t k = mxGetNumberOfElements(v);
  if (k > 8) mexErrMsgIdAndTxt("gbm3d:opts", "opts.%s: at most 8 match spins", name);
  if (!mxIsDouble(v) && k > 0) mexErrMsgIdAndTxt("gbm3d:opts", "opts.%s must be a double vector", name);
  const double* p = (const double*)mxGetData(v);
  for (size_t i = 0; i < k; ++i) dst[i] = (int)p[i];
  *n = (int)k;
}

/* The library's option struct from a MATLAB opts struct.  Fields absent from
 * opts keep checkBM3Dopts' defaults (GBM3D.m always passes a checked struct). */
static void gm_opts(const mxArray* o, gbm3d_opts* out) {
  if (o && !mxIsStruct(o)) mexErrMsgIdAndTxt("gbm3d:opts", "opts must be a struct");
  gbm3d_default_opts("default", out);
  out->numMax = gm_int_field(o, "numMax", out->numMax);
  out->numMin = gm_int_field(o, "numMin", out->numMin);
  out->blockSize = gm_int_field(o, "blockSize", out->blockSize);
  out->blockSizeWie = gm_int_field(o, "blockSizeWie", out->blockSizeWie);
  out->matchSize = gm_int_field(o, "matchSize", out->matchSize);
  out->refStride = gm_int_field(o, "refStride", 0);
  out->refStrideWie = gm_int_field(o, "refStrideWie", 0);
  out->levels = gm_int_field(o, "levels", out->levels);
  out->cycleSpin = gm_int_field(o, "cycleSpin", out->cycleSpin);
  out->tauMode = gm_int_field(o, "tauMode", out->tauMode);
  out->Wiener = gm_int_field(o, "Wiener", out->Wiener) != 0;
  out->staleWeights = gm_int_field(o, "staleWeights", out->staleWeights) != 0;
  gm_spins(o, "matchSpins", &out->nMatchSpins, out->matchSpins);
  gm_spins(o, "matchSpinsWie", &out->nMatchSpinsWie, out->matchSpinsWie);
  const mxArray* ft = gm_field(o, "filtType");
  if (ft) {
    char s[16] = {0};
    if (!mxIsChar(ft) || mxGetString(ft, s, sizeof(s)) != 0) mexErrMsgIdAndTxt("gbm3d:opts", "unrecognized filtering");
    if (strcmp(s, "ht") == 0) out->filtType = 0;
    else if (strcmp(s, "median") == 0) out->filtType = 1;
    else mexErrMsgIdAndTxt("gbm3d:opts", "unrecognized filtering");  /* denoiseAndAggregateGPU.m:54 */
  }
  const mxArray* wn = gm_field(o, "wname");
  if (wn && mxIsChar(wn)) {
    char s[16] = {0};
    mxGetString(wn, s, sizeof(s));
    out->wavelet = strcmp(s, "haar") == 0 ? 1 : 0;
  }
}

/* The video functions' options: VBM3D.m:8-19's defaults for absent fields
 * (blockSize 32, numMax = numMin = 16, levels 3, cycleSpin 2, tauMode 2) and
 * the one bank it supports, getWaveFilters3D('sym','db',4,1). */
static void gm_video_opts(const mxArray* o, gbm3d_opts* out) {
  if (o && !mxIsStruct(o)) mexErrMsgIdAndTxt("gbm3d:opts", "opts must be a struct");
  gbm3d_default_opts("default", out);
  out->blockSize = gm_int_field(o, "blockSize", 32);
  out->blockSizeWie = out->blockSize;
  out->matchSize = 2 * out->blockSize;
  out->numMax = gm_int_field(o, "numMax", 16);
  out->numMin = gm_int_field(o, "numMin", 16);
  out->levels = gm_int_field(o, "levels", 3);
  out->cycleSpin = gm_int_field(o, "cycleSpin", 2);
  out->tauMode = gm_int_field(o, "tauMode", 2);
  out->Wiener = 0;
  out->wavelet = 2;
  out->videoFrames = gm_int_field(o, "nF", 11);
  const char* want[2][2] = {{"wname", "sym"}, {"wnamez", "db"}};
  for (int k = 0; k < 2; ++k) {
    const mxArray* v = gm_field(o, want[k][0]);
    char s[16] = {0};
    if (v && (!mxIsChar(v) || mxGetString(v, s, sizeof(s)) != 0 || strcmp(s, want[k][1]) != 0))
      mexErrMsgIdAndTxt("gbm3d:opts", "opts.%s: the video path supports '%s' only", want[k][0], want[k][1]);
  }
  if (gm_int_field(o, "order", 4) != 4 || gm_int_field(o, "orderz", 1) != 1)
    mexErrMsgIdAndTxt("gbm3d:opts", "the video path supports opts.order = 4 and opts.orderz = 1 only");
}

/* ---- arguments ----------------------------------------------------------------- */

static const double* gm_real_double(const mxArray* a, const char* what) {
  if (!mxIsDouble(a) || mxIsComplex(a) || mxIsSparse(a))
    mexErrMsgIdAndTxt("gbm3d:args", "%s must be a real full double array", what);
  return (const double*)mxGetData(a);
}

static const float* gm_real_single(const mxArray* a, const char* what) {
  if (!mxIsSingle(a) || mxIsComplex(a)) mexErrMsgIdAndTxt("gbm3d:args", "%s must be a real single array", what);
  return (const float*)mxGetData(a);
}

static mwSize gm_dim(const mxArray* a, int k) {
  const mwSize nd = mxGetNumberOfDimensions(a);
  return k < (int)nd ? mxGetDimensions(a)[k] : 1;
}

/* sigma as matchBlocksCPU.m:21 uses it: a matrix (coloured noise) becomes mean(sqrt(sigma(:))). */
static double gm_sigma_scalar(const mxArray* s) {
  const double* p = gm_real_double(s, "sigma");
  const size_t n = mxGetNumberOfElements(s);
  if (n == 0) mexErrMsgIdAndTxt("gbm3d:args", "sigma is empty");
  if (mxGetM(s) <= 1) return p[0];
  double a = 0.0;
  for (size_t i = 0; i < n; ++i) a += sqrt(p[i]);
  return a / (double)n;
}

/* The cell array S (M x N cells of uint32 or double columns) flattened to the
 * library's K x M x N uint32 array; cnt[g] = numel(S{g}) (<= K). */
static void gm_S_from_cell(const mxArray* C, int K, uint32_t* S, int32_t* cnt) {
  if (!mxIsCell(C)) mexErrMsgIdAndTxt("gbm3d:args", "S must be a cell array");
  const size_t G = mxGetNumberOfElements(C);
  for (size_t g = 0; g < G; ++g) {
    const mxArray* e = mxGetCell(C, g);
    const size_t n = e ? mxGetNumberOfElements(e) : 0;
    if (n < 1 || n > (size_t)K) mexErrMsgIdAndTxt("gbm3d:args", "S{%d} must hold 1..numMax indices", (int)g + 1);
    memset(S + g * K, 0, (size_t)K * sizeof(uint32_t));
    if (mxIsUint32(e)) {
      memcpy(S + g * K, mxGetData(e), n * sizeof(uint32_t));
    } else if (mxIsDouble(e)) {
      const double* p = (const double*)mxGetData(e);
      for (size_t k = 0; k < n; ++k) S[g * K + k] = (uint32_t)p[k];
    } else {
      mexErrMsgIdAndTxt("gbm3d:args", "S{%d} must be uint32 or double", (int)g + 1);
    }
    cnt[g] = (int32_t)n;
  }
}

/* S as the reference returns it: cell(M, N), S{i,j} a uint32 column of cnt entries. */
static mxArray* gm_cell_from_S(const uint32_t* S, const int32_t* cnt, int K, int M, int N) {
  mxArray* C = mxCreateCellMatrix((mwSize)M, (mwSize)N);
  for (size_t g = 0; g < (size_t)M * N; ++g) {
    const int n = cnt ? cnt[g] : K;
    mxArray* col = mxCreateNumericMatrix((mwSize)n, 1, mxUINT32_CLASS, mxREAL);
    memcpy(mxGetData(col), S + g * K, (size_t)n * sizeof(uint32_t));
    mxSetCell(C, (mwIndex)g, col);
  }
  return C;
}

/* A gpuArray argument (Psi/Psi2 on a machine with a GPU, getWaveFilters3Dbior.m:33-36)
 * is gathered to host memory first. */
static const mxArray* gm_gathered(const mxArray* a, mxArray** owned) {
  *owned = NULL;
  if (mxIsNumeric(a)) return a;
  mxArray* in[1] = {(mxArray*)a};
  mxArray* out[1] = {NULL};
  if (mexCallMATLAB(1, out, 1, in, "gather") != 0 || !out[0]) mexErrMsgIdAndTxt("gbm3d:args", "cannot gather argument");
  *owned = out[0];
  return out[0];
}

static int gm_stride(int s, int d) { return s > 0 ? s : d; }

#endif /* GBM3D_MEX_H */
