/* Shared body of the two Wiener gateways (denoiseAndAggregateWieFast and the
 * legacy denoiseAndAggregateWie): [U,W] = f(V1,V2,S,sigma,opts). */
#ifndef GBM3D_WIENER_GATEWAY_H
#define GBM3D_WIENER_GATEWAY_H
#include "gbm3d_mex.h"

static void gm_wiener(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[], int legacy, const char* fn) {
  if (nrhs != 5 || nlhs > 2) mexErrMsgIdAndTxt("gbm3d:args", "usage: [U,W] = %s(V1,V2,S,sigma,opts)", fn);
  gbm3d_opts o;
  gm_opts(prhs[4], &o);
  const float* V1 = gm_real_single(prhs[0], "V1");
  const float* V2 = gm_real_single(prhs[1], "V2");
  const int d = (int)gm_dim(prhs[0], 0), K = (int)gm_dim(prhs[0], 2);
  const int M = (int)gm_dim(prhs[0], 3), N = (int)gm_dim(prhs[0], 4);
  if ((int)gm_dim(prhs[0], 1) != d || mxGetNumberOfElements(prhs[1]) != mxGetNumberOfElements(prhs[0]))
    mexErrMsgIdAndTxt("gbm3d:args", "V1 and V2 must both be d x d x K x M x N");
  if (!mxIsCell(prhs[2]) || (int)mxGetM(prhs[2]) != M || (int)mxGetN(prhs[2]) != N)
    mexErrMsgIdAndTxt("gbm3d:args", "S must be an M x N cell array");
  o.blockSizeWie = d;
  o.numMax = K;
  if (o.numMin > K) o.numMin = K;
  uint32_t* S = (uint32_t*)mxMalloc((size_t)K * M * N * sizeof(uint32_t));
  int32_t* cnt = (int32_t*)mxMalloc((size_t)M * N * sizeof(int32_t));
  gm_S_from_cell(prhs[2], K, S, cnt);
  for (size_t g = 0; g < (size_t)M * N; ++g)
    if (cnt[g] != K) mexErrMsgIdAndTxt("gbm3d:args", "every S{i,j} must hold numMax indices");
  const double* sg = gm_real_double(prhs[3], "sigma");
  const size_t ns = mxGetNumberOfElements(prhs[3]);
  const int s = gm_stride(o.refStrideWie, d);
  const int mo = (M - 1) * s + d, no = (N - 1) * s + d;
  plhs[0] = mxCreateDoubleMatrix((mwSize)mo, (mwSize)no, mxREAL);
  mxArray* W = mxCreateDoubleMatrix((mwSize)mo, (mwSize)no, mxREAL);
  int rc;
  if (legacy) {
    if (ns != 1) mexErrMsgIdAndTxt("gbm3d:args", "sigma must be a scalar");
    rc = gbm3d_denoiseAndAggregateWie(gm_ctx(), V1, V2, S, M, N, sg[0], &o, (double*)mxGetData(plhs[0]),
                                      (double*)mxGetData(W));
  } else {
    /* sigmaWie: a scalar, or d x d broadcast over the slots (GBM3D.m:35) */
    if (ns != 1 && ((int)mxGetM(prhs[3]) != d || (int)mxGetN(prhs[3]) != d))
      mexErrMsgIdAndTxt("gbm3d:args", "sigma must be a scalar or a d x d matrix");
    rc = gbm3d_denoiseAndAggregateWieFast(gm_ctx(), V1, V2, S, M, N, sg, ns > 1, &o, (double*)mxGetData(plhs[0]),
                                          (double*)mxGetData(W));
  }
  mxFree(S);
  mxFree(cnt);
  gm_check(rc, fn);
  if (nlhs > 1) plhs[1] = W; else mxDestroyArray(W);
}
#endif
