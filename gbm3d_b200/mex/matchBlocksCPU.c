/* [S,Volume] = matchBlocksCPU(I,sigma,opts) — shadows source/matchBlocksCPU.m:1-116.
 * S: cell(M,N) of uint32 columns (numel(S{i,j}) < numMax only in the tolerance
 * branch, numMin < numMax); Volume: single m x n x numMax (tile-space
 * (M d) x (N d) x numMax when opts.refStride differs from blockSize). */
#include "gbm3d_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 3 || nlhs > 2) mexErrMsgIdAndTxt("gbm3d:args", "usage: [S,Volume] = matchBlocksCPU(I,sigma,opts)");
  gbm3d_opts o;
  gm_opts(prhs[2], &o);
  const double* I = gm_real_double(prhs[0], "I");
  if (mxGetNumberOfDimensions(prhs[0]) != 2) mexErrMsgIdAndTxt("gbm3d:args", "I must be a 2D image");
  const int m = (int)mxGetM(prhs[0]), n = (int)mxGetN(prhs[0]);
  const int d = o.blockSize, K = o.numMax, s = gm_stride(o.refStride, d);
  if (m < d || n < d || K < 1) mexErrMsgIdAndTxt("gbm3d:args", "image smaller than blockSize");
  const int M = (m - d) / s + 1, N = (n - d) / s + 1;
  uint32_t* S = (uint32_t*)mxMalloc((size_t)K * M * N * sizeof(uint32_t));
  int32_t* cnt = (int32_t*)mxMalloc((size_t)M * N * sizeof(int32_t));
  mxArray* V = NULL;
  if (nlhs > 1) {
    mwSize vd[3] = {(mwSize)(s == d ? m : M * d), (mwSize)(s == d ? n : N * d), (mwSize)K};
    V = mxCreateNumericArray(3, vd, mxSINGLE_CLASS, mxREAL);
  }
  gm_check(gbm3d_matchBlocksCPU(gm_ctx(), I, m, n, gm_sigma_scalar(prhs[1]), &o, S, cnt, V ? (float*)mxGetData(V) : NULL),
           "matchBlocksCPU");
  plhs[0] = gm_cell_from_S(S, cnt, K, M, N);
  if (V) plhs[1] = V;
  mxFree(S);
  mxFree(cnt);
}
