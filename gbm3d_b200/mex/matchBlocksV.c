/* [S,Volume] = matchBlocksV(I,sigma,opts) — shadows source/matchBlocksV.m:1-116
 * (top-K branch, numMin = numMax).  I: m x n x F double frames, F odd (the
 * centre frame holds the references).  S: cell(M,N) of numMax x 1 uint32
 * indices into the d x d x F candidate window (S{i,j}(1) is the reference);
 * Volume: single m x n x numMax. */
#include "gbm3d_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 3 || nlhs > 2) mexErrMsgIdAndTxt("gbm3d:args", "usage: [S,Volume] = matchBlocksV(I,sigma,opts)");
  gbm3d_opts o;
  gm_video_opts(prhs[2], &o);
  const double* I = gm_real_double(prhs[0], "I");
  if (mxGetNumberOfDimensions(prhs[0]) > 3) mexErrMsgIdAndTxt("gbm3d:args", "I must be m x n x frames");
  const int m = (int)gm_dim(prhs[0], 0), n = (int)gm_dim(prhs[0], 1), F = (int)gm_dim(prhs[0], 2);
  if (F % 2 != 1) mexErrMsgIdAndTxt("gbm3d:args", "input volume should have odd number of frames");  /* matchBlocksV.m:24 */
  (void)gm_real_double(prhs[1], "sigma");  /* used by the tolerance branch only */
  const int d = o.blockSize, K = o.numMax;
  if (d < 1 || m < d || n < d) mexErrMsgIdAndTxt("gbm3d:args", "frames smaller than blockSize");
  const int M = m / d, N = n / d;
  uint32_t* S = (uint32_t*)mxMalloc((size_t)K * M * N * sizeof(uint32_t));
  mwSize vd[3] = {(mwSize)m, (mwSize)n, (mwSize)K};
  mxArray* V = mxCreateNumericArray(3, vd, mxSINGLE_CLASS, mxREAL);
  gm_check(gbm3d_matchBlocksV(gm_ctx(), I, m, n, F, &o, S, (float*)mxGetData(V)), "matchBlocksV");
  plhs[0] = gm_cell_from_S(S, NULL, K, M, N);
  if (nlhs > 1) plhs[1] = V; else mxDestroyArray(V);
  mxFree(S);
}
