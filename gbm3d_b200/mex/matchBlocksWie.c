/* [S,V1,V2] = matchBlocksWie(I,In,sigma,opts) — shadows source/matchBlocksWie.m:1-92.
 * V1 (pilot blocks) and V2 (noisy blocks): single d x d x K x M x N. */
#include "gbm3d_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 4 || nlhs > 3) mexErrMsgIdAndTxt("gbm3d:args", "usage: [S,V1,V2] = matchBlocksWie(I,In,sigma,opts)");
  gbm3d_opts o;
  gm_opts(prhs[3], &o);
  const double* I = gm_real_double(prhs[0], "I");
  const double* In = gm_real_double(prhs[1], "In");
  const int m = (int)mxGetM(prhs[0]), n = (int)mxGetN(prhs[0]);
  if ((int)mxGetM(prhs[1]) != m || (int)mxGetN(prhs[1]) != n) mexErrMsgIdAndTxt("gbm3d:args", "I and In differ in size");
  const int d = o.blockSizeWie, K = o.numMax, s = gm_stride(o.refStrideWie, d);
  if (m < d || n < d || K < 1) mexErrMsgIdAndTxt("gbm3d:args", "image smaller than blockSizeWie");
  const int M = (m - d) / s + 1, N = (n - d) / s + 1;
  mwSize vd[5] = {(mwSize)d, (mwSize)d, (mwSize)K, (mwSize)M, (mwSize)N};
  mxArray* V1 = nlhs > 1 ? mxCreateNumericArray(5, vd, mxSINGLE_CLASS, mxREAL) : NULL;
  mxArray* V2 = nlhs > 2 ? mxCreateNumericArray(5, vd, mxSINGLE_CLASS, mxREAL) : NULL;
  uint32_t* S = (uint32_t*)mxMalloc((size_t)K * M * N * sizeof(uint32_t));
  gm_check(gbm3d_matchBlocksWie(gm_ctx(), I, In, m, n, gm_sigma_scalar(prhs[2]), &o, S,
                                V1 ? (float*)mxGetData(V1) : NULL, V2 ? (float*)mxGetData(V2) : NULL),
           "matchBlocksWie");
  plhs[0] = gm_cell_from_S(S, NULL, K, M, N);
  if (V1) plhs[1] = V1;
  if (V2) plhs[2] = V2;
  mxFree(S);
}
