/* S = matchBlocksGPU(I,sigma,opts) — shadows source/matchBlocksGPU.m:1-91.
 * Global circular search; S{i,j} holds 1-based linear indices into the m x n
 * image (no slot-1 override). */
#include "gbm3d_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 3 || nlhs > 1) mexErrMsgIdAndTxt("gbm3d:args", "usage: S = matchBlocksGPU(I,sigma,opts)");
  gbm3d_opts o;
  gm_opts(prhs[2], &o);
  const double* I = gm_real_double(prhs[0], "I");
  const int m = (int)mxGetM(prhs[0]), n = (int)mxGetN(prhs[0]);
  const int d = o.blockSize, K = o.numMax;
  if (m < d || n < d || K < 1) mexErrMsgIdAndTxt("gbm3d:args", "image smaller than blockSize");
  const int M = m / d, N = n / d;
  uint32_t* S = (uint32_t*)mxMalloc((size_t)K * M * N * sizeof(uint32_t));
  int32_t* cnt = (int32_t*)mxMalloc((size_t)M * N * sizeof(int32_t));
  gm_check(gbm3d_matchBlocksGPU(gm_ctx(), I, m, n, gm_sigma_scalar(prhs[1]), &o, S, cnt), "matchBlocksGPU");
  plhs[0] = gm_cell_from_S(S, cnt, K, M, N);
  mxFree(S);
  mxFree(cnt);
}
