/* [U,out] = denoiseAndAggregateV(Y,Volume,I,S,sigma,opts)
 * — shadows source/denoiseAndAggregateV.m:1-89.  Y is unused (as in the
 * reference); I gives the frame size m x n and the frame count F.  Volume:
 * (M d) x (N d) x numMax (single or double; the library computes in single).
 * U and out.K: m x n x F double; out.Z: m x n, the group size of each block.
 * VBM3D pads its frames to multiples of blockSize; other frame sizes are
 * rejected. */
#include "gbm3d_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 6 || nlhs > 2)
    mexErrMsgIdAndTxt("gbm3d:args", "usage: [U,out] = denoiseAndAggregateV(Y,Volume,I,S,sigma,opts)");
  gbm3d_opts o;
  gm_video_opts(prhs[5], &o);
  const int d = o.blockSize, K = o.numMax;
  const int m = (int)gm_dim(prhs[2], 0), n = (int)gm_dim(prhs[2], 1), F = (int)gm_dim(prhs[2], 2);
  const int M = (int)mxGetM(prhs[3]), N = (int)mxGetN(prhs[3]);
  if (!mxIsCell(prhs[3]) || M < 1 || N < 1) mexErrMsgIdAndTxt("gbm3d:args", "S must be a non-empty cell array");
  if (m != M * d || n != N * d)
    mexErrMsgIdAndTxt("gbm3d:args", "frames must be (size(S,1)*blockSize) x (size(S,2)*blockSize)");
  const mxArray* Va = prhs[1];
  if ((int)gm_dim(Va, 0) != m || (int)gm_dim(Va, 1) != n || (int)gm_dim(Va, 2) != K)
    mexErrMsgIdAndTxt("gbm3d:args", "Volume must be m x n x numMax");
  const size_t nv = (size_t)m * n * K;
  float* tmp = NULL;
  const float* V;
  if (mxIsSingle(Va)) {
    V = gm_real_single(Va, "Volume");
  } else {
    const double* Vd = gm_real_double(Va, "Volume");
    tmp = (float*)mxMalloc(nv * sizeof(float));
    for (size_t i = 0; i < nv; ++i) tmp[i] = (float)Vd[i];
    V = tmp;
  }
  double sigma = mxGetScalar(prhs[4]);
  if (!mxIsDouble(prhs[4]) || mxGetNumberOfElements(prhs[4]) != 1)
    mexErrMsgIdAndTxt("gbm3d:args", "sigma must be a double scalar");
  double* tau = (double*)mxMalloc((size_t)o.levels * 7 * sizeof(double));
  gbm3d_get_tau(o.levels, o.tauMode, tau);  /* tau = sigma * getTau(levels, tauMode), denoiseAndAggregateV.m:17 */
  for (int i = 0; i < o.levels * 7; ++i) tau[i] *= sigma;
  uint32_t* S = (uint32_t*)mxMalloc((size_t)K * M * N * sizeof(uint32_t));
  int32_t* cnt = (int32_t*)mxMalloc((size_t)M * N * sizeof(int32_t));
  gm_S_from_cell(prhs[3], K, S, cnt);
  for (int g = 0; g < M * N; ++g)
    if (cnt[g] != K) mexErrMsgIdAndTxt("gbm3d:args", "every S{i,j} must hold numMax indices");
  mwSize ud[3] = {(mwSize)m, (mwSize)n, (mwSize)F};
  plhs[0] = mxCreateNumericArray(3, ud, mxDOUBLE_CLASS, mxREAL);
  mxArray* W = mxCreateNumericArray(3, ud, mxDOUBLE_CLASS, mxREAL);
  gm_check(gbm3d_denoiseAndAggregateV(gm_ctx(), V, S, M, N, F, tau, NULL, &o, (double*)mxGetData(plhs[0]),
                                      (double*)mxGetData(W)),
           "denoiseAndAggregateV");
  if (nlhs > 1) {
    const char* names[2] = {"K", "Z"};
    mxArray* out = mxCreateStructMatrix(1, 1, 2, names);
    mxArray* Z = mxCreateDoubleMatrix((mwSize)m, (mwSize)n, mxREAL);
    double* z = (double*)mxGetData(Z);
    for (size_t i = 0; i < (size_t)m * n; ++i) z[i] = K;
    mxSetField(out, 0, "K", W);
    mxSetField(out, 0, "Z", Z);
    plhs[1] = out;
  } else {
    mxDestroyArray(W);
  }
  if (tmp) mxFree(tmp);
  mxFree(tau);
  mxFree(S);
  mxFree(cnt);
}
