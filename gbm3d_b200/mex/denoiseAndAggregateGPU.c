/* [U,W] = denoiseAndAggregateGPU(Volume,S,tau,Psi,Psi2,opts)
 * — shadows source/denoiseAndAggregateGPU.m:1-92.  Psi/Psi2 (single, possibly
 * gpuArray) must be separable banks; they are factorised into 1D filters. */
#include "gbm3d_mex.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 6 || nlhs > 2)
    mexErrMsgIdAndTxt("gbm3d:args", "usage: [U,W] = denoiseAndAggregateGPU(Volume,S,tau,Psi,Psi2,opts)");
  gbm3d_opts o;
  gm_opts(prhs[5], &o);
  const float* V = gm_real_single(prhs[0], "Volume");
  const int d = o.blockSize, K = o.numMax, s = gm_stride(o.refStride, d);
  const int M = (int)mxGetM(prhs[1]), N = (int)mxGetN(prhs[1]);
  if (!mxIsCell(prhs[1]) || M < 1 || N < 1) mexErrMsgIdAndTxt("gbm3d:args", "S must be a non-empty cell array");
  if ((int)gm_dim(prhs[0], 0) < M * d || (int)gm_dim(prhs[0], 1) < N * d || (int)gm_dim(prhs[0], 2) != K)
    mexErrMsgIdAndTxt("gbm3d:args", "Volume must be at least (M*blockSize) x (N*blockSize) x numMax");
  const double* tau = gm_real_double(prhs[2], "tau");
  if ((int)mxGetM(prhs[2]) != o.levels || mxGetN(prhs[2]) != 7) mexErrMsgIdAndTxt("gbm3d:args", "tau must be levels x 7");
  mxArray *own1, *own2;
  const mxArray* P1 = gm_gathered(prhs[3], &own1);
  const mxArray* P2 = gm_gathered(prhs[4], &own2);
  const int L = (int)gm_dim(P1, 0), Lz = (int)gm_dim(P1, 2);
  if (gm_dim(P1, 1) != (mwSize)L || gm_dim(P1, 3) != 8 || mxGetNumberOfElements(P2) != mxGetNumberOfElements(P1))
    mexErrMsgIdAndTxt("gbm3d:args", "Psi/Psi2 must be L x L x Lz x 8");
  gbm3d_filters f;
  if (gbm3d_filters_from_bank(gm_real_single(P1, "Psi"), gm_real_single(P2, "Psi2"), L, Lz, &f) != GBM3D_OK)
    mexErrMsgIdAndTxt("gbm3d:args", "Psi/Psi2 are not separable 3D filter banks");
  if (own1) mxDestroyArray(own1);
  if (own2) mxDestroyArray(own2);
  /* a Volume exactly M*d x N*d x K is read in place; an image-shaped one with
   * trailing rows/cols (m not a multiple of d) is compacted first */
  const int vm = (int)gm_dim(prhs[0], 0), vn = (int)gm_dim(prhs[0], 1);
  const float* Vt = V;
  float* tmp = NULL;
  if (vm != M * d || vn != N * d) {
    tmp = (float*)mxMalloc((size_t)M * d * N * d * K * sizeof(float));
    for (int k = 0; k < K; ++k)
      for (int c = 0; c < N * d; ++c)
        memcpy(tmp + (size_t)M * d * (c + (size_t)N * d * k), V + (size_t)vm * (c + (size_t)vn * k),
               (size_t)M * d * sizeof(float));
    Vt = tmp;
  }
  uint32_t* S = (uint32_t*)mxMalloc((size_t)K * M * N * sizeof(uint32_t));
  int32_t* cnt = (int32_t*)mxMalloc((size_t)M * N * sizeof(int32_t));
  gm_S_from_cell(prhs[1], K, S, cnt);
  const int mo = (M - 1) * s + d, no = (N - 1) * s + d;
  plhs[0] = mxCreateDoubleMatrix((mwSize)mo, (mwSize)no, mxREAL);
  mxArray* W = mxCreateDoubleMatrix((mwSize)mo, (mwSize)no, mxREAL);
  gm_check(gbm3d_denoiseAndAggregateGPU(gm_ctx(), Vt, S, cnt, M, N, tau, &f, &o, (double*)mxGetData(plhs[0]),
                                        (double*)mxGetData(W)),
           "denoiseAndAggregateGPU");
  if (nlhs > 1) plhs[1] = W; else mxDestroyArray(W);
  if (tmp) mxFree(tmp);
  mxFree(S);
  mxFree(cnt);
}
