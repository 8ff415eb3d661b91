/* [U,W] = denoiseAndAggregateWieFast(V1,V2,S,sigma,opts)
 * — shadows source/denoiseAndAggregateWieFast.m:1-100. */
#include "gbm3d_wiener_gateway.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  gm_wiener(nlhs, plhs, nrhs, prhs, 0, "denoiseAndAggregateWieFast");
}
