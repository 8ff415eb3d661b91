/* [U,W] = denoiseAndAggregateWie(V1,V2,S,sigma,opts)
 * — shadows source/denoiseAndAggregateWie.m:1-90 (inverse DCT by the
 * transpose, output clamped to [0,1]). */
#include "gbm3d_wiener_gateway.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  gm_wiener(nlhs, plhs, nrhs, prhs, 1, "denoiseAndAggregateWie");
}
