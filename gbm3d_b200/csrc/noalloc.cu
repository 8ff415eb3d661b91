// Allocation-free block matching: gbm3d_matchBlocks_noalloc (include/gbm3d.h).
//
// Who needs this: callers that are not allowed to allocate device memory
// while they run.  A video or inference server that reserves all of its GPU
// memory at start-up, so that a call can never fail with out-of-memory or
// stall in the device-wide synchronisation a cudaFree implies, or a host
// application whose allocator owns every device buffer, cannot let a library
// call cudaMalloc behind its back.  The context-based entry points allocate
// their workspace on first use; this one never does.
//
// How: the only scratch the matcher needs, the padded search image of the
// reference (matchBlocksCPU.m:57-61), lives in the file-scope device array
// g_noalloc_pad below, which every GPU that loads the library holds until the
// process exits.  Its device address is looked up once per device with
// cudaGetSymbolAddress (host code may not use the array's name as a device
// pointer).  The inputs and outputs are the caller's device buffers.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/gbm3d.h"
#include "common.cuh"
#include "kernels.cuh"

namespace {

static __device__ __align__(256) float g_noalloc_pad[GBM3D_NOALLOC_MAX_FLOATS];

constexpr int kMaxDevices = 64;
float* g_pad_ptr[kMaxDevices] = {};
std::mutex g_pad_mu;

// Device address of g_noalloc_pad on the current device (set up on the first
// call per device, with that device current).
cudaError_t scratch_for_current_device(float** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pad_mu);
  if (!g_pad_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_pad);
    if (e != cudaSuccess) return e;
    g_pad_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_pad_ptr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int gbm3d_matchBlocks_noalloc(const float* I, int m, int n, double sigma, const gbm3d_opts* o,
                                         uint32_t* S, int32_t* S_count, void* stream) {
  if (!I || !S || !o) return GBM3D_ERR_ARG;
  const int d = o->blockSize, d2 = o->matchSize, K = o->numMax;
  if (o->numMin < 1 || o->numMin > K || K < 1 || K > 32 || (d2 & 1) || d2 * d2 < K) return GBM3D_ERR_ARG;
  if (!gbm3d::match_supported(d, d2)) return GBM3D_ERR_UNSUPPORTED;
  if (o->refStride != 0 && o->refStride != d) return GBM3D_ERR_UNSUPPORTED;  // the reference's tiling only
  if (m < d2 || n < d2 || m < d || n < d) return GBM3D_ERR_ARG;
  const int P = (m + d2 + 3) & ~3;
  if ((size_t)P * (size_t)(n + d2) > (size_t)GBM3D_NOALLOC_MAX_FLOATS) return GBM3D_ERR_TOO_LARGE;
  float* pad = nullptr;
  if (scratch_for_current_device(&pad) != cudaSuccess) return GBM3D_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // every element of the search image that the matcher reads is rewritten
  // here, so no part of the shared array has to be cleared between calls
  if (gbm3d::launch_make_pad(I, m, n, d2, 0, pad, P, st) != cudaSuccess) return GBM3D_ERR_CUDA;
  gbm3d::MatchArgs A{};
  A.pad = pad;
  A.P = P;
  A.M = m / d;
  A.N = n / d;
  A.K = K;
  A.s = d;
  A.numMin = o->numMin;
  A.tol = (float)(0.005 * sigma * sigma * d * d);
  A.tol_branch = o->numMin != K;
  A.S = S;
  A.cnt = S_count;
  A.m = m;
  A.n = n;
  A.R = m + d2;  // the search image's rows and columns (the matcher's TMA tensor map)
  A.Q = n + d2;
  if (gbm3d::launch_match(d, d2, A, st) != cudaSuccess) return GBM3D_ERR_CUDA;
  return GBM3D_OK;
}
