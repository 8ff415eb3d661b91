// Shared device helpers for the GBM3D sm_100a kernels.
//
// Numerical contract: the library is compiled with --fmad=false, so no a*b+c
// is fused unless a kernel writes fmaf() itself.  Together with IEEE division
// and square root (nvcc defaults) this makes every kernel's float result a
// fixed function of its inputs, reproduced bit for bit by the CPU oracle's
// FP32 mode.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define GBM3D_MAX_TAPS 16
#define GBM3D_MAX_LEVELS 6

namespace gbm3d {

__host__ __device__ __forceinline__ int pmod(int a, int L) {
  int r = a % L;
  return r < 0 ? r + L : r;
}

// Row (or column) of the image that row r of the reference's search image
// Ipad holds (source/matchBlocksCPU.m:57-61: 2x2 tiling cropped to L+d2,
// then circshift by h=d2/2).  Rows 0..h-1 hold image rows h..2h-1.
__host__ __device__ __forceinline__ int pad_index(int r, int L, int h) {
  return r < h ? r + h : (r - h) % L;
}

// 4-byte asynchronous global -> shared copy: no register round trip, so all of
// a tile's or a group's loads are in flight together.  The copying thread calls
// cp_async_wait_all() before the barrier (or __syncwarp) that publishes them.
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// One axis of a separable filter bank with its nonzero taps in ascending order.
struct Taps {
  int n;
  int k[GBM3D_MAX_TAPS];
  float h[GBM3D_MAX_TAPS];
};

// Analysis (lo, hi) and synthesis (lo, hi) taps of one axis.
struct AxisBank {
  Taps a[2];
  Taps s[2];
};

}  // namespace gbm3d
