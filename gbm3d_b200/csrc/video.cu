// Video: block matching across a window of frames and aggregation into the
// frames — matchBlocksV.m:21-116 (top-K branch) and the aggregation loop of
// denoiseAndAggregateV.m:59-89.  The 3D wavelet hard threshold between them
// is the step-1 one (wavelet.cu) with the video's filter bank.
#include "common.cuh"
#include "kernels.cuh"

namespace gbm3d {

namespace {

// One CTA per reference block of the centre frame (stride d).  For every
// frame f of the window, the 2d x 2d window of that frame's search image is
// staged in shared memory and the exact FP32 SSD of each of the d x d
// candidate offsets is computed in row-major order (t = ref - cand,
// acc = fmaf(t, t, acc)).  Keys (distance bits << 32 | index a + b d + f d^2)
// sit in shared memory; the K smallest are taken in K rounds of a block-wide
// minimum (the stable (value, index) order of mink).  S(1) is the reference.
template <int D>
__global__ void __launch_bounds__(128) k_match_video(VideoMatchArgs A) {
  constexpr int WD = 2 * D, H = D / 2, DD = D * D;
  extern __shared__ unsigned long long keys[];   // F * D^2
  float* win = reinterpret_cast<float*>(keys + A.F * DD);  // WD x WD, column-major
  float* xr = win + WD * WD;                               // reference block, row-major
  __shared__ unsigned long long red[4];
  __shared__ uint32_t sel[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = blockIdx.x, i = g % A.M, j = g / A.M;
  const int ref = (A.F - 1) / 2;
  const int nc = A.F * DD;
  {  // the reference block: offset (d/2, d/2) of the centre frame's window
    const float* pr = A.pads[ref];
    for (int e = tid; e < DD; e += 128) {
      const int r = e / D, c = e % D;
      xr[e] = pr[(size_t)(i * D + H + r) + (size_t)(j * D + H + c) * A.P];
    }
  }
  for (int f = 0; f < A.F; ++f) {
    const float* pad = A.pads[f];
    __syncthreads();
    for (int e = tid; e < WD * WD; e += 128) {
      const int r = e % WD, c = e / WD;
      win[e] = pad[(size_t)(i * D + r) + (size_t)(j * D + c) * A.P];
    }
    __syncthreads();
    if constexpr (D == 32) {
      // 1024 candidates, 8 per thread: lane a = candidate row, warp w the
      // columns b = 8w .. 8w+7.  Per pixel (r, c) the reference value is one
      // broadcast and the 8 candidates' window values slide along the row
      // a + r in registers (one new shared load per c), so the loop runs at
      // the FP32 issue rate instead of two shared loads per FMA.  Each
      // candidate still accumulates in the order (r, then c).
      constexpr int NB = 8;
      const int a = tid & 31, b0 = (tid >> 5) * NB;
      float acc[NB];
#pragma unroll
      for (int q = 0; q < NB; ++q) acc[q] = 0.f;
      for (int r = 0; r < D; ++r) {
        const float* wr = win + (a + r) + b0 * WD;  // row a + r of the window, from column b0
        const float4* x4p = reinterpret_cast<const float4*>(xr + r * D);
        float wv[NB];  // wv[j & 7] = window column b0 + j of this row
#pragma unroll
        for (int q = 0; q < NB - 1; ++q) wv[q] = wr[q * WD];
#pragma unroll
        for (int c4 = 0; c4 < D / 4; ++c4) {
          const float4 x4 = x4p[c4];
          const float xs[4] = {x4.x, x4.y, x4.z, x4.w};
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int c = c4 * 4 + u;
            wv[(c + NB - 1) & (NB - 1)] = wr[(c + NB - 1) * WD];
#pragma unroll
            for (int q = 0; q < NB; ++q) {
              const float t = xs[u] - wv[(c + q) & (NB - 1)];
              acc[q] = fmaf(t, t, acc[q]);
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const uint32_t idx = (uint32_t)(a + (b0 + q) * D + f * DD);
        keys[idx] = ((unsigned long long)__float_as_uint(acc[q]) << 32) | idx;
      }
    } else {
      for (int cand = tid; cand < DD; cand += 128) {
        const int a = cand % D, b = cand / D;
        float acc = 0.f;
        for (int r = 0; r < D; ++r)
#pragma unroll 8
          for (int c = 0; c < D; ++c) {
            const float t = xr[r * D + c] - win[(a + r) + (b + c) * WD];
            acc = fmaf(t, t, acc);
          }
        const uint32_t idx = (uint32_t)(a + b * D + f * DD);
        keys[idx] = ((unsigned long long)__float_as_uint(acc) << 32) | idx;
      }
    }
  }
  __syncthreads();
  // K rounds of a block-wide minimum over the keys
  for (int k = 0; k < A.K; ++k) {
    unsigned long long best = ~0ull;
    for (int e = tid; e < nc; e += 128) best = min(best, keys[e]);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) red[warp] = best;
    __syncthreads();
    if (tid == 0) {
      const unsigned long long b = min(min(red[0], red[1]), min(red[2], red[3]));
      sel[k] = (uint32_t)(b & 0xffffffffu);
      keys[sel[k]] = ~0ull;
    }
    __syncthreads();
  }
  if (tid == 0) sel[0] = (uint32_t)(DD * A.F / 2 + H);  // S(1) = d^2 F/2 + d/2 + 1 (matchBlocksV.m:103), 0-based
  __syncthreads();
  for (int k = tid; k < A.K; k += 128) A.S[(size_t)g * A.K + k] = sel[k] + 1;
  // Volume(i d + r, j d + c, k): the selected block, image-shaped m x n x K
  const size_t mn = (size_t)A.m * A.n;
  for (int e = tid; e < A.K * DD; e += 128) {
    const int k = e / DD, r = e % D, c = (e / D) % D;
    const uint32_t s = sel[k];
    const int a = (int)(s % D), b = (int)((s / D) % D), f = (int)(s / DD);
    A.volume[(size_t)(i * D + r) + (size_t)A.m * (j * D + c) + mn * k] =
        A.pads[f][(size_t)(i * D + a + r) + (size_t)(j * D + b + c) * A.P];
  }
}

// Owner-computes aggregation into the F frames: thread = output pixel (r, c)
// of frame fr; contributions (reference y, x, slot k) in the reference's loop
// order, block k of (y, x) starting at (a + y d - d/2, b + x d - d/2) of frame
// f (skipped when the start is negative); each term fl(w * block) is added in
// double (the reference's U and out.K are double arrays).  DT is the patch
// size at compile time (the index decoding becomes shifts), 0 = A.d.
template <int DT>
__global__ void k_aggregate_video(VideoAggArgs A) {
  const size_t total = (size_t)A.m * A.n * A.F;
  const int d = DT ? DT : A.d, h = d / 2, K = A.K;
  const size_t mn = (size_t)A.m * A.n;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(p % A.m), c = (int)((p / A.m) % A.n), fr = (int)(p / mn);
    // references whose blocks can cover row r: y d - h <= r <= y d - h + 2d - 2, i.e.
    // ceil((r + h - 2d + 2) / d) <= y <= floor((r + h) / d) (the numerators are >= -2d;
    // adding 4d keeps the integer division a floor)
    const int ylo = max(0, (r + h - d + 1 + 4 * d) / d - 4), yhi = min(A.M - 1, (r + h) / d);
    const int xlo = max(0, (c + h - d + 1 + 4 * d) / d - 4), xhi = min(A.N - 1, (c + h) / d);
    double u = 0.0, w = 0.0;
    for (int y = ylo; y <= yhi; ++y)
      for (int x = xlo; x <= xhi; ++x) {
        const int g = y + A.M * x;
        const float wg = A.wgt[g];
        for (int k = 0; k < K; ++k) {
          const int e = (int)A.S[(size_t)g * K + k] - 1;
          const int a = e % d, b = (e / d) % d, f = e / (d * d);
          if (f != fr) continue;
          const int R0 = a + y * d - h, C0 = b + x * d - h;
          if (R0 < 0 || C0 < 0) continue;
          const int rr = r - R0, cc = c - C0;
          if ((unsigned)rr >= (unsigned)d || (unsigned)cc >= (unsigned)d) continue;
          const float blk = A.vsum[(size_t)(y * d + rr) + (size_t)A.m * (x * d + cc) + mn * k];
          u += (double)(wg * blk);
          w += (double)wg;
        }
      }
    A.U[p] = u;
    A.W[p] = w;
  }
}

__global__ void k_clamp01(float* __restrict__ v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    v[i] = fminf(v[i], 1.f);
}

}  // namespace

bool video_match_supported(int d, int F, int K) {
  return (d == 8 || d == 16 || d == 32) && F >= 1 && (F & 1) && F <= 31 && K >= 1 && K <= 32 && F * d * d >= K &&
         (size_t)F * d * d * 8 + (size_t)(4 * d * d + d * d) * 4 <= 200 * 1024;
}

cudaError_t launch_match_video(int d, const VideoMatchArgs& A, cudaStream_t st) {
  if (!video_match_supported(d, A.F, A.K)) return cudaErrorInvalidValue;
  const size_t sm = (size_t)A.F * d * d * 8 + (size_t)(4 * d * d + d * d) * 4;
  const int G = A.M * A.N;
#define GBM3D_VM_CASE(DD)                                                                                   \
  if (d == DD) {                                                                                            \
    cudaError_t e = cudaFuncSetAttribute(k_match_video<DD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
    if (e != cudaSuccess) return e;                                                                         \
    k_match_video<DD><<<G, 128, sm, st>>>(A);                                                               \
    return cudaGetLastError();                                                                              \
  }
  GBM3D_VM_CASE(8) GBM3D_VM_CASE(16) GBM3D_VM_CASE(32)
#undef GBM3D_VM_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_aggregate_video(const VideoAggArgs& A, cudaStream_t st) {
  switch (A.d) {
    case 8: k_aggregate_video<8><<<1184, 256, 0, st>>>(A); break;
    case 16: k_aggregate_video<16><<<1184, 256, 0, st>>>(A); break;
    case 32: k_aggregate_video<32><<<1184, 256, 0, st>>>(A); break;
    default: k_aggregate_video<0><<<1184, 256, 0, st>>>(A); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_clamp01(float* v, size_t n, cudaStream_t st) {
  k_clamp01<<<1184, 256, 0, st>>>(v, n);
  return cudaGetLastError();
}

}  // namespace gbm3d
