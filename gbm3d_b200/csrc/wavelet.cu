// Step 1: global 3D wavelet hard thresholding of the block-group volume.
//
// Restates denoiseAndAggregateGPU.m:27-47 with myWavDec3DFFT.m:10-23 and
// myWavRec3DGPUfast.m:10-40.  The reference filters the whole m x n x K volume
// with circular 3D convolutions through fftn; the filters are outer products
// of 1D factors, so each level here is three separable passes computed
// directly (no FFT), tile by tile in shared memory:
//
//   analysis  : z-pass (slot axis), x-pass, y-pass, each with decimation by 2,
//               c[q] = sum_k h[k] u[(2q - k) mod L]; hard threshold fused into
//               the y-pass store (strict |c| > tau, the approximation kept).
//   synthesis : y-pass, x-pass, z-pass, each upsampling by 2 and correlating,
//               r[p] = sum_band sum_k g[k] up[(p + k) mod L] (lo band first).
//
// Every sum is a serial fmaf chain over nonzero taps in ascending tap index,
// the order the CPU oracle follows.  The cycle spin of the reference
// (circshift of the volume by [s,s,s] before analysis and back after
// synthesis) is folded into the level-1 read and write indices, and the
// average over spins with the clamp max(.,0) is fused into the last level-1
// synthesis pass.
#include "common.cuh"
#include "kernels.cuh"

namespace gbm3d {

constexpr int TQ = 32;  // analysis output tile (coefficients per axis)
constexpr int TP = 32;  // synthesis output tile (samples per axis)

__global__ void __launch_bounds__(256) k_wav_analysis(const float* __restrict__ in, int Ly, int Lx,
                                                      int Lz, int shift, float* __restrict__ out,
                                                      WaveletBank bk, LevelBands th) {
  extern __shared__ float sm[];
  const int R = bk.reach_a;
  const int NY = 2 * TQ + R;
  float* tz = sm;                // [2][NY(x)][NY(y)]
  float* tx = sm + 2 * NY * NY;  // [4][TQ(qx)][NY(y)]
  const int Oy = Ly >> 1, Ox = Lx >> 1, Oz = Lz >> 1;
  const int qy0 = blockIdx.x * TQ, qx0 = blockIdx.y * TQ, qz = blockIdx.z;
  const int y0 = 2 * qy0 - R, x0 = 2 * qx0 - R;
  const size_t plane = (size_t)Ly * Lx;

  // load + z-pass (slot axis)
  for (int e = threadIdx.x; e < NY * NY; e += blockDim.x) {
    const int yy = e % NY, xx = e / NY;
    const int y = pmod(y0 + yy - shift, Ly), x = pmod(x0 + xx - shift, Lx);
    const float* col = in + y + (size_t)Ly * x;
#pragma unroll
    for (int fz = 0; fz < 2; ++fz) {
      const Taps& t = bk.z.a[fz];
      float acc = 0.f;
      for (int u = 0; u < t.n; ++u) {
        const int k = t.k[u];
        if (k >= Lz) continue;
        acc = fmaf(t.h[u], col[plane * pmod(2 * qz - k - shift, Lz)], acc);
      }
      tz[fz * NY * NY + e] = acc;
    }
  }
  __syncthreads();
  // x-pass
  for (int e = threadIdx.x; e < 4 * TQ * NY; e += blockDim.x) {
    const int yy = e % NY, qx = (e / NY) % TQ, comb = e / (NY * TQ);
    const int fx = comb & 1, fz = comb >> 1;
    const float* src = tz + fz * NY * NY + yy;
    const Taps& t = bk.xy.a[fx];
    float acc = 0.f;
    for (int u = 0; u < t.n; ++u) {
      const int k = t.k[u];
      if (k >= Lx) continue;
      acc = fmaf(t.h[u], src[(2 * qx + R - k) * NY], acc);
    }
    tx[(comb * TQ + qx) * NY + yy] = acc;
  }
  __syncthreads();
  // y-pass + hard threshold + store
  const size_t bsz = (size_t)Oy * Ox * Oz;
  for (int e = threadIdx.x; e < 8 * TQ * TQ; e += blockDim.x) {
    const int qy = e % TQ, qx = (e / TQ) % TQ, code = e / (TQ * TQ);
    if (qy0 + qy >= Oy || qx0 + qx >= Ox) continue;
    const int fy = code & 1, comb = code >> 1;
    const float* src = tx + (comb * TQ + qx) * NY;
    const Taps& t = bk.xy.a[fy];
    float acc = 0.f;
    for (int u = 0; u < t.n; ++u) {
      const int k = t.k[u];
      if (k >= Ly) continue;
      acc = fmaf(t.h[u], src[2 * qy + R - k], acc);
    }
    if (code) acc = acc * (fabsf(acc) > th.tau[code] ? 1.f : 0.f);
    out[code * bsz + (qy0 + qy) + (size_t)Oy * ((qx0 + qx) + (size_t)Ox * qz)] = acc;
  }
}

__global__ void __launch_bounds__(256) k_wav_synthesis(const float* __restrict__ bands,
                                                       const float* __restrict__ approx, int Oy,
                                                       int Ox, int Oz, SynthOut o, WaveletBank bk) {
  extern __shared__ float sm[];
  const int Iy = Oy >> 1, Ix = Ox >> 1, Iz = Oz >> 1;
  const int NQ = (TP - 1 + bk.reach_s) / 2 + 1;
  float* B = sm;                  // [8][NQ(qx)][NQ(qy)]
  float* Y = B + 8 * NQ * NQ;     // [4][NQ(qx)][TP(py)]
  float* X = Y + 4 * NQ * TP;     // [2][TP(px)][TP(py)]
  const int py0 = blockIdx.x * TP, px0 = blockIdx.y * TP, qz = blockIdx.z;
  const int qy0 = py0 >> 1, qx0 = px0 >> 1;
  const size_t bsz = (size_t)Iy * Ix * Iz;

  for (int e = threadIdx.x; e < 8 * NQ * NQ; e += blockDim.x) {
    const int qyl = e % NQ, qxl = (e / NQ) % NQ, code = e / (NQ * NQ);
    const int qy = (qy0 + qyl) % Iy, qx = (qx0 + qxl) % Ix;
    const float* src = code ? bands + code * bsz : approx;
    B[e] = src[qy + (size_t)Iy * (qx + (size_t)Ix * qz)];
  }
  __syncthreads();
  // y-pass: combine fy for each (fx, fz)
  for (int e = threadIdx.x; e < 4 * NQ * TP; e += blockDim.x) {
    const int py = e % TP, qxl = (e / TP) % NQ, comb = e / (TP * NQ);
    float acc = 0.f;
#pragma unroll
    for (int fy = 0; fy < 2; ++fy) {
      const float* src = B + (fy + 2 * comb) * NQ * NQ + qxl * NQ;
      const Taps& t = bk.xy.s[fy];
      for (int u = 0; u < t.n; ++u) {
        const int k = t.k[u];
        if (k >= Oy || ((py + k) & 1)) continue;
        acc = fmaf(t.h[u], src[(py + k) >> 1], acc);
      }
    }
    Y[(comb * NQ + qxl) * TP + py] = acc;
  }
  __syncthreads();
  // x-pass: combine fx for each fz
  for (int e = threadIdx.x; e < 2 * TP * TP; e += blockDim.x) {
    const int py = e % TP, px = (e / TP) % TP, fz = e / (TP * TP);
    float acc = 0.f;
#pragma unroll
    for (int fx = 0; fx < 2; ++fx) {
      const float* src = Y + (fx + 2 * fz) * NQ * TP + py;
      const Taps& t = bk.xy.s[fx];
      for (int u = 0; u < t.n; ++u) {
        const int k = t.k[u];
        if (k >= Ox || ((px + k) & 1)) continue;
        acc = fmaf(t.h[u], src[((px + k) >> 1) * TP], acc);
      }
    }
    X[(fz * TP + px) * TP + py] = acc;
  }
  __syncthreads();
  // z-pass: outputs pz = 2qz (tap 0) and pz = 2qz-1 (tap 1); write / accumulate
  for (int e = threadIdx.x; e < 2 * TP * TP; e += blockDim.x) {
    const int py = e % TP, px = (e / TP) % TP, which = e / (TP * TP);
    if (py0 + py >= Oy || px0 + px >= Ox) continue;
    const int pz = pmod(2 * qz - which, Oz);
    float acc = 0.f;
#pragma unroll
    for (int fz = 0; fz < 2; ++fz) {
      const Taps& t = bk.z.s[fz];
      for (int u = 0; u < t.n; ++u) {
        const int k = t.k[u];
        if (k >= Oz || k != which) continue;
        acc = fmaf(t.h[u], X[(fz * TP + px) * TP + py], acc);
      }
    }
    const int oy = pmod(py0 + py - o.shift, Oy), ox = pmod(px0 + px - o.shift, Ox), oz = pmod(pz - o.shift, Oz);
    float* dst = o.out + oy + (size_t)Oy * (ox + (size_t)Ox * oz);
    float v = o.first ? acc : *dst + acc;
    if (o.last) {
      v = v / o.cycles;
      v = v > 0.f ? v : 0.f;
    }
    *dst = v;
  }
}

// getBM3DAggWeights(3,1) (getBM3DAggWeights.m:11-19) and weight = 1/(D+eps)
// (denoiseAndAggregateGPU.m:191), one warp per group.  Each of the three sums
// is a fixed-order reduction: lane l adds the elements l, l+32, ... of the
// column-major difference array in order, then an xor butterfly.
__device__ __forceinline__ float d3(float u0, float u1, float u2, float u3) {
  const float a0 = u1 - u0, a1 = u2 - u1, a2 = u3 - u2;
  const float b0 = a1 - a0, b1 = a2 - a1;
  return b1 - b0;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__global__ void __launch_bounds__(128) k_ht_weights(const float* __restrict__ V, int m, int n, int M,
                                                    int N, int d, int K, const int32_t* __restrict__ cnt,
                                                    float* __restrict__ wgt) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = blockIdx.x * 4 + warp;
  if (g >= M * N) return;
  const int i = g % M, j = g / M;
  const int nm = cnt ? cnt[g] : K;
  const size_t sz = (size_t)m * n;
  const float* base = V + (size_t)i * d + (size_t)j * d * m;
  auto at = [&](int r, int c, int k) { return base[r + (size_t)c * m + sz * k]; };
  const int dm = d - 3;
  float tx = 0.f, ty = 0.f, tz = 0.f;
  const int nx = d * dm * nm;
  for (int e = lane; e < nx; e += 32) {
    const int r = e % d, c = (e / d) % dm, k = e / (d * dm);
    tx = tx + fabsf(d3(at(r, c, k), at(r, c + 1, k), at(r, c + 2, k), at(r, c + 3, k)));
  }
  for (int e = lane; e < nx; e += 32) {
    const int r = e % dm, c = (e / dm) % d, k = e / (dm * d);
    ty = ty + fabsf(d3(at(r, c, k), at(r + 1, c, k), at(r + 2, c, k), at(r + 3, c, k)));
  }
  const int nzz = d * d * (nm - 1);
  for (int e = lane; e < nzz; e += 32) {
    const int r = e % d, c = (e / d) % d, k = e / (d * d);
    tz = tz + fabsf(at(r, c, k + 1) - at(r, c, k));
  }
  tx = warp_sum(tx);
  ty = warp_sum(ty);
  tz = warp_sum(tz);
  if (lane == 0) {
    float w = tx * 0.25f + ty * 0.25f;
    w = w + tz;
    wgt[g] = 1.f / (w + 2.220446049250313e-16f);
  }
}

static size_t analysis_smem(int reach) {
  const int NY = 2 * TQ + reach;
  return (size_t)(2 * NY * NY + 4 * TQ * NY) * sizeof(float);
}

static size_t synthesis_smem(int reach) {
  const int NQ = (TP - 1 + reach) / 2 + 1;
  return (size_t)(8 * NQ * NQ + 4 * NQ * TP + 2 * TP * TP) * sizeof(float);
}

cudaError_t launch_wav_analysis(const float* in, int Ly, int Lx, int Lz, int shift, float* out,
                                const WaveletBank& bk, const LevelBands& th, cudaStream_t st) {
  const size_t sm = analysis_smem(bk.reach_a);
  cudaError_t e = cudaFuncSetAttribute(k_wav_analysis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  dim3 grid((Ly / 2 + TQ - 1) / TQ, (Lx / 2 + TQ - 1) / TQ, Lz / 2);
  k_wav_analysis<<<grid, 256, sm, st>>>(in, Ly, Lx, Lz, shift, out, bk, th);
  return cudaGetLastError();
}

cudaError_t launch_wav_synthesis(const float* bands, const float* approx, int Oy, int Ox, int Oz,
                                 const SynthOut& o, const WaveletBank& bk, cudaStream_t st) {
  const size_t sm = synthesis_smem(bk.reach_s);
  cudaError_t e = cudaFuncSetAttribute(k_wav_synthesis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  dim3 grid((Oy + TP - 1) / TP, (Ox + TP - 1) / TP, Oz / 2);
  k_wav_synthesis<<<grid, 256, sm, st>>>(bands, approx, Oy, Ox, Oz, o, bk);
  return cudaGetLastError();
}

cudaError_t launch_ht_weights(const float* Vavg, int m, int n, int M, int N, int d, int K,
                              const int32_t* cnt, float* wgt, cudaStream_t st) {
  const int G = M * N;
  k_ht_weights<<<(G + 3) / 4, 128, 0, st>>>(Vavg, m, n, M, N, d, K, cnt, wgt);
  return cudaGetLastError();
}

}  // namespace gbm3d
