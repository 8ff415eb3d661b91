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
                                                      WaveletBank bk, LevelBands th, int tx0) {
  extern __shared__ float sm[];
  const int R = bk.reach_a;
  const int NY = 2 * TQ + R;
  float* tz = sm;                // [2][NY(x)][NY(y)]
  float* tx = sm + 2 * NY * NY;  // [4][TQ(qx)][NY(y)]
  const int Oy = Ly >> 1, Ox = Lx >> 1, Oz = Lz >> 1;
  const int ntx = (Ox + TQ - 1) / TQ, bx = blockIdx.y + tx0;  // column tile: the window's, modulo the count
  const int qy0 = blockIdx.x * TQ, qx0 = (bx >= ntx ? bx - ntx : bx) * TQ, qz = blockIdx.z;
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
                                                       int Ox, int Oz, SynthOut o, WaveletBank bk, int tx0) {
  extern __shared__ float sm[];
  const int Iy = Oy >> 1, Ix = Ox >> 1, Iz = Oz >> 1;
  const int NQ = (TP - 1 + bk.reach_s) / 2 + 1;
  float* B = sm;                  // [8][NQ(qx)][NQ(qy)]
  float* Y = B + 8 * NQ * NQ;     // [4][NQ(qx)][TP(py)]
  float* X = Y + 4 * NQ * TP;     // [2][TP(px)][TP(py)]
  const int ntx = (Ox + TP - 1) / TP, bx = blockIdx.y + tx0;
  const int py0 = blockIdx.x * TP, px0 = (bx >= ntx ? bx - ntx : bx) * TP, qz = blockIdx.z;
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

// ---------------------------------------------------------------------------
// Dense banks: every spatial filter has the taps 0..R and the slot filters
// the taps 0, 1 (sym4 x Haar, getWaveFilters3D('sym','db',4,1), VBM3D's bank:
// R = 7).  These are the generic kernels' three passes with the tile shapes
// and tap loops fixed at compile time, single wraps in place of the modulo
// (the launcher checks the sizes that make one wrap enough), and in the
// synthesis y-pass the two output parities of a coefficient pair computed by
// one thread (the generic pass predicates off half the taps in alternate
// lanes).  Every output is the same serial fmaf chain, over the same taps in
// the same order, as in the generic kernels.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int wrap_once(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

// T: coefficients per axis of a CTA's output tile (16: a 22 KB staging area,
// eight CTAs per SM, where the 32 of the generic kernel allows two).
template <int R, int T>
__global__ void __launch_bounds__(256) k_wav_analysis_dense(const float* __restrict__ in, int Ly, int Lx, int Lz,
                                                            int shift, float* __restrict__ out, WaveletBank bk,
                                                            LevelBands th, int tx0) {
  constexpr int TQ = T;
  constexpr int NY = 2 * TQ + R;
  extern __shared__ float sm[];
  float* tz = sm;                // [2][NY(x)][NY(y)]
  float* tx = sm + 2 * NY * NY;  // [4][TQ(qx)][NY(y)]
  const int Oy = Ly >> 1, Ox = Lx >> 1, Oz = Lz >> 1;
  const int ntx = (Ox + TQ - 1) / TQ, bx = blockIdx.y + tx0;
  const int qy0 = blockIdx.x * TQ, qx0 = (bx >= ntx ? bx - ntx : bx) * TQ, qz = blockIdx.z;
  const int y0 = 2 * qy0 - R - shift, x0 = 2 * qx0 - R - shift;
  const size_t plane = (size_t)Ly * Lx;
  // the slot taps k = 0, 1 read slots (2 qz - k - shift) mod Lz
  const size_t zo0 = plane * (size_t)wrap_once(2 * qz - shift, Lz);
  const size_t zo1 = plane * (size_t)wrap_once(2 * qz - 1 - shift, Lz);
  float hz[2][2];
#pragma unroll
  for (int f = 0; f < 2; ++f) {
    hz[f][0] = bk.z.a[f].h[0];
    hz[f][1] = bk.z.a[f].h[1];
  }
  // load + z-pass (slot axis)
  for (int e = threadIdx.x; e < NY * NY; e += 256) {
    const int yy = e % NY, xx = e / NY;
    const int y = wrap_once(y0 + yy, Ly), x = wrap_once(x0 + xx, Lx);
    const float* col = in + y + (size_t)Ly * x;
    const float v0 = col[zo0], v1 = col[zo1];
#pragma unroll
    for (int fz = 0; fz < 2; ++fz) tz[fz * NY * NY + e] = fmaf(hz[fz][1], v1, fmaf(hz[fz][0], v0, 0.f));
  }
  __syncthreads();
  // x-pass: the four (fx, fz) combinations as an unrolled outer loop, so
  // each one's taps are compile-time indices into the bank
#pragma unroll
  for (int comb = 0; comb < 4; ++comb) {
    const Taps& t = bk.xy.a[comb & 1];
    const float* tzc = tz + (comb >> 1) * NY * NY + R * NY;
    for (int e = threadIdx.x; e < TQ * NY; e += 256) {
      const int yy = e % NY, qx = e / NY;
      const float* src = tzc + yy + 2 * qx * NY;
      float acc = 0.f;
#pragma unroll
      for (int u = 0; u <= R; ++u) acc = fmaf(t.h[u], src[-u * NY], acc);
      tx[(comb * TQ + qx) * NY + yy] = acc;
    }
  }
  __syncthreads();
  // y-pass + hard threshold + store: a thread's coefficient (qy, qx) in all
  // eight bands
  const size_t bsz = (size_t)Oy * Ox * Oz;
  for (int e = threadIdx.x; e < TQ * TQ; e += 256) {
    const int qy = e % TQ, qx = e / TQ;
    if (qy0 + qy >= Oy || qx0 + qx >= Ox) continue;
    const float* src0 = tx + qx * NY + 2 * qy + R;
    float* dst = out + (qy0 + qy) + (size_t)Oy * ((qx0 + qx) + (size_t)Ox * qz);
#pragma unroll
    for (int code = 0; code < 8; ++code) {
      const Taps& t = bk.xy.a[code & 1];
      const float* src = src0 + (code >> 1) * TQ * NY;
      float acc = 0.f;
#pragma unroll
      for (int u = 0; u <= R; ++u) acc = fmaf(t.h[u], src[-u], acc);
      if (code) acc = acc * (fabsf(acc) > th.tau[code] ? 1.f : 0.f);
      dst[code * bsz] = acc;
    }
  }
}

template <int R>
__global__ void __launch_bounds__(256) k_wav_synthesis_dense(const float* __restrict__ bands,
                                                             const float* __restrict__ approx, int Oy, int Ox,
                                                             int Oz, SynthOut o, WaveletBank bk, int tx0) {
  constexpr int NQ = (TP - 1 + R) / 2 + 1;
  extern __shared__ float sm[];
  float* B = sm;               // [8][NQ(qx)][NQ(qy)]
  float* Y = B + 8 * NQ * NQ;  // [4][NQ(qx)][TP(py)]
  float* X = Y + 4 * NQ * TP;  // [2][TP(px)][TP(py)]
  const int Iy = Oy >> 1, Ix = Ox >> 1, Iz = Oz >> 1;
  const int ntx = (Ox + TP - 1) / TP, bx = blockIdx.y + tx0;
  const int py0 = blockIdx.x * TP, px0 = (bx >= ntx ? bx - ntx : bx) * TP, qz = blockIdx.z;
  const int qy0 = py0 >> 1, qx0 = px0 >> 1;
  const size_t bsz = (size_t)Iy * Ix * Iz;

  for (int e = threadIdx.x; e < 8 * NQ * NQ; e += 256) {
    const int qyl = e % NQ, qxl = (e / NQ) % NQ, code = e / (NQ * NQ);
    const int qy = wrap_once(qy0 + qyl, Iy), qx = wrap_once(qx0 + qxl, Ix);
    const float* src = code ? bands + code * bsz : approx;
    B[e] = src[qy + (size_t)Iy * (qx + (size_t)Ix * qz)];
  }
  __syncthreads();
  // y-pass: outputs py = 2j (even taps) and 2j + 1 (odd taps) of one thread,
  // each summing fy = 0 then 1, taps in ascending order
  for (int e = threadIdx.x; e < 4 * NQ * (TP / 2); e += 256) {
    const int j = e % (TP / 2), qxl = (e / (TP / 2)) % NQ, comb = e / ((TP / 2) * NQ);
    float ae = 0.f, ao = 0.f;
#pragma unroll
    for (int fy = 0; fy < 2; ++fy) {
      const float* src = B + (fy + 2 * comb) * NQ * NQ + qxl * NQ + j;
#pragma unroll
      for (int u = 0; u <= R; ++u) {
        const float h = fy ? bk.xy.s[1].h[u] : bk.xy.s[0].h[u];
        if (u & 1) ao = fmaf(h, src[(u + 1) >> 1], ao);  // (2j + 1 + u) / 2
        else ae = fmaf(h, src[u >> 1], ae);              // (2j + u) / 2
      }
    }
    *reinterpret_cast<float2*>(Y + (comb * NQ + qxl) * TP + 2 * j) = make_float2(ae, ao);
  }
  __syncthreads();
  // x-pass: combine fx for each fz (px is uniform across a warp)
  for (int e = threadIdx.x; e < 2 * TP * TP; e += 256) {
    const int py = e % TP, px = (e / TP) % TP, fz = e / (TP * TP);
    float acc = 0.f;
#pragma unroll
    for (int fx = 0; fx < 2; ++fx) {
      const float* src = Y + (fx + 2 * fz) * NQ * TP + py;
#pragma unroll
      for (int u = 0; u <= R; ++u) {
        if ((px + u) & 1) continue;
        acc = fmaf(fx ? bk.xy.s[1].h[u] : bk.xy.s[0].h[u], src[((px + u) >> 1) * TP], acc);
      }
    }
    X[(fz * TP + px) * TP + py] = acc;
  }
  __syncthreads();
  // z-pass: output pz = 2qz takes the slot tap 0 of both bands, pz = 2qz - 1 tap 1
  for (int e = threadIdx.x; e < 2 * TP * TP; e += 256) {
    const int py = e % TP, px = (e / TP) % TP, which = e / (TP * TP);
    if (py0 + py >= Oy || px0 + px >= Ox) continue;
    const int pz = wrap_once(2 * qz - which, Oz);
    float acc = 0.f;
#pragma unroll
    for (int fz = 0; fz < 2; ++fz)
      acc = fmaf(which ? bk.z.s[fz].h[1] : bk.z.s[fz].h[0], X[(fz * TP + px) * TP + py], acc);
    const int oy = wrap_once(py0 + py - o.shift, Oy), ox = wrap_once(px0 + px - o.shift, Ox),
              oz = wrap_once(pz - o.shift, Oz);
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
// (denoiseAndAggregateGPU.m:75), one warp per group.  Each of the three sums
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
                                                    float* __restrict__ wgt, int g0, int gn) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = window_group(blockIdx.x * 4 + warp, g0, gn, M * N);
  if (g < 0) return;
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

// ---------------------------------------------------------------------------
// Fast path for the two banks GBM3D uses: bior1.5 x Haar (the reference's
// getWaveFilters3Dbior) and 3D Haar.  Both have the shape
//   analysis  lo: taps 0..LA-1      hi: taps HA0, HA0+1
//   synthesis lo: taps SL0, SL0+1   hi: taps 0..SH-1
//   slot axis: taps 0, 1 for all four filters
// (bior: LA=SH=10, HA0=SL0=4; Haar: LA=SH=2, HA0=SL0=0).  With the tap
// positions known at compile time every loop unrolls, even and odd outputs
// are produced together (no divergent parity tests), shared memory rows that
// a stride-2 filter reads are stored de-interleaved, and no division is left
// in the inner loops.  Each output is the same serial fmaf chain, in the same
// tap order, as the generic kernels and the oracle.
// ---------------------------------------------------------------------------
struct FastBank {
  float alo[16], ahi[2], slo[2], shi[16];
  float azl[2], azh[2], szl[2], szh[2];
};

__device__ __forceinline__ int wrap1(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

constexpr int FQY = 32, FQX = 16;  // fast analysis tile: coefficients along y (fast axis) and x

// WIN: the column-tile window of the strip form (tx0); without it the grid
// covers every tile in order.
template <int LA, int HA0, bool WIN>
__global__ void __launch_bounds__(256) k_wav_analysis_fast(const float* __restrict__ in, int Ly, int Lx, int Lz,
                                                           int shift, float* __restrict__ out, FastBank fb,
                                                           LevelBands th, int tx0) {
  constexpr int HALO = LA - 1;
  constexpr int NY = 2 * FQY + HALO;  // staged rows
  constexpr int NX = 2 * FQX + HALO;  // staged columns
  constexpr int NYH = (NY + 1) / 2;   // de-interleaved half rows
  constexpr int NYHP = ((NYH + 15) / 32) * 32 + 16;  // = 16 mod 32: even and odd rows in different banks
  constexpr int RT = (NY + 31) / 32;  // row chunks per lane
  extern __shared__ float sm[];
  float* tz = sm;                     // [2 fz][NX x][NY y]
  float* tx = sm + 2 * NX * NY;       // [4 comb][FQX qx][2 parity][NYHP]
  const int Oy = Ly >> 1, Ox = Lx >> 1, Oz = Lz >> 1;
  const int ntx = (Ox + FQX - 1) / FQX, bx = WIN ? blockIdx.y + tx0 : blockIdx.y;
  const int qy0 = blockIdx.x * FQY, qx0 = (WIN && bx >= ntx ? bx - ntx : bx) * FQX, qz = blockIdx.z;
  const int y0 = 2 * qy0 - HALO - shift, x0 = 2 * qx0 - HALO - shift;
  const size_t zA = (size_t)Ly * Lx * pmod(2 * qz - shift, Lz), zB = (size_t)Ly * Lx * pmod(2 * qz - 1 - shift, Lz);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

  // stage 1: load the input tile of two slots and apply the slot-axis pass
  // (warps over columns, lanes over rows)
  int gy[RT];
#pragma unroll
  for (int t = 0; t < RT; ++t) gy[t] = wrap1(y0 + lane + 32 * t, Ly);
#pragma unroll 3
  for (int xx = w; xx < NX; xx += 8) {
    const float* col = in + (size_t)Ly * wrap1(x0 + xx, Lx);
#pragma unroll
    for (int t = 0; t < RT; ++t) {
      const int yy = lane + 32 * t;
      if (yy < NY) {
        const float u0 = __ldg(col + gy[t] + zA), u1 = __ldg(col + gy[t] + zB);  // taps k=0, k=1
        tz[xx * NY + yy] = fmaf(fb.azl[1], u1, fmaf(fb.azl[0], u0, 0.f));
        tz[NX * NY + xx * NY + yy] = fmaf(fb.azh[1], u1, fmaf(fb.azh[0], u0, 0.f));
      }
    }
  }
  __syncthreads();
  // stage 2: pass along the slow axis, lo and hi together from the same inputs.
  // Item = (fz, run of RX coefficients qx, row yy), lanes over rows; the run's
  // inputs (staged columns 2 q0 .. 2 (q0 + RX - 1) + HALO) are read once into
  // registers.
  constexpr int RX = 8, NRX = FQX / RX, NV = 2 * RX + LA - 2;
  for (int it = threadIdx.x; it < 2 * NRX * NY; it += 256) {
    const int yy = it % NY, r = it / NY, run = r % NRX, fz = r / NRX;
    const int q0 = run * RX;
    const float* col = tz + fz * NX * NY + yy + 2 * q0 * NY;
    float v[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = col[j * NY];
    float* dst = tx + (yy & 1) * NYHP + (yy >> 1);
#pragma unroll
    for (int q = 0; q < RX; ++q) {
      float lo = 0.f, hi = 0.f;  // tap k reads input x = 2 qx - k: staged column 2 q + HALO - k of the run
#pragma unroll
      for (int k = 0; k < LA; ++k) lo = fmaf(fb.alo[k], v[2 * q + HALO - k], lo);
#pragma unroll
      for (int k = 0; k < 2; ++k) hi = fmaf(fb.ahi[k], v[2 * q + HALO - HA0 - k], hi);
      dst[((0 + 2 * fz) * FQX + q0 + q) * 2 * NYHP] = lo;
      dst[((1 + 2 * fz) * FQX + q0 + q) * 2 * NYHP] = hi;
    }
  }
  __syncthreads();
  // stage 3: pass along the fast axis, threshold, store (lanes along qy)
  const int qy = lane;
  const size_t bsz = (size_t)Oy * Ox * Oz;
  const bool row_ok = qy0 + qy < Oy;
  for (int j = w; j < 4 * FQX; j += 8) {
    const int qx = j % FQX, comb = j / FQX;
    if (!row_ok || qx0 + qx >= Ox) continue;
    const float* src = tx + (comb * FQX + qx) * 2 * NYHP;
    float v[LA];
#pragma unroll
    for (int k = 0; k < LA; ++k) {
      const int R = HALO - k;  // row 2qy + HALO - k
      v[k] = src[(R & 1) * NYHP + qy + (R >> 1)];
    }
    float lo = 0.f, hi = 0.f;
#pragma unroll
    for (int k = 0; k < LA; ++k) lo = fmaf(fb.alo[k], v[k], lo);
#pragma unroll
    for (int k = 0; k < 2; ++k) hi = fmaf(fb.ahi[k], v[HA0 + k], hi);
    const int code_lo = 2 * comb, code_hi = 2 * comb + 1;
    if (code_lo) lo = lo * (fabsf(lo) > th.tau[code_lo] ? 1.f : 0.f);
    hi = hi * (fabsf(hi) > th.tau[code_hi] ? 1.f : 0.f);
    const size_t o = (qy0 + qy) + (size_t)Oy * ((qx0 + qx) + (size_t)Ox * qz);
    out[code_lo * bsz + o] = lo;
    out[code_hi * bsz + o] = hi;
  }
}

constexpr int FSY = 64, FSX = 32;  // fast synthesis tile: samples along y and x

// Synthesis of one level for the bior / Haar banks.  A CTA makes FSY x FSX
// outputs of the two slots of one qz: the 8 bands' coefficients it needs are
// staged in shared memory, then each output is the same serial fmaf chain, in
// the same tap order, as the generic kernel and the oracle.  Each thread
// produces a run of outputs from one window of coefficients held in
// registers, so a staged coefficient is read from shared memory about once
// per run instead of once per tap:
//   y-pass: a thread makes 16 consecutive outputs (8 even/odd pairs) of one
//           (band combination, qx) column from 8 + LO lo and 8 + HI hi values;
//   x-pass: a thread makes 8 consecutive columns of one output row for both
//           slot bands, then the slot pass and the write/accumulate, in
//           registers.
// Row strides of the staged arrays are odd, so lanes that walk neighbouring
// rows hit distinct banks.  Four CTAs fit an SM by shared memory (46.7 KB
// each), so the register budget is that of four: up to 64 per thread.
template <int SL0, int SH>
__global__ void __launch_bounds__(256, 4) k_wav_synthesis_win(const float* __restrict__ bands,
                                                           const float* __restrict__ approx, int Oy, int Ox,
                                                           int Oz, SynthOut o, FastBank fb, int tx0) {
  constexpr int REACH = SH - 1 > SL0 + 1 ? SH - 1 : SL0 + 1;
  constexpr int NQY = (FSY - 1 + REACH) / 2 + 1;  // staged coefficients along y
  constexpr int NQX = (FSX - 1 + REACH) / 2 + 1;  // and along x
  constexpr int BQ = NQY | 1;                     // row stride of the staged coefficients
  constexpr int YS = FSY + 1;                     // row stride of the y-pass outputs
  constexpr int LW = (SL0 + 2) / 2;               // lo reach beyond a pair index (t + LW at most)
  constexpr int HW = SH / 2;                      // hi reach
  static_assert(FSY % 16 == 0 && FSX % 8 == 0 && FSY * (FSX / 8) == 256, "tile shape");
  extern __shared__ float sm[];
  float* B = sm;                    // [8 code][NQX qx][BQ]
  float* Y = sm + 8 * NQX * BQ;     // [4 comb][NQX qx][YS]
  const int Iy = Oy >> 1, Ix = Ox >> 1, Iz = Oz >> 1;
  const int ntx = (Ox + FSX - 1) / FSX, bx = blockIdx.y + tx0;
  const int py0 = blockIdx.x * FSY, px0 = (bx >= ntx ? bx - ntx : bx) * FSX, qz = blockIdx.z;
  const int qy0 = py0 >> 1, qx0 = px0 >> 1;
  const size_t bsz = (size_t)Iy * Ix * Iz, zoff = (size_t)Iy * Ix * qz;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  constexpr int QT = (NQY + 31) / 32;

  // stage the 8 bands (warps over (code, qx) rows, lanes over qy)
  int qyv[QT];
#pragma unroll
  for (int t = 0; t < QT; ++t) qyv[t] = wrap1(qy0 + lane + 32 * t, Iy);
  for (int qxl = w; qxl < NQX; qxl += 8) {  // the 8 bands' rows of column qx, one band after another
    const size_t coff = zoff + (size_t)Iy * wrap1(qx0 + qxl, Ix);
#pragma unroll
    for (int code = 0; code < 8; ++code) {
      const float* src = (code ? bands + code * bsz : approx) + coff;
      float* dst = B + (code * NQX + qxl) * BQ;
#pragma unroll
      for (int t = 0; t < QT; ++t) {
        const int qyl = lane + 32 * t;
        if (qyl < NQY) cp_async4(dst + qyl, src + qyv[t]);
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  // y-pass: item = (comb, run, qx); outputs py = 16 run .. 16 run + 15 of column qx
  constexpr int NRUN = FSY / 16;
  for (int it = threadIdx.x; it < 4 * NRUN * NQX; it += 256) {
    const int qxl = it % NQX, r = it / NQX, run = r % NRUN, comb = r / NRUN;
    const float* bl = B + ((2 * comb) * NQX + qxl) * BQ + 8 * run;
    const float* bh = B + ((2 * comb + 1) * NQX + qxl) * BQ + 8 * run;
    float lw[8 + LW], hw[8 + HW];
#pragma unroll
    for (int j = 0; j < 8 + LW; ++j) lw[j] = bl[j];
#pragma unroll
    for (int j = 0; j < 8 + HW; ++j) hw[j] = bh[j];
    float* dst = Y + (comb * NQX + qxl) * YS + 16 * run;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      float ev = 0.f, od = 0.f;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int k = SL0 + u;
        if (k % 2 == 0) ev = fmaf(fb.slo[u], lw[t + k / 2], ev);
        else od = fmaf(fb.slo[u], lw[t + (k + 1) / 2], od);
      }
#pragma unroll
      for (int k = 0; k < SH; ++k) {
        if (k % 2 == 0) ev = fmaf(fb.shi[k], hw[t + k / 2], ev);
        else od = fmaf(fb.shi[k], hw[t + (k + 1) / 2], od);
      }
      dst[2 * t] = ev;
      dst[2 * t + 1] = od;
    }
  }
  __syncthreads();
  // x-pass for both slot bands, then the slot pass: thread = (run of 8 columns, row py)
  const int py = threadIdx.x % FSY, run = threadIdx.x / FSY;
  float xv[2][8];
#pragma unroll
  for (int fz = 0; fz < 2; ++fz) {
    const float* yl = Y + ((2 * fz) * NQX + 4 * run) * YS + py;      // lo in x
    const float* yh = Y + ((2 * fz + 1) * NQX + 4 * run) * YS + py;  // hi in x
    float lw[4 + LW], hw[4 + HW];
#pragma unroll
    for (int j = 0; j < 4 + LW; ++j) lw[j] = yl[j * YS];
#pragma unroll
    for (int j = 0; j < 4 + HW; ++j) hw[j] = yh[j * YS];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      float ev = 0.f, od = 0.f;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int k = SL0 + u;
        if (k % 2 == 0) ev = fmaf(fb.slo[u], lw[t + k / 2], ev);
        else od = fmaf(fb.slo[u], lw[t + (k + 1) / 2], od);
      }
#pragma unroll
      for (int k = 0; k < SH; ++k) {
        if (k % 2 == 0) ev = fmaf(fb.shi[k], hw[t + k / 2], ev);
        else od = fmaf(fb.shi[k], hw[t + (k + 1) / 2], od);
      }
      xv[fz][2 * t] = ev;
      xv[fz][2 * t + 1] = od;
    }
  }
  // slot-axis pass: slot 2qz from tap 0, slot 2qz-1 from tap 1; write or accumulate
  const int gy = py0 + py;
  if (gy < Oy) {
    const int oy = wrap1(gy - o.shift, Oy);
    float* r0 = o.out + oy + (size_t)Oy * Ox * pmod(2 * qz - o.shift, Oz);
    float* r1 = o.out + oy + (size_t)Oy * Ox * pmod(2 * qz - 1 - o.shift, Oz);
    const int gx0 = px0 + 8 * run;
    int ox = wrap1(gx0 - o.shift, Ox);  // output column of gx0, then stepped by one with wrap
#pragma unroll
    for (int px = 0; px < 8; ++px) {
      if (gx0 + px < Ox) {
        const float x0 = xv[0][px], x1 = xv[1][px];
        const float v0 = fmaf(fb.szh[0], x1, fmaf(fb.szl[0], x0, 0.f));
        const float v1 = fmaf(fb.szh[1], x1, fmaf(fb.szl[1], x0, 0.f));
        const size_t col = (size_t)Oy * ox;
        float* d0 = r0 + col;
        float* d1 = r1 + col;
        float a0 = o.first ? v0 : *d0 + v0;
        float a1 = o.first ? v1 : *d1 + v1;
        if (o.last) {
          a0 = a0 / o.cycles;
          a0 = a0 > 0.f ? a0 : 0.f;
          a1 = a1 / o.cycles;
          a1 = a1 > 0.f ? a1 : 0.f;
        }
        *d0 = a0;
        *d1 = a1;
      }
      ox = ox + 1 == Ox ? 0 : ox + 1;
    }
  }
}

// Which fast kernel (if any) a bank maps to: 1 = bior shape, 2 = Haar shape.
static bool taps_are(const Taps& t, int first, int count) {
  if (t.n != count) return false;
  for (int u = 0; u < count; ++u)
    if (t.k[u] != first + u) return false;
  return true;
}

static int fast_kind(const WaveletBank& bk) {
  for (int f = 0; f < 2; ++f)
    if (!taps_are(bk.z.a[f], 0, 2) || !taps_are(bk.z.s[f], 0, 2)) return 0;
  if (taps_are(bk.xy.a[0], 0, 10) && taps_are(bk.xy.a[1], 4, 2) && taps_are(bk.xy.s[0], 4, 2) &&
      taps_are(bk.xy.s[1], 0, 10))
    return 1;
  if (taps_are(bk.xy.a[0], 0, 2) && taps_are(bk.xy.a[1], 0, 2) && taps_are(bk.xy.s[0], 0, 2) &&
      taps_are(bk.xy.s[1], 0, 2))
    return 2;
  return 0;
}

static FastBank fast_bank(const WaveletBank& bk) {
  FastBank f{};
  for (int u = 0; u < bk.xy.a[0].n; ++u) f.alo[u] = bk.xy.a[0].h[u];
  for (int u = 0; u < 2; ++u) {
    f.ahi[u] = bk.xy.a[1].h[u];
    f.slo[u] = bk.xy.s[0].h[u];
    f.azl[u] = bk.z.a[0].h[u];
    f.azh[u] = bk.z.a[1].h[u];
    f.szl[u] = bk.z.s[0].h[u];
    f.szh[u] = bk.z.s[1].h[u];
  }
  for (int u = 0; u < bk.xy.s[1].n; ++u) f.shi[u] = bk.xy.s[1].h[u];
  return f;
}

template <int LA, int HA0, bool WIN>
static cudaError_t launch_analysis_fast_t(const float* in, int Ly, int Lx, int Lz, int shift, float* out,
                                        const FastBank& fb, const LevelBands& th, cudaStream_t st,
                                        const ColRange& qcols) {
  constexpr int NY = 2 * FQY + LA - 1, NX = 2 * FQX + LA - 1, NYH = (NY + 1) / 2;
  constexpr int NYHP = ((NYH + 15) / 32) * 32 + 16;
  const size_t sm = (size_t)(2 * NX * NY + 4 * FQX * 2 * NYHP) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_wav_analysis_fast<LA, HA0, WIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int t0, nt;
  tile_span(qcols, Lx / 2, FQX, t0, nt);
  if (nt == 0) return cudaSuccess;
  dim3 grid((Ly / 2 + FQY - 1) / FQY, nt, Lz / 2);
  k_wav_analysis_fast<LA, HA0, WIN><<<grid, 256, sm, st>>>(in, Ly, Lx, Lz, shift, out, fb, th, t0);
  return cudaGetLastError();
}

template <int LA, int HA0>
static cudaError_t launch_analysis_fast(const float* in, int Ly, int Lx, int Lz, int shift, float* out,
                                        const FastBank& fb, const LevelBands& th, cudaStream_t st,
                                        const ColRange& qcols) {
  return qcols.all(Lx / 2) ? launch_analysis_fast_t<LA, HA0, false>(in, Ly, Lx, Lz, shift, out, fb, th, st, qcols)
                           : launch_analysis_fast_t<LA, HA0, true>(in, Ly, Lx, Lz, shift, out, fb, th, st, qcols);
}

template <int SL0, int SH>
static cudaError_t launch_synthesis_fast(const float* bands, const float* approx, int Oy, int Ox, int Oz,
                                         const SynthOut& o, const FastBank& fb, cudaStream_t st,
                                         const ColRange& cols) {
  constexpr int REACH = SH - 1 > SL0 + 1 ? SH - 1 : SL0 + 1;
  constexpr int NQY = (FSY - 1 + REACH) / 2 + 1, NQX = (FSX - 1 + REACH) / 2 + 1;
  const size_t sm = ((size_t)8 * NQX * (NQY | 1) + (size_t)4 * NQX * (FSY + 1)) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_wav_synthesis_win<SL0, SH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int t0, nt;
  tile_span(cols, Ox, FSX, t0, nt);
  if (nt == 0) return cudaSuccess;
  dim3 grid((Oy + FSY - 1) / FSY, nt, Oz / 2);
  k_wav_synthesis_win<SL0, SH><<<grid, 256, sm, st>>>(bands, approx, Oy, Ox, Oz, o, fb, t0);
  return cudaGetLastError();
}

// Compile-time block size version of k_ht_weights.  The group is streamed one
// slot at a time through a shared-memory slice (read once, coalesced).  Every
// difference array is slot-major, so walking the slots in order keeps each
// lane's elements (e = lane + 32 t of each array) in increasing e: the sums
// are the same fixed-order reductions as the generic kernel and the oracle.
template <int D>
__global__ void __launch_bounds__(128) k_ht_weights_t(const float* __restrict__ V, int m, int n, int M, int N,
                                                      int K, const int32_t* __restrict__ cnt,
                                                      float* __restrict__ wgt, int g0, int gn) {
  constexpr int DM = D - 3, SL = D * D, SX = D * DM;  // slice size, per-slot elements of the x/y terms
  __shared__ float sl[4][2][SL];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = window_group(blockIdx.x * 4 + warp, g0, gn, M * N);
  if (g < 0) return;
  const int i = g % M, j = g / M;
  const int nm = cnt ? cnt[g] : K;
  const size_t sz = (size_t)m * n;
  const float* base = V + (size_t)i * D + (size_t)j * D * m;
  float tx = 0.f, ty = 0.f, tz = 0.f;
  for (int k = 0; k < nm; ++k) {
    float* cur = sl[warp][k & 1];
    const float* prv = sl[warp][(k & 1) ^ 1];
    for (int t = lane; t < SL; t += 32) cur[t] = __ldg(base + (t % D) + (size_t)(t / D) * m + sz * k);
    __syncwarp();
    // x term: element r + D (c + DM k); this lane's first element of slot k
    for (int e = ((lane - k * SX) % 32 + 32) % 32; e < SX; e += 32) {
      const int r = e % D, c = e / D;
      const float* p = cur + r + c * D;
      tx = tx + fabsf(d3(p[0], p[D], p[2 * D], p[3 * D]));
    }
    // y term: element r + DM (c + D k)
    for (int e = ((lane - k * SX) % 32 + 32) % 32; e < SX; e += 32) {
      const int r = e % DM, c = e / DM;
      const float* p = cur + r + c * D;
      ty = ty + fabsf(d3(p[0], p[1], p[2], p[3]));
    }
    // slot term: element r + D (c + D (k-1)) for the pair (k-1, k)
    if (k > 0)
      for (int e = ((lane - (k - 1) * SL) % 32 + 32) % 32; e < SL; e += 32) tz = tz + fabsf(cur[e] - prv[e]);
    __syncwarp();
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

// medfilt3(Volume,[3 3 3]) (denoiseAndAggregateGPU.m:49-52) with 'symmetric'
// padding, which for a one-voxel border repeats the edge voxel.  The median
// of 27 values is a selection, exact in any order: an odd-even transposition
// sort in registers.
__global__ void __launch_bounds__(256) k_medfilt3(const float* __restrict__ V, int m, int n, int K,
                                                  float* __restrict__ out) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)m * n * K) return;
  const int y = (int)(idx % m);
  const size_t r1 = idx / m;
  const int x = (int)(r1 % n), z = (int)(r1 / n);
  float v[27];
  int q = 0;
#pragma unroll
  for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy) {
        const int yy = min(max(y + dy, 0), m - 1), xx = min(max(x + dx, 0), n - 1), zz = min(max(z + dz, 0), K - 1);
        v[q++] = __ldg(V + yy + (size_t)m * (xx + (size_t)n * zz));
      }
#pragma unroll
  for (int pass = 0; pass < 27; ++pass)
#pragma unroll
    for (int i = pass & 1; i + 1 < 27; i += 2) {
      const float a = fminf(v[i], v[i + 1]), b = fmaxf(v[i], v[i + 1]);
      v[i] = a;
      v[i + 1] = b;
    }
  out[idx] = v[13];
}

cudaError_t launch_medfilt3(const float* V, int m, int n, int K, float* out, cudaStream_t st) {
  const size_t N = (size_t)m * n * K;
  k_medfilt3<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(V, m, n, K, out);
  return cudaGetLastError();
}

static size_t analysis_smem(int reach) {
  const int NY = 2 * TQ + reach;
  return (size_t)(2 * NY * NY + 4 * TQ * NY) * sizeof(float);
}

static size_t synthesis_smem(int reach) {
  const int NQ = (TP - 1 + reach) / 2 + 1;
  return (size_t)(8 * NQ * NQ + 4 * NQ * TP + 2 * TP * TP) * sizeof(float);
}

// R when every spatial filter has exactly the taps 0..R and every slot filter
// the taps 0 and 1, else -1
static int dense_reach(const WaveletBank& bk) {
  const int R = bk.xy.a[0].n - 1;
  auto dense = [](const Taps& t, int n) {
    if (t.n != n) return false;
    for (int u = 0; u < n; ++u)
      if (t.k[u] != u) return false;
    return true;
  };
  for (int f = 0; f < 2; ++f)
    if (!dense(bk.xy.a[f], R + 1) || !dense(bk.xy.s[f], R + 1) || !dense(bk.z.a[f], 2) || !dense(bk.z.s[f], 2))
      return -1;
  return R;
}

// analysis (AN) or synthesis of a dense bank of reach R; the synthesis tile
// grid is the generic kernel's, the analysis tiles DENSE_TQ coefficients wide
constexpr int DENSE_TQ = 16;
template <bool AN, int R>
static cudaError_t launch_dense(const float* in, const float* approx, int Ly, int Lx, int Lz, int shift, float* out,
                                const SynthOut& o, const WaveletBank& bk, const LevelBands& th, cudaStream_t st,
                                const ColRange& cols) {
  if (AN) {
    constexpr int T = DENSE_TQ, NY = 2 * T + R;
    const size_t sm = (size_t)(2 * NY * NY + 4 * T * NY) * sizeof(float);
    cudaError_t e =
        cudaFuncSetAttribute(k_wav_analysis_dense<R, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    int t0, nt;
    tile_span(cols, Lx / 2, T, t0, nt);
    if (nt == 0) return cudaSuccess;
    dim3 grid((Ly / 2 + T - 1) / T, nt, Lz / 2);
    k_wav_analysis_dense<R, T><<<grid, 256, sm, st>>>(in, Ly, Lx, Lz, shift, out, bk, th, t0);
  } else {
    const size_t sm = synthesis_smem(R);
    cudaError_t e = cudaFuncSetAttribute(k_wav_synthesis_dense<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    int t0, nt;
    tile_span(cols, Lx, TP, t0, nt);
    if (nt == 0) return cudaSuccess;
    dim3 grid((Ly + TP - 1) / TP, nt, Lz / 2);
    k_wav_synthesis_dense<R><<<grid, 256, sm, st>>>(in, approx, Ly, Lx, Lz, o, bk, t0);
  }
  return cudaGetLastError();
}

cudaError_t launch_wav_analysis(const float* in, int Ly, int Lx, int Lz, int shift, float* out,
                                const WaveletBank& bk, const LevelBands& th, cudaStream_t st,
                                const ColRange& qcols) {
  const int kind = fast_kind(bk);
  // the fast kernel wraps each halo coordinate at most once
  if (kind && Ly > 2 * TQ + 16 && Lx > 2 * TQ + 16 && Lz >= 2) {
    const FastBank fb = fast_bank(bk);
    if (kind == 1) return launch_analysis_fast<10, 4>(in, Ly, Lx, Lz, shift, out, fb, th, st, qcols);
    return launch_analysis_fast<2, 0>(in, Ly, Lx, Lz, shift, out, fb, th, st, qcols);
  }
  // dense sym4 x Haar bank: one wrap of every index is enough when the level
  // exceeds a tile plus the filter reach and the shift is below every size
  if (dense_reach(bk) == 7 && shift >= 0 && Ly >= 2 * DENSE_TQ + 7 + shift && Lx >= 2 * DENSE_TQ + 7 + shift &&
      Lz >= 2 && shift + 1 <= Lz)
    return launch_dense<true, 7>(in, nullptr, Ly, Lx, Lz, shift, out, SynthOut{}, bk, th, st, qcols);
  const size_t sm = analysis_smem(bk.reach_a);
  cudaError_t e = cudaFuncSetAttribute(k_wav_analysis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int t0, nt;
  tile_span(qcols, Lx / 2, TQ, t0, nt);
  if (nt == 0) return cudaSuccess;
  dim3 grid((Ly / 2 + TQ - 1) / TQ, nt, Lz / 2);
  k_wav_analysis<<<grid, 256, sm, st>>>(in, Ly, Lx, Lz, shift, out, bk, th, t0);
  return cudaGetLastError();
}

cudaError_t launch_wav_synthesis(const float* bands, const float* approx, int Oy, int Ox, int Oz,
                                 const SynthOut& o, const WaveletBank& bk, cudaStream_t st,
                                 const ColRange& cols) {
  const int kind = fast_kind(bk);
  // coefficient tiles of 37 per axis must wrap at most once; shifts below the size
  if (kind && Oy >= 128 && Ox >= 128 && Oz >= 2 && o.shift >= 0 && o.shift < Oy && o.shift < Ox) {
    const FastBank fb = fast_bank(bk);
    if (kind == 1) return launch_synthesis_fast<4, 10>(bands, approx, Oy, Ox, Oz, o, fb, st, cols);
    return launch_synthesis_fast<0, 2>(bands, approx, Oy, Ox, Oz, o, fb, st, cols);
  }
  if (dense_reach(bk) == 7 && Oy >= 2 * TP + 8 && Ox >= 2 * TP + 8 && Oz >= 2 && o.shift >= 0 && o.shift < Oy &&
      o.shift < Ox && o.shift < Oz)
    return launch_dense<false, 7>(bands, approx, Oy, Ox, Oz, 0, nullptr, o, bk, LevelBands{}, st, cols);
  const size_t sm = synthesis_smem(bk.reach_s);
  cudaError_t e = cudaFuncSetAttribute(k_wav_synthesis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int t0, nt;
  tile_span(cols, Ox, TP, t0, nt);
  if (nt == 0) return cudaSuccess;
  dim3 grid((Oy + TP - 1) / TP, nt, Oz / 2);
  k_wav_synthesis<<<grid, 256, sm, st>>>(bands, approx, Oy, Ox, Oz, o, bk, t0);
  return cudaGetLastError();
}

// k_ht_weights for patch 8: the whole group (nm slots of 8 x 8) is staged in
// shared memory slot-major ([k][c][r]), then each lane walks its elements
// e = lane + 32 t of the three difference arrays in increasing e, as the
// other versions do.  In that layout the slot term's element e sits at e and
// e + 64, and the x term's at e + 24 k (k = e / 40), so most of the per-term
// index arithmetic goes away.
__global__ void __launch_bounds__(128) k_ht_weights_8(const float* __restrict__ V, int m, int n, int M, int N,
                                                      int K, const int32_t* __restrict__ cnt,
                                                      float* __restrict__ wgt, int g0, int gn) {
  constexpr int D = 8, DM = D - 3, SL = D * D, SX = D * DM;
  extern __shared__ float shw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = window_group(blockIdx.x * 4 + warp, g0, gn, M * N);
  if (g < 0) return;
  float* sg = shw + warp * K * SL;
  const int i = g % M, j = g / M;
  const int nm = cnt ? cnt[g] : K;
  const size_t sz = (size_t)m * n;
  // lane: row r = lane % 8 of columns lane / 8 and lane / 8 + 4 of every slot
  const float* p0 = V + (size_t)i * D + (size_t)(j * D + (lane >> 3)) * m + (lane & 7);
  const float* p1 = p0 + (size_t)4 * m;
  // slots in batches of 4: eight independent loads in flight per lane
  int k = 0;
  for (; k + 4 <= nm; k += 4) {
    float a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = __ldg(p0 + sz * (k + u));
      b[u] = __ldg(p1 + sz * (k + u));
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      sg[(k + u) * SL + lane] = a[u];
      sg[(k + u) * SL + 32 + lane] = b[u];
    }
  }
  for (; k < nm; ++k) {
    sg[k * SL + lane] = __ldg(p0 + sz * k);
    sg[k * SL + 32 + lane] = __ldg(p1 + sz * k);
  }
  __syncwarp();
  float tx = 0.f, ty = 0.f, tz = 0.f;
  // x term: element r + D (c + DM k) -> V(r, c .. c+3, k) at r + D c + SL k = e + (SL - SX) k
  for (int e = lane; e < nm * SX; e += 32) {
    const int k = e / SX;
    const float* q = sg + e + (SL - SX) * k;
    tx = tx + fabsf(d3(q[0], q[D], q[2 * D], q[3 * D]));
  }
  // y term: element r + DM (c + D k) -> V(r .. r+3, c, k)
  for (int e = lane; e < nm * SX; e += 32) {
    const int k = e / SX, rem = e - k * SX, c = rem / DM, r = rem - c * DM;
    const float* q = sg + k * SL + c * D + r;
    ty = ty + fabsf(d3(q[0], q[1], q[2], q[3]));
  }
  // slot term: element r + D (c + D k) of the pair (k, k+1)
  for (int e = lane; e < (nm - 1) * SL; e += 32) tz = tz + fabsf(sg[e + SL] - sg[e]);
  tx = warp_sum(tx);
  ty = warp_sum(ty);
  tz = warp_sum(tz);
  if (lane == 0) {
    float w = tx * 0.25f + ty * 0.25f;
    w = w + tz;
    wgt[g] = 1.f / (w + 2.220446049250313e-16f);
  }
}

cudaError_t launch_ht_weights(const float* Vavg, int m, int n, int M, int N, int d, int K,
                              const int32_t* cnt, float* wgt, cudaStream_t st, const ColRange& jcols) {
  int g0, gn;
  group_span(jcols, M, N, g0, gn);
  if (gn < 0) return cudaSuccess;
  const int G = gn > 0 ? gn : M * N;
  if (d == 16) {
    k_ht_weights_t<16><<<(G + 3) / 4, 128, 0, st>>>(Vavg, m, n, M, N, K, cnt, wgt, g0, gn);
    return cudaGetLastError();
  }
  if (d == 8) {
    const size_t smb = (size_t)4 * K * 64 * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(k_ht_weights_8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb);
    if (e != cudaSuccess) return e;
    k_ht_weights_8<<<(G + 3) / 4, 128, smb, st>>>(Vavg, m, n, M, N, K, cnt, wgt, g0, gn);
    return cudaGetLastError();
  }
  if (d == 32) {
    k_ht_weights_t<32><<<(G + 3) / 4, 128, 0, st>>>(Vavg, m, n, M, N, K, cnt, wgt, g0, gn);
    return cudaGetLastError();
  }
  k_ht_weights<<<(G + 3) / 4, 128, 0, st>>>(Vavg, m, n, M, N, d, K, cnt, wgt, g0, gn);
  return cudaGetLastError();
}

}  // namespace gbm3d
