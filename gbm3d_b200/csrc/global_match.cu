// Global block matching — matchBlocksGPU.m:19-91 (named by the task; no
// caller in GBM3D.m).
//
// The reference searches the whole image for every reference block with
// circular FFT cross-correlations, after a sym4 2D wavelet hard-threshold
// prefilter when sigma > 30/255 (five cycle shifts, three levels, tau = 2
// sigma).  Here:
//   * the prefilter runs as separable 2D analysis/synthesis passes (x-pass then
//     y-pass for analysis, y-pass then x-pass for synthesis), each output a
//     serial fmaf chain over the filter taps in ascending order;
//   * k_match_global gives each reference block one CTA: every thread computes
//     exact circular SSDs for a strided subset of the m*n positions (rows of
//     the block outer, columns inner), keeps a sorted list of its best
//     (distance, position) pairs, and the CTA merges the lists by repeated
//     block-wide arg-min in (distance, position) order.  S holds 1-based
//     positions in the m x n image; there is no slot-1 override.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.cuh"

namespace gbm3d {

// ---- 2D wavelet passes ------------------------------------------------------------
// analysis along x (slow axis): out[y][q] = sum_k h[k] in[y][(2q - k) mod Lx]
__global__ void k_w2_ax(const float* __restrict__ in, int Ly, int Lx, float* __restrict__ lo,
                        float* __restrict__ hi, Taps t0, Taps t1) {
  const int Ox = Lx / 2;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)Ly * Ox) return;
  const int y = (int)(idx % Ly), q = (int)(idx / Ly);
  float a = 0.f, b = 0.f;
  for (int u = 0; u < t0.n; ++u)
    if (t0.k[u] < Lx) a = fmaf(t0.h[u], in[y + (size_t)Ly * pmod(2 * q - t0.k[u], Lx)], a);
  for (int u = 0; u < t1.n; ++u)
    if (t1.k[u] < Lx) b = fmaf(t1.h[u], in[y + (size_t)Ly * pmod(2 * q - t1.k[u], Lx)], b);
  lo[idx] = a;
  hi[idx] = b;
}

// analysis along y (fast axis) with the hard threshold of detail bands
__global__ void k_w2_ay(const float* __restrict__ in, int Ly, int Ox, float* __restrict__ lo,
                        float* __restrict__ hi, Taps t0, Taps t1, float tau, int thr_lo) {
  const int Oy = Ly / 2;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)Oy * Ox) return;
  const int q = (int)(idx % Oy), x = (int)(idx / Oy);
  const float* col = in + (size_t)Ly * x;
  float a = 0.f, b = 0.f;
  for (int u = 0; u < t0.n; ++u)
    if (t0.k[u] < Ly) a = fmaf(t0.h[u], col[pmod(2 * q - t0.k[u], Ly)], a);
  for (int u = 0; u < t1.n; ++u)
    if (t1.k[u] < Ly) b = fmaf(t1.h[u], col[pmod(2 * q - t1.k[u], Ly)], b);
  if (thr_lo) a = a * (fabsf(a) > tau ? 1.f : 0.f);
  b = b * (fabsf(b) > tau ? 1.f : 0.f);
  lo[idx] = a;
  hi[idx] = b;
}

// synthesis along y: out[p][x] = sum_band sum_k g[k] up[(p + k) mod Oy] (lo band first)
__global__ void k_w2_sy(const float* __restrict__ lo, const float* __restrict__ hi, int Iy, int Ox,
                        float* __restrict__ out, Taps s0, Taps s1) {
  const int Oy = 2 * Iy;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)Oy * Ox) return;
  const int p = (int)(idx % Oy), x = (int)(idx / Oy);
  float acc = 0.f;
  for (int band = 0; band < 2; ++band) {
    const Taps& t = band ? s1 : s0;
    const float* src = (band ? hi : lo) + (size_t)Iy * x;
    for (int u = 0; u < t.n; ++u) {
      const int k = t.k[u];
      if (k >= Oy) continue;
      const int pk = (p + k) % Oy;
      if (pk & 1) continue;
      acc = fmaf(t.h[u], src[pk >> 1], acc);
    }
  }
  out[idx] = acc;
}

// synthesis along x
__global__ void k_w2_sx(const float* __restrict__ lo, const float* __restrict__ hi, int Oy, int Ix,
                        float* __restrict__ out, Taps s0, Taps s1) {
  const int Ox = 2 * Ix;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)Oy * Ox) return;
  const int y = (int)(idx % Oy), p = (int)(idx / Oy);
  float acc = 0.f;
  for (int band = 0; band < 2; ++band) {
    const Taps& t = band ? s1 : s0;
    const float* src = band ? hi : lo;
    for (int u = 0; u < t.n; ++u) {
      const int k = t.k[u];
      if (k >= Ox) continue;
      const int pk = (p + k) % Ox;
      if (pk & 1) continue;
      acc = fmaf(t.h[u], src[y + (size_t)Oy * (pk >> 1)], acc);
    }
  }
  out[idx] = acc;
}

// sh = circshift(I, [k, k])
__global__ void k_w2_shift(const float* __restrict__ I, int m, int n, int k, float* __restrict__ out) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)m * n) return;
  const int r = (int)(idx % m), c = (int)(idx / m);
  out[idx] = I[pmod(r - k, m) + (size_t)m * pmod(c - k, n)];
}

// avg = avg + circshift(rec, [-k, -k]) / 5   (matchBlocksGPU.m:47)
__global__ void k_w2_accum(const float* __restrict__ rec, int m, int n, int k, float* __restrict__ avg, int first) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)m * n) return;
  const int r = (int)(idx % m), c = (int)(idx / m);
  const float v = rec[pmod(r + k, m) + (size_t)m * pmod(c + k, n)] / 5.f;
  avg[idx] = first ? 0.f + v : avg[idx] + v;
}

// ---- global search ------------------------------------------------------------------
constexpr int GT = 256;  // threads per reference block

template <int D, int KT>
__global__ void __launch_bounds__(GT) k_match_global(GlobalMatchArgs A) {
  __shared__ float xr[D * D];
  __shared__ uint32_t hk[GT], hi_[GT];
  __shared__ uint32_t sel[32];
  __shared__ int s_total;
  const int tid = threadIdx.x, g = blockIdx.x;
  const int m = A.m, n = A.n, i = g % A.M, j = g / A.M;
  for (int t = tid; t < D * D; t += GT) xr[t] = A.I[(i * D + t % D) + (size_t)m * (j * D + t / D)];
  if (tid == 0) s_total = 0;
  __syncthreads();
  float nR = 0.f;
  if (A.tol_branch)
    for (int c = 0; c < D; ++c)
      for (int r = 0; r < D; ++r) nR = fmaf(xr[r + D * c], xr[r + D * c], nR);
  // per-thread sorted best list, and (tolerance branch) the first hits by position
  uint32_t tk[KT], ti[KT], fnd[KT];
#pragma unroll
  for (int q = 0; q < KT; ++q) { tk[q] = 0xffffffffu; ti[q] = 0xffffffffu; fnd[q] = 0xffffffffu; }
  int nfound = 0;
  const size_t P = (size_t)m * n;
  for (size_t p = tid; p < P; p += GT) {
    const int pr = (int)(p % m), pc = (int)(p / m);
    float acc = 0.f;
    for (int r = 0; r < D; ++r) {
      int yr = pr + r;
      if (yr >= m) yr -= m;
      for (int c = 0; c < D; ++c) {
        int xc = pc + c;
        if (xc >= n) xc -= n;
        const float t = xr[r + D * c] - __ldg(A.I + yr + (size_t)m * xc);
        acc = fmaf(t, t, acc);
      }
    }
    uint32_t key = __float_as_uint(acc), ix = (uint32_t)p;
    if (A.tol_branch && acc / nR < A.tol) {
      if (nfound < KT) {
#pragma unroll
        for (int q = 0; q < KT; ++q)
          if (q == nfound) fnd[q] = ix;
      }
      ++nfound;
    }
    if (key < tk[KT - 1]) {
#pragma unroll
      for (int q = 0; q < KT; ++q) {
        if (key < tk[q] || (key == tk[q] && ix < ti[q])) {
          const uint32_t a = tk[q], b = ti[q];
          tk[q] = key;
          ti[q] = ix;
          key = a;
          ix = b;
        }
      }
    }
  }
  // tolerance branch (matchBlocksGPU.m:74-83): find(D < tol) clamped by mink
  int want = A.K;
  bool by_position = false;
  if (A.tol_branch) {
    atomicAdd(&s_total, nfound);
    __syncthreads();
    const int total = s_total;
    if (total > A.K) want = A.K;
    else if (total < A.numMin) want = A.numMin;
    else { want = total; by_position = true; }
  }
  // merge: `want` rounds of block-wide arg-min over the list heads
  int head = 0;
  for (int round = 0; round < want; ++round) {
    uint32_t k0 = 0xffffffffu, i0 = 0xffffffffu;
#pragma unroll
    for (int q = 0; q < KT; ++q)
      if (q == head) {
        if (by_position) { k0 = fnd[q]; i0 = fnd[q]; }
        else { k0 = tk[q]; i0 = ti[q]; }
      }
    if (by_position && head >= min(nfound, KT)) { k0 = 0xffffffffu; i0 = 0xffffffffu; }
    hk[tid] = k0;
    hi_[tid] = i0;
    __syncthreads();
    for (int s = GT / 2; s > 0; s >>= 1) {
      if (tid < s) {
        const uint32_t ka = hk[tid], ia = hi_[tid], kb = hk[tid + s], ib = hi_[tid + s];
        if (kb < ka || (kb == ka && ib < ia)) { hk[tid] = kb; hi_[tid] = ib; }
      }
      __syncthreads();
    }
    const uint32_t wk = hk[0], wi = hi_[0];
    if (tid == 0) sel[round] = wi;
    if (k0 == wk && i0 == wi && i0 != 0xffffffffu) ++head;
    __syncthreads();
  }
  if (tid < A.K) A.S[(size_t)g * A.K + tid] = tid < want ? sel[tid] + 1 : 0u;
  if (tid == 0 && A.cnt) A.cnt[g] = want;
}

bool global_match_supported(int d, int K) {
  return (d == 8 || d == 16 || d == 32) && K >= 1 && K <= 32;
}

cudaError_t launch_match_global(int d, const GlobalMatchArgs& A, cudaStream_t st) {
  const int G = A.M * A.N;
  const int kt = A.K <= 16 ? 16 : 32;
#define GBM3D_GM_CASE(DD, KK)                                  \
  if (d == DD && kt == KK) {                                   \
    k_match_global<DD, KK><<<G, GT, 0, st>>>(A);               \
    return cudaGetLastError();                                 \
  }
  GBM3D_GM_CASE(8, 16) GBM3D_GM_CASE(8, 32) GBM3D_GM_CASE(16, 16) GBM3D_GM_CASE(16, 32)
  GBM3D_GM_CASE(32, 16) GBM3D_GM_CASE(32, 32)
#undef GBM3D_GM_CASE
  return cudaErrorInvalidValue;
}

static inline unsigned nblk(size_t n) { return (unsigned)((n + 255) / 256); }

// sym4 prefilter of matchBlocksGPU.m:34-50 on a device image I (m x n);
// work must hold 8 * m * n floats.
cudaError_t launch_sym4_prefilter(float* I, int m, int n, float tau, float* work, cudaStream_t st) {
  static const double lo[8] = {-0.07576571478927333, -0.02963552764599851, 0.49761866763201545, 0.8037387518059161,
                               0.29785779560527736, -0.09921954357684722, -0.012603967262037833, 0.0322231006040427};
  static const double hi[8] = {-0.0322231006040427, -0.012603967262037833, 0.09921954357684722, 0.29785779560527736,
                               -0.8037387518059161, 0.49761866763201545, 0.02963552764599851, -0.07576571478927333};
  Taps L{}, H{};
  L.n = H.n = 8;
  for (int k = 0; k < 8; ++k) {
    L.k[k] = H.k[k] = k;
    L.h[k] = (float)lo[k];
    H.h[k] = (float)hi[k];
  }
  const size_t px = (size_t)m * n;
  float* avg = work;          // m*n
  float* sh = work + px;      // m*n
  float* tx0 = sh + px;       // m*n/2
  float* tx1 = tx0 + px / 2;  // m*n/2
  float* coef = tx1 + px / 2;                // 4 bands per level: 4 * (m*n/4 + m*n/16 + m*n/64)
  float* rec = coef + px + px / 4 + px / 16;  // m*n (synthesis output / ping-pong)
  float* ytmp = rec + px;                     // m*n; the whole workspace is < 7 * m*n floats
  const int levels = 3;
  for (int k = 0; k < 5; ++k) {
    k_w2_shift<<<nblk(px), 256, 0, st>>>(I, m, n, k, sh);
    // analysis
    const float* A = sh;
    int y = m, x = n;
    float* lvl[3];
    float* c = coef;
    for (int lv = 0; lv < levels; ++lv) {
      const size_t q = (size_t)(y / 2) * (x / 2);
      lvl[lv] = c;
      k_w2_ax<<<nblk((size_t)y * (x / 2)), 256, 0, st>>>(A, y, x, tx0, tx1, L, H);
      // bands: code fy + 2 fx at c + code * q
      k_w2_ay<<<nblk(q), 256, 0, st>>>(tx0, y, x / 2, c + 0 * q, c + 1 * q, L, H, tau, 0);
      k_w2_ay<<<nblk(q), 256, 0, st>>>(tx1, y, x / 2, c + 2 * q, c + 3 * q, L, H, tau, 1);
      A = c;
      c += 4 * q;
      y /= 2;
      x /= 2;
    }
    // synthesis: from the coarsest level up; the approximation is band 0
    const float* R = lvl[levels - 1];
    for (int lv = levels - 1; lv >= 0; --lv) {
      const int oy = m >> lv, ox = n >> lv, iy = oy / 2, ix = ox / 2;
      const size_t q = (size_t)iy * ix;
      const float* B = lvl[lv];
      float* Y0 = tx0;
      float* Y1 = tx1;
      k_w2_sy<<<nblk((size_t)oy * ix), 256, 0, st>>>(R, B + 1 * q, iy, ix, Y0, L, H);
      k_w2_sy<<<nblk((size_t)oy * ix), 256, 0, st>>>(B + 2 * q, B + 3 * q, iy, ix, Y1, L, H);
      float* out = (lv % 2 == 0) ? rec : ytmp;
      k_w2_sx<<<nblk((size_t)oy * ox), 256, 0, st>>>(Y0, Y1, oy, ix, out, L, H);
      R = out;
    }
    k_w2_accum<<<nblk(px), 256, 0, st>>>(R, m, n, k, avg, k == 0);
  }
  return cudaMemcpyAsync(I, avg, px * sizeof(float), cudaMemcpyDeviceToDevice, st);
}

}  // namespace gbm3d
