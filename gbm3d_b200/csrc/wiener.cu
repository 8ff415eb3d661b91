// Step 2: empirical Wiener collaborative filter, one warp per group.
//
// Restates denoiseAndAggregateWieFast.m:23-81 with myWavDec1D.m:10-26 and
// myWavRec1D.m:6-26 (and the legacy denoiseAndAggregateWie.m:16-90 when
// clamp_one is set and Ti is the transposed DCT).  Per group (d x d x K):
//   gather pilot (V1) and noisy (V2) blocks through S, or read them from
//   V1/V2 arrays;
//   page-wise DCT  Y = T X T'           (pagemtimes, serial fmaf chains)
//   circular Haar along the slots, 3 levels (2 when K < 16);
//   filt = |Y1|^2 / (|Y1|^2 + sigma^2), filt(1,1,15:end) = 1;
//   Y2 .* filt, inverse Haar, X = Ti (Y Ti'), clamp max(.,0) (and min(.,1));
//   n2 = norm(filt)^2 with the fixed 32-way reduction order, sqrt then square.
// The filtered groups and n2 feed the owner-ordered aggregation kernel.
#include "common.cuh"
#include "kernels.cuh"

namespace gbm3d {

// Circular Haar of K slots, LV = 3 levels (2 when K < 16), in registers.
// Detail of level lv at q: fmaf(cc, u[2q-1 mod L], -cc*u[2q]); approximation
// fmaf(cc, u[2q-1 mod L], cc*u[2q]).  Output layout: level-1 details,
// level-2 details, ..., approximation (myWavDec1D.m:14-25).
template <int K>
__device__ __forceinline__ void haar_dec(float* v, float cc) {
  constexpr int LV = K < 16 ? 2 : 3;
  float out[K];
  float U[K];
#pragma unroll
  for (int q = 0; q < K; ++q) U[q] = v[q];
#pragma unroll
  for (int lv = 0; lv < LV; ++lv) {
    const int L = K >> lv, cntp = K - L;
    float a[K / 2];
#pragma unroll
    for (int q = 0; q < L / 2; ++q) {
      const float u0 = U[2 * q], u1 = U[q == 0 ? L - 1 : 2 * q - 1];
      out[cntp + q] = fmaf(cc, u1, (-cc) * u0);
      a[q] = fmaf(cc, u1, cc * u0);
    }
#pragma unroll
    for (int q = 0; q < L / 2; ++q) U[q] = a[q];
  }
  constexpr int LA = K >> LV;
#pragma unroll
  for (int q = 0; q < LA; ++q) out[K - LA + q] = U[q];
#pragma unroll
  for (int q = 0; q < K; ++q) v[q] = out[q];
}

// Inverse of haar_dec (myWavRec1D.m:10-25): at each level, the detail
// contribution and the upsampled approximation contribution are formed
// separately and then added.
template <int K>
__device__ __forceinline__ void haar_rec(float* v, float cc) {
  constexpr int LV = K < 16 ? 2 : 3;
  float R[K];
#pragma unroll
  for (int q = 0; q < (K >> LV); ++q) R[q] = v[K - (K >> LV) + q];
#pragma unroll
  for (int s = 0; s < LV; ++s) {
    const int lv = LV - 1 - s;
    const int L = K >> (lv + 1), Lo = 2 * L, off = K - (K >> lv);
    float o[K];
#pragma unroll
    for (int q = 0; q < L; ++q) {
      const float dd = v[off + q];
      o[2 * q] = ((-cc) * dd) + (cc * R[q]);
      o[q == 0 ? Lo - 1 : 2 * q - 1] = (cc * dd) + (cc * R[q]);
    }
#pragma unroll
    for (int q = 0; q < Lo; ++q) R[q] = o[q];
  }
#pragma unroll
  for (int q = 0; q < K; ++q) v[q] = R[q];
}

template <int D, int K>
__global__ void __launch_bounds__(128) k_wiener(WienerArgs A) {
  constexpr int DD = D * D, GS = DD * K;
  // shared layout of one group: element (r, c) of slot page k at k*PG + r + D*c
  // (column-major pages).  The page stride D*D + D puts the 32/D pages a warp
  // touches at once on distinct bank groups, so row accesses (lane = (page,
  // row)), coefficient accesses (lane = element) and 16-byte column reads are
  // free of bank conflicts.
  constexpr int PG = DD + D, GSP = PG * K;
  constexpr int RPG = 32 / D;  // pages per 32-task round
  extern __shared__ float sm[];
  float* Tm = sm;
  float* Ti = sm + DD;
  float* s2 = sm + 2 * DD;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* b1 = sm + 3 * DD + warp * 2 * GSP;  // pilot group, later its Wiener gains
  float* b2 = b1 + GSP;                      // noisy group
  float* wvs = sm + 3 * DD + 4 * 2 * GSP + warp * DD;  // this group's aggregation weights
  for (int t = threadIdx.x; t < DD; t += blockDim.x) {
    Tm[t] = A.T[t];
    Ti[t] = A.Ti[t];
    s2[t] = A.s2[t];
  }
  __syncthreads();
  const int g = window_group(blockIdx.x * 4 + warp, A.g0, A.gn, A.M * A.N);
  if (g < 0) return;
  const float cc = 0.70710678118654752440f;
  // every task a lane runs has row r = lane % D (rounds of 32 tasks hold whole pages)
  const int r = lane % D, kq = lane / D;
  float Trow[D], Tirow[D];
#pragma unroll
  for (int j = 0; j < D; ++j) {
    Trow[j] = Tm[r + j * D];
    Tirow[j] = Ti[r + j * D];
  }

  // ---- load the two groups -----------------------------------------------
  if (A.padP) {
    const int i = g % A.M, j = g / A.M;
    // lane k decodes match k (window offsets a, b), then the offsets are broadcast
    int ma = 0, mb = 0;
    if (lane < K) {
      int e = (int)A.S[(size_t)g * K + lane] - 1;
      if ((unsigned)e >= (unsigned)(A.d2 * A.d2)) e = (A.d2 / 2) * (A.d2 + 1);  // never read outside the window
      mb = e / A.d2;
      ma = e - mb * A.d2;
    }
    // the lane's elements t = lane + 32 u of a page: row t % D, column t / D
    constexpr int NU = (DD + 31) / 32;
    size_t toff[NU];
#pragma unroll
    for (int u = 0; u < NU; ++u) {
      const int t = lane + 32 * u;
      toff[u] = (size_t)(t % D) + (size_t)(t / D) * A.P;
    }
    const size_t ibase = (size_t)(i * A.s) + (size_t)(j * A.s) * A.P;
    for (int k = 0; k < K; ++k) {
      const int a = __shfl_sync(0xffffffffu, ma, k), b = __shfl_sync(0xffffffffu, mb, k);
      const size_t o = ibase + a + (size_t)b * A.P;
#pragma unroll
      for (int u = 0; u < NU; ++u) {
        const int t = lane + 32 * u;
        if (t < DD) {
          cp_async4(b1 + k * PG + t, A.padP + o + toff[u]);
          cp_async4(b2 + k * PG + t, A.padN + o + toff[u]);
        }
      }
    }
    cp_async_wait_all();
  } else {
    const float* v1 = A.V1 + (size_t)g * GS;
    const float* v2 = A.V2 + (size_t)g * GS;
    for (int t = lane; t < GS; t += 32) {
      const int k = t / DD, e = t % DD;
      b1[k * PG + e] = v1[t];
      b2[k * PG + e] = v2[t];
    }
  }
  __syncwarp();

  // ---- forward DCT of each slot page, in place: lane (k, r) makes row r of
  // T X T'.  P[n] = sum_j T(r,j) X(j,n), then Y(r,l) = sum_n P[n] T(l,n), each
  // a serial fmaf chain from 0 in ascending j / n.  A round holds whole pages,
  // so all their rows are read before any is written.
  auto fwd = [&](float* X) {
#pragma unroll 1
    for (int k0 = 0; k0 < K; k0 += RPG) {
      const float* x = X + (k0 + kq) * PG;
      float P[D];
#pragma unroll
      for (int n = 0; n < D; ++n) {
        float col[D];
#pragma unroll
        for (int q = 0; q < D; q += 4) {
          const float4 v = *reinterpret_cast<const float4*>(x + n * D + q);
          col[q] = v.x; col[q + 1] = v.y; col[q + 2] = v.z; col[q + 3] = v.w;
        }
        float acc = 0.f;
#pragma unroll
        for (int jj = 0; jj < D; ++jj) acc = fmaf(Trow[jj], col[jj], acc);
        P[n] = acc;
      }
      float Y[D];
#pragma unroll
      for (int l = 0; l < D; ++l) {
        float acc = 0.f;
#pragma unroll
        for (int n = 0; n < D; ++n) acc = fmaf(P[n], A.T[l + n * D], acc);
        Y[l] = acc;
      }
      __syncwarp();
#pragma unroll
      for (int l = 0; l < D; ++l) X[(k0 + kq) * PG + r + D * l] = Y[l];
      __syncwarp();
    }
  };
  fwd(b1);
  fwd(b2);

  // ---- Haar along slots, Wiener gain, inverse Haar (lane per coefficient) ----
  for (int e = lane; e < DD; e += 32) {
    float v1[K], v2[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      v1[k] = b1[k * PG + e];
      v2[k] = b2[k * PG + e];
    }
    haar_dec<K>(v1, cc);
    haar_dec<K>(v2, cc);
    const float sg = s2[e];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const float p = v1[k] * v1[k];
      float f = p / (p + sg);
      if (e == 0 && k >= 14) f = 1.f;
      b1[k * PG + e] = f;
      v2[k] = v2[k] * f;
    }
    haar_rec<K>(v2, cc);
#pragma unroll
    for (int k = 0; k < K; ++k) b2[k * PG + e] = v2[k];
  }
  __syncwarp();

  // ---- n2 = norm(col(filt))^2: lane l adds elements o = l, l+32, ... ----------
  float s = 0.f;
  for (int o = lane; o < GS; o += 32) {
    const float f = b1[(o / DD) * PG + o % DD];
    s = s + f * f;
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, off);
  // weight = w / norm(col(filt))^2 (denoiseAndAggregateWieFast.m:81), one
  // division per window position, shared by the K blocks of the group
  const float nr = sqrtf(s), n2 = nr * nr;
  if (lane == 0) A.n2[g] = n2;
  for (int e = lane; e < DD; e += 32) {
    const float wv = A.win[e] / n2;
    wvs[e] = wv;
    A.wt[(size_t)g * DD + e] = wv;
  }
  __syncwarp();

  // ---- inverse DCT, lane (k, r): P(r,l) = sum_n Y(r,n) Ti(l,n) into b1 (the
  // gains are no longer needed), then X(r,l) = sum_j Ti(r,j) P(j,l) to global.
  float* og = A.out + (size_t)g * GS;
#pragma unroll 1
  for (int k0 = 0; k0 < K; k0 += RPG) {
    const int k = k0 + kq;
    const float* y = b2 + k * PG;
    float Yr[D];
#pragma unroll
    for (int n = 0; n < D; ++n) Yr[n] = y[r + D * n];
#pragma unroll
    for (int l = 0; l < D; ++l) {
      float acc = 0.f;
#pragma unroll
      for (int n = 0; n < D; ++n) acc = fmaf(Yr[n], A.Ti[l + n * D], acc);
      b1[k * PG + r + D * l] = acc;
    }
  }
  __syncwarp();
#pragma unroll 1
  for (int k0 = 0; k0 < K; k0 += RPG) {
    const int k = k0 + kq;
    const float* p = b1 + k * PG;
#pragma unroll
    for (int l = 0; l < D; ++l) {
      float col[D];
#pragma unroll
      for (int q = 0; q < D; q += 4) {
        const float4 v = *reinterpret_cast<const float4*>(p + l * D + q);
        col[q] = v.x; col[q + 1] = v.y; col[q + 2] = v.z; col[q + 3] = v.w;
      }
      float acc = 0.f;
#pragma unroll
      for (int jj = 0; jj < D; ++jj) acc = fmaf(Tirow[jj], col[jj], acc);
      float v = acc > 0.f ? acc : 0.f;
      if (A.clamp_one && v > 1.f) v = 1.f;
      og[k * DD + r + l * D] = wvs[r + l * D] * v;  // weight.*blocks(:,:,i) (:84-90)
    }
  }
}

bool wiener_supported(int d, int K) { return (d == 4 || d == 8 || d == 16) && (K == 8 || K == 16 || K == 32); }

template <int D, int K>
static cudaError_t launch_wiener_t(const WienerArgs& A, cudaStream_t st) {
  const size_t sm = (size_t)(3 * D * D + 4 * 2 * (D * D + D) * K + 4 * D * D) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_wiener<D, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int G = A.gn > 0 ? A.gn : A.M * A.N;
  if (A.gn < 0) return cudaSuccess;  // an empty window
  k_wiener<D, K><<<(G + 3) / 4, 128, sm, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_wiener(int d, const WienerArgs& A, cudaStream_t st) {
  if (A.padP && (A.s < 1 || A.s > d)) return cudaErrorInvalidValue;
#define GBM3D_WIE_CASE(DD, KK) \
  if (d == DD && A.K == KK) return launch_wiener_t<DD, KK>(A, st);
  GBM3D_WIE_CASE(8, 16) GBM3D_WIE_CASE(8, 8) GBM3D_WIE_CASE(8, 32)
  GBM3D_WIE_CASE(4, 16) GBM3D_WIE_CASE(4, 8) GBM3D_WIE_CASE(4, 32)
  GBM3D_WIE_CASE(16, 16) GBM3D_WIE_CASE(16, 8)
#undef GBM3D_WIE_CASE
  return cudaErrorInvalidValue;
}

}  // namespace gbm3d
