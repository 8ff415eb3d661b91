// Deterministic owner-computes aggregation — denoiseAndAggregateGPU.m:186-208
// and denoiseAndAggregateWieFast.m:84-100.
//
// The reference adds every matched block, weighted, into U and W in the loop
// order (reference row y, reference column x, match i), each add rounded to
// single.  Here each output pixel is owned by one lane, which applies its
// contributions in exactly that order, so the result is bit-identical to the
// sequential loop and needs no atomics.
//
// Contributions falling outside the cropped image are never produced (the
// reference crops them away, denoiseAndAggregateGPU.m:207-208).
#include "common.cuh"
#include "kernels.cuh"

namespace gbm3d {

__host__ __device__ inline int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
__host__ __device__ inline int ceil_div(int a, int b) { return -floor_div(-a, b); }

constexpr int TR = 8, TC = 4;  // warp tile: 8 rows (fast axis) x 4 columns, one pixel per lane
constexpr int LCAP = 96;       // list chunk per warp (entries); walked whenever it may overflow
constexpr int BIAS = 1 << 12;  // offset added to tile-relative block origins before packing

// One warp owns TR x TC pixels, one per lane.  Candidates (reference i, j,
// slot k) whose search window can reach the tile are enumerated in the
// reference's loop order, 32 per round; the ones whose block intersects the
// tile are compacted, in order, into a shared-memory list.  An entry holds the
// block's tile-relative origin and the offsets of its data and weights minus
// that origin, so a lane reaches its own element by adding a lane constant.
// Each lane walks the list four entries at a time: four coverage tests and
// four (predicated) loads are issued together, then the covered
// contributions are added to the lane's pixel in list order.
//   step 1: value (wg * Vavg) * mask, weight wg * mask   (denoiseAndAggregateGPU.m:200-201)
//   step 2: value and weight precomputed by the Wiener kernel (:84-90 of
//           denoiseAndAggregateWieFast.m), the same single-precision products
template <int D, int D2, bool WIE, bool KAHAN>
__global__ void __launch_bounds__(128) k_aggregate_px(AggArgs A) {
  extern __shared__ int smi[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* win = reinterpret_cast<float*>(smi);
  int4* lst = reinterpret_cast<int4*>(smi + ((D * D + 3) & ~3)) + warp * LCAP;
  if (!WIE)
    for (int t = threadIdx.x; t < D * D; t += blockDim.x) win[t] = A.win[t];
  __syncthreads();
  const int tiles_r = (A.m + TR - 1) / TR, tiles_c = (A.n + TC - 1) / TC;
  const int tile = blockIdx.x * 4 + warp;
  if (tile >= tiles_r * tiles_c) return;
  const int R0 = (tile % tiles_r) * TR, C0 = (tile / tiles_r) * TC;
  const int K = A.K, s = A.s;
  const int mv = A.M * D;  // rows of the tile-space step-1 blocks
  constexpr int H = D2 / 2;
  const int PR0 = R0 + H, PC0 = C0 + H;  // tile origin in the reference's padded U
  // references whose window (origin i s, extent D + D2 - 1) can reach the tile
  const int i_lo = max(0, ceil_div(PR0 - D - D2 + 2, s)), i_hi = min(A.M - 1, floor_div(PR0 + TR - 1, s));
  const int j_lo = max(0, ceil_div(PC0 - D - D2 + 2, s)), j_hi = min(A.N - 1, floor_div(PC0 + TC - 1, s));
  const int NI = i_hi - i_lo + 1, NJ = j_hi - j_lo + 1;
  const int total = (NI > 0 && NJ > 0) ? NI * NJ * K : 0;
  const size_t mn = (size_t)mv * (A.N * D);
  const unsigned FULL = 0xffffffffu;
  // lane's candidate: slot k = lane % K when K divides 32, else by division
  const bool kdiv = (32 % K) == 0;
  const int step = kdiv ? 32 / K : 0;
  const int k_l = kdiv ? lane % K : 0, rq = kdiv ? lane / K : 0;
  int ii = rq / max(NJ, 1), jj = rq - ii * max(NJ, 1);

  const int pr = lane & 7, pc = lane >> 3;  // lane's pixel in the tile
  const int vlane = WIE ? pr + pc * D : pr + mv * pc;
  const int wlane = pr + pc * D;
  float u = 0.f, w = 0.f;
  float cu = 0.f, cw = 0.f;  // Kahan compensations
  // acc += x, rounded to single (the reference's order), or compensated
  auto add = [&](float& acc, float& comp, float x) {
    if (KAHAN) {
      const float y = x - comp;
      const float t = acc + y;
      comp = (t - acc) - y;
      acc = t;
    } else {
      acc = acc + x;
    }
  };
  auto walk = [&](int count) {
    for (int e0 = 0; e0 < count; e0 += 4) {
      int4 en[4];
      bool cov[4];
      float val[4], wv[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const bool valid = e0 + t < count;
        en[t] = lst[valid ? e0 + t : 0];
        const int rr = pr - ((en[t].x & 0xffff) - BIAS), cc = pc - ((en[t].x >> 16) - BIAS);
        cov[t] = valid && (unsigned)rr < (unsigned)D && (unsigned)cc < (unsigned)D;
        val[t] = cov[t] ? __ldg(A.blocks + ((size_t)(unsigned)(en[t].y + vlane))) : 0.f;
        if (WIE) wv[t] = cov[t] ? __ldg(A.gw + ((size_t)(unsigned)(en[t].z + wlane))) : 0.f;
        else wv[t] = cov[t] ? win[rr + cc * D] : 0.f;
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        if (cov[t]) {
          if (WIE) {
            add(u, cu, val[t]);
            add(w, cw, wv[t]);
          } else {
            const float wg = __int_as_float(en[t].z);
            add(u, cu, (wg * val[t]) * wv[t]);
            add(w, cw, wg * wv[t]);
          }
        }
      }
    }
  };

  int count = 0;
  for (int base = 0; base < total; base += 32) {
    bool hit = false;
    int4 ent = make_int4(0, 0, 0, 0);
    int k, i, j;
    if (kdiv) {
      k = k_l;
      i = i_lo + ii;
      j = j_lo + jj;
    } else {
      const int q = base + lane, r2 = q / K;
      k = q - r2 * K;
      const int i2 = r2 / NJ;
      i = i_lo + i2;
      j = j_lo + (r2 - i2 * NJ);
    }
    if (base + lane < total) {
      const int g = i + A.M * j;
      const int nm = A.cnt ? A.cnt[g] : K;
      if (k < nm) {
        const int e = (int)A.S[(size_t)g * K + k] - 1;
        const int r0 = i * s + e % D2 - PR0, c0 = j * s + e / D2 - PC0;
        hit = r0 < TR && r0 + D > 0 && c0 < TC && c0 + D > 0;
        if (hit) {
          ent.x = (r0 + BIAS) | ((c0 + BIAS) << 16);
          if (WIE) {
            ent.y = (g * K + k) * (D * D) - r0 - c0 * D;
            ent.z = g * (D * D) - r0 - c0 * D;
          } else {
            ent.y = (int)((size_t)i * D + (size_t)mv * (j * D) + mn * k) - r0 - mv * c0;
            ent.z = __float_as_int(A.gw[g]);
          }
        }
      }
    }
    if (kdiv) {  // advance this lane's reference by 32/K positions in loop order
      jj += step;
      while (jj >= NJ) { jj -= NJ; ++ii; }
    }
    const unsigned bal = __ballot_sync(FULL, hit);
    if (hit) lst[count + __popc(bal & ((1u << lane) - 1u))] = ent;
    count += __popc(bal);
    if (count > LCAP - 32) {
      __syncwarp();
      walk(count);
      __syncwarp();
      count = 0;
    }
  }
  __syncwarp();
  walk(count);
  const int orow = R0 + pr, ocol = C0 + pc;
  if (orow < A.m && ocol < A.n) {
    A.U[orow + (size_t)A.m * ocol] = u;
    A.W[orow + (size_t)A.m * ocol] = w;
  }
}

// CTA-level enumeration.  A CTA of 8 warps owns CR x CC pixels (16 warp
// tiles of TR x TC, two per warp).  The CTA enumerates the candidates (i, j, k)
// whose search window reaches its pixels once, in the reference's loop order,
// 256 per round, and compacts the blocks that intersect its pixels into a
// shared-memory list in that order (a block-wide ordered compaction: warp
// ballots, then the warps' counts in warp order).  Each warp then filters the
// CTA list, in order, for the entries that touch one of its warp tiles and
// walks them as above.  Enumerating per CTA instead of per warp tile cuts the
// reads of S and the index arithmetic about eightfold; the order in which each
// pixel receives its contributions is unchanged, so results stay bit-identical.
constexpr int CR = 32, CC = 16;                    // CTA pixel tile
constexpr int NSR = CR / TR, NSC = CC / TC;        // warp tiles per CTA tile: 4 x 4
constexpr int CAPC = 2048;                         // CTA list capacity (entries)
constexpr int NTC = 256;                           // threads per CTA
constexpr int SUBS = NSR * NSC / (NTC / 32);       // warp tiles per warp: 2

template <int D, int D2, bool WIE, bool KAHAN>
__global__ void __launch_bounds__(NTC) k_aggregate_cta(AggArgs A) {
  extern __shared__ int smi[];
  __shared__ int wcnt[NTC / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
  float* win = reinterpret_cast<float*>(smi);
  int4* lstC = reinterpret_cast<int4*>(smi + ((D * D + 3) & ~3));
  int4* lst = lstC + CAPC + warp * LCAP;
  if (!WIE)
    for (int t = tid; t < D * D; t += NTC) win[t] = A.win[t];
  const int tiles_r = (A.m + CR - 1) / CR;
  const int R0 = (blockIdx.x % tiles_r) * CR, C0 = (blockIdx.x / tiles_r) * CC;
  const int K = A.K, s = A.s;
  const int mv = A.M * D;
  constexpr int H = D2 / 2;
  const int PR0 = R0 + H, PC0 = C0 + H;
  const int i_lo = max(0, ceil_div(PR0 - D - D2 + 2, s)), i_hi = min(A.M - 1, floor_div(PR0 + CR - 1, s));
  const int j_lo = max(0, ceil_div(PC0 - D - D2 + 2, s)), j_hi = min(A.N - 1, floor_div(PC0 + CC - 1, s));
  const int NI = i_hi - i_lo + 1, NJ = j_hi - j_lo + 1;
  const int total = (NI > 0 && NJ > 0) ? NI * NJ * K : 0;
  const size_t mn = (size_t)mv * (A.N * D);
  const unsigned FULL = 0xffffffffu;

  // this lane's pixel in each of the warp's tiles (CTA-relative)
  const int pr = lane & 7, pc = lane >> 3;
  int prc[SUBS], pcc[SUBS], vlane[SUBS], wlane[SUBS];
  float u[SUBS], w[SUBS], cu[SUBS], cw[SUBS];
#pragma unroll
  for (int a = 0; a < SUBS; ++a) {
    const int sid = warp + (NTC / 32) * a;
    prc[a] = (sid % NSR) * TR + pr;
    pcc[a] = (sid / NSR) * TC + pc;
    vlane[a] = WIE ? prc[a] + pcc[a] * D : prc[a] + mv * pcc[a];
    wlane[a] = prc[a] + pcc[a] * D;
    u[a] = w[a] = cu[a] = cw[a] = 0.f;
  }
  auto add = [&](float& acc, float& comp, float x) {
    if (KAHAN) {
      const float y = x - comp;
      const float t = acc + y;
      comp = (t - acc) - y;
      acc = t;
    } else {
      acc = acc + x;
    }
  };
  // entries whose block covers the lane's pixel, in list order
  auto walk = [&](int a, int count) {
    for (int e0 = 0; e0 < count; e0 += 4) {
      int4 en[4];
      bool cov[4];
      float val[4], wv[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const bool valid = e0 + t < count;
        en[t] = lst[valid ? e0 + t : 0];
        const int rr = prc[a] - ((en[t].x & 0xffff) - BIAS), cc = pcc[a] - ((en[t].x >> 16) - BIAS);
        cov[t] = valid && (unsigned)rr < (unsigned)D && (unsigned)cc < (unsigned)D;
        val[t] = cov[t] ? __ldg(A.blocks + ((size_t)(unsigned)(en[t].y + vlane[a]))) : 0.f;
        if (WIE) wv[t] = cov[t] ? __ldg(A.gw + ((size_t)(unsigned)(en[t].z + wlane[a]))) : 0.f;
        else wv[t] = cov[t] ? win[rr + cc * D] : 0.f;
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        if (cov[t]) {
          if (WIE) {
            add(u[a], cu[a], val[t]);
            add(w[a], cw[a], wv[t]);
          } else {
            const float wg = __int_as_float(en[t].z);
            add(u[a], cu[a], (wg * val[t]) * wv[t]);
            add(w[a], cw[a], wg * wv[t]);
          }
        }
      }
    }
  };
  // every warp: its tiles' entries of the CTA list, in order
  auto process = [&](int count) {
#pragma unroll
    for (int a = 0; a < SUBS; ++a) {
      const int sr = prc[a] - pr, sc = pcc[a] - pc;  // warp tile origin (CTA-relative)
      int cnt = 0;
      for (int e0 = 0; e0 < count; e0 += 32) {
        const int e = e0 + lane;
        bool hit = false;
        int4 en = make_int4(0, 0, 0, 0);
        if (e < count) {
          en = lstC[e];
          const int r0 = (en.x & 0xffff) - BIAS - sr, c0 = (en.x >> 16) - BIAS - sc;
          hit = r0 < TR && r0 + D > 0 && c0 < TC && c0 + D > 0;
        }
        const unsigned bal = __ballot_sync(FULL, hit);
        if (hit) lst[cnt + __popc(bal & ((1u << lane) - 1u))] = en;
        cnt += __popc(bal);
        if (cnt > LCAP - 32) {
          __syncwarp();
          walk(a, cnt);
          __syncwarp();
          cnt = 0;
        }
      }
      __syncwarp();
      walk(a, cnt);
      __syncwarp();
    }
  };

  __syncthreads();  // win
  int countC = 0;
  for (int base = 0; base < total; base += NTC) {
    const int q = base + tid;
    bool hit = false;
    int4 ent = make_int4(0, 0, 0, 0);
    if (q < total) {
      const int r2 = q / K, k = q - r2 * K;
      const int i2 = r2 / NJ;
      const int i = i_lo + i2, j = j_lo + (r2 - i2 * NJ);
      const int g = i + A.M * j;
      const int nm = A.cnt ? A.cnt[g] : K;
      if (k < nm) {
        const int e = (int)A.S[(size_t)g * K + k] - 1;
        const int r0 = i * s + e % D2 - PR0, c0 = j * s + e / D2 - PC0;
        hit = r0 < CR && r0 + D > 0 && c0 < CC && c0 + D > 0;
        if (hit) {
          ent.x = (r0 + BIAS) | ((c0 + BIAS) << 16);
          if (WIE) {
            ent.y = (g * K + k) * (D * D) - r0 - c0 * D;
            ent.z = g * (D * D) - r0 - c0 * D;
          } else {
            ent.y = (int)((size_t)i * D + (size_t)mv * (j * D) + mn * k) - r0 - mv * c0;
            ent.z = __float_as_int(A.gw[g]);
          }
        }
      }
    }
    const unsigned bal = __ballot_sync(FULL, hit);
    if (lane == 0) wcnt[warp] = __popc(bal);
    __syncthreads();
    int off = countC, tot = 0;
#pragma unroll
    for (int v = 0; v < NTC / 32; ++v) {
      off += v < warp ? wcnt[v] : 0;
      tot += wcnt[v];
    }
    if (hit) lstC[off + __popc(bal & ((1u << lane) - 1u))] = ent;
    countC += tot;
    __syncthreads();
    if (countC > CAPC - NTC) {
      process(countC);
      countC = 0;
      __syncthreads();
    }
  }
  process(countC);
#pragma unroll
  for (int a = 0; a < SUBS; ++a) {
    const int orow = R0 + prc[a], ocol = C0 + pcc[a];
    if (orow < A.m && ocol < A.n) {
      A.U[orow + (size_t)A.m * ocol] = u[a];
      A.W[orow + (size_t)A.m * ocol] = w[a];
    }
  }
}

template <int D, int D2, bool WIE, bool KAHAN = false>
static cudaError_t launch_px(const AggArgs& A, cudaStream_t st) {
  const size_t sm = (size_t)((D * D + 3) & ~3) * sizeof(float) + (size_t)(CAPC + (NTC / 32) * LCAP) * sizeof(int4);
  cudaError_t e =
      cudaFuncSetAttribute(k_aggregate_cta<D, D2, WIE, KAHAN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int tiles = ((A.m + CR - 1) / CR) * ((A.n + CC - 1) / CC);
  k_aggregate_cta<D, D2, WIE, KAHAN><<<tiles, NTC, sm, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_aggregate(const AggArgs& A, cudaStream_t st) {
  // block data offsets are 32-bit in the list entries
  if ((size_t)A.m * A.n * A.K >= ((size_t)1 << 31) || (size_t)A.M * A.N * A.K * A.d * A.d >= ((size_t)1 << 31) ||
      A.s < 1 || A.s > A.d)
    return cudaErrorInvalidValue;
  if (A.kahan) {  // precision form: patch 8
#define GBM3D_AGGK_CASE(DD2) \
  if (A.d == 8 && A.d2 == DD2) return A.wiener ? launch_px<8, DD2, true, true>(A, st) : launch_px<8, DD2, false, true>(A, st);
    GBM3D_AGGK_CASE(16) GBM3D_AGGK_CASE(24) GBM3D_AGGK_CASE(32)
#undef GBM3D_AGGK_CASE
    return cudaErrorInvalidValue;
  }
#define GBM3D_AGG_CASE(DD, DD2)                                                                 \
  if (A.d == DD && A.d2 == DD2)                                                                 \
    return A.wiener ? launch_px<DD, DD2, true>(A, st) : launch_px<DD, DD2, false>(A, st);
  GBM3D_AGG_CASE(8, 16) GBM3D_AGG_CASE(8, 24) GBM3D_AGG_CASE(8, 32)
  GBM3D_AGG_CASE(16, 16) GBM3D_AGG_CASE(16, 24) GBM3D_AGG_CASE(16, 32)
  GBM3D_AGG_CASE(32, 16) GBM3D_AGG_CASE(32, 24) GBM3D_AGG_CASE(32, 32)
  GBM3D_AGG_CASE(4, 16) GBM3D_AGG_CASE(4, 24) GBM3D_AGG_CASE(4, 32)
#undef GBM3D_AGG_CASE
  return cudaErrorInvalidValue;
}

}  // namespace gbm3d
