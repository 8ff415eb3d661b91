// Deterministic owner-computes aggregation — denoiseAndAggregateGPU.m:58-92 (loop :70-89)
// and denoiseAndAggregateWieFast.m:84-100.
//
// The reference adds every matched block, weighted, into U and W in the loop
// order (reference row y, reference column x, match i), each add rounded to
// single.  Here each output pixel is owned by one lane, which applies its
// contributions in exactly that order, so the result is bit-identical to the
// sequential loop and needs no atomics.
//
// Contributions falling outside the cropped image are never produced (the
// reference crops them away, denoiseAndAggregateGPU.m:91-92).
#include "common.cuh"
#include "kernels.cuh"

namespace gbm3d {

__host__ __device__ inline int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
__host__ __device__ inline int ceil_div(int a, int b) { return -floor_div(-a, b); }

constexpr int TR = 8, TC = 4;  // warp tile: 8 rows (fast axis) x 4 columns, one pixel per lane
constexpr int LCAP = 96;       // list chunk per warp (entries); walked whenever it may overflow
constexpr int BIAS = 1 << 12;  // offset added to tile-relative block origins before packing

// A CTA of 8 warps owns CR x CC output pixels (16 warp tiles of TR x TC, two
// per warp, one pixel per lane).
//  1. The CTA enumerates the candidates (reference i, j, slot k) whose search
//     window reaches its pixels, in the reference's loop order, 256 per
//     round, and compacts the blocks that intersect its pixels into a
//     shared-memory list in that order (warp ballots, then the warps' counts
//     in warp order).
//  2. Each warp filters the CTA list, in order, for the entries touching one
//     of its warp tiles, computing for each the mask of lanes it covers and
//     the lane-independent part of its offsets (a warp list of at most LCAP
//     entries, walked whenever it may overflow).
//  3. The walk: all lanes step through the warp list together, WB entries at
//     a time; a covered lane loads its element and adds the contribution.
// Every pixel receives its contributions in the reference's order, so the
// sums are bit-identical to the sequential loop.
//   step 1: value (wg * Vavg) * mask, weight wg * mask   (denoiseAndAggregateGPU.m:84-85)
//   step 2: value and weight precomputed by the Wiener kernel (:84-90 of
//           denoiseAndAggregateWieFast.m), the same single-precision products
constexpr int CR = 32, CC = 16;                    // CTA pixel tile
constexpr int NSR = CR / TR, NSC = CC / TC;        // warp tiles per CTA tile: 4 x 4
constexpr int NTC = 256;                           // threads per CTA
constexpr int SUBS = NSR * NSC / (NTC / 32);       // warp tiles per warp: 2
constexpr int WB = 8;                              // walk batch: entries tested and loaded together

// CAPC: CTA list capacity (entries).  A list that would overflow is walked in
// order and refilled, so any capacity gives the same sums; a small one suits
// sparse reference grids (fewer entries per tile) and lets more CTAs reside.
template <int D, int D2, bool WIE, bool KAHAN, int CAPC>
__global__ void __launch_bounds__(NTC) k_aggregate_cta(AggArgs A) {
  extern __shared__ int smi[];
  __shared__ int wcnt[NTC / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
  float* win = reinterpret_cast<float*>(smi);
  int4* lstC = reinterpret_cast<int4*>(smi + ((D * D + 3) & ~3));
  int4* lst = lstC + CAPC + warp * LCAP;
  if (!WIE)
    for (int t = tid; t < D * D; t += NTC) win[t] = A.win[t];
  const int tiles_r = (A.m + CR - 1) / CR, tiles_c = (A.n + CC - 1) / CC;
  const int tcol = (int)(blockIdx.x / tiles_r) + A.ct0;  // the window's column tiles, modulo the count
  const int R0 = (blockIdx.x % tiles_r) * CR, C0 = (tcol >= tiles_c ? tcol - tiles_c : tcol) * CC;
  const int K = A.K, s = A.s;
  const int mv = A.M * D;
  constexpr int H = D2 / 2;
  const int PR0 = R0 + H, PC0 = C0 + H;
  const int i_lo = max(0, ceil_div(PR0 - D - D2 + 2, s)), i_hi = min(A.M - 1, floor_div(PR0 + CR - 1, s));
  const int j_lo = max(0, ceil_div(PC0 - D - D2 + 2, s)), j_hi = min(A.N - 1, floor_div(PC0 + CC - 1, s));
  const int NI = i_hi - i_lo + 1, NJ = j_hi - j_lo + 1;
  const int total = (NI > 0 && NJ > 0) ? NI * NJ * K : 0;
  const unsigned invK = K > 1 ? (unsigned)(0xFFFFFFFFu / (unsigned)K) + 1u : 0u;  // ceil(2^32 / K)
  const unsigned invNJ = NJ > 1 ? (unsigned)(0xFFFFFFFFu / (unsigned)NJ) + 1u : 0u;
  const size_t mn = (size_t)mv * (A.N * D);
  const unsigned FULL = 0xffffffffu;

  // this lane's pixel in each of the warp's tiles (CTA-relative)
  const int pr = lane & 7, pc = lane >> 3;
  int prc[SUBS], pcc[SUBS];
  float u[SUBS], w[SUBS], cu[SUBS], cw[SUBS];
#pragma unroll
  for (int a = 0; a < SUBS; ++a) {
    const int sid = warp + (NTC / 32) * a;
    prc[a] = (sid % NSR) * TR + pr;
    pcc[a] = (sid / NSR) * TC + pc;
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
  // Warp-list entries carry what the lanes need precomputed for their warp
  // tile: x = the 32-bit mask of lanes whose pixel the block covers, y and z
  // the offsets of the block's data and weights minus the lane-independent
  // part, w the group weight (step 1).  A lane's element is then y + a lane
  // constant.  All lanes step through the entries together (the loads of one
  // entry fall in a few sectors); uncovered lanes skip the adds.
  const int voff = WIE ? pr + pc * D : pr + mv * pc;  // lane offset in a block's data
  const int woff = pr + pc * D;                       // lane offset in a d x d table
  auto walk = [&](int a, int count) {
    for (int e0 = 0; e0 < count; e0 += WB) {  // the list is padded to WB with empty masks
      int4 en[WB];
      bool cov[WB];
      float val[WB], wv[WB];
#pragma unroll
      for (int t = 0; t < WB; ++t) {
        en[t] = lst[e0 + t];
        cov[t] = (en[t].x >> lane) & 1;
        val[t] = cov[t] ? __ldg(A.blocks + ((size_t)(unsigned)(en[t].y + voff))) : 0.f;
        if (WIE) wv[t] = cov[t] ? __ldg(A.gw + ((size_t)(unsigned)(en[t].z + woff))) : 0.f;
        else wv[t] = cov[t] ? win[woff - en[t].z] : 0.f;
      }
#pragma unroll
      for (int t = 0; t < WB; ++t) {
        if (cov[t]) {
          if (WIE) {
            add(u[a], cu[a], val[t]);
            add(w[a], cw[a], wv[t]);
          } else {
            const float wg = __int_as_float(en[t].w);
            add(u[a], cu[a], (wg * val[t]) * wv[t]);
            add(w[a], cw[a], wg * wv[t]);
          }
        }
      }
    }
  };
  // every warp: its tiles' entries of the CTA list, in order, converted to
  // warp-list entries (mask and warp-tile-relative offsets)
  auto process = [&](int count) {
#pragma unroll
    for (int a = 0; a < SUBS; ++a) {
      const int sr = prc[a] - pr, sc = pcc[a] - pc;  // warp tile origin (CTA-relative)
      int cnt = 0;
      auto flush = [&]() {
        const int pad = (WB - (cnt % WB)) % WB;  // empty entries up to a multiple of WB
        if (lane < pad) lst[cnt + lane] = make_int4(0, 0, 0, 0);
        __syncwarp();
        walk(a, cnt + pad);
        __syncwarp();
        cnt = 0;
      };
      for (int e0 = 0; e0 < count; e0 += 32) {
        const int e = e0 + lane;
        bool hit = false;
        int4 en = make_int4(0, 0, 0, 0);
        if (e < count) {
          const int4 ec = lstC[e];
          const int r0 = (ec.x & 0xffff) - BIAS - sr, c0 = (ec.x >> 16) - BIAS - sc;  // warp-tile-relative origin
          const int rlo = max(r0, 0), rhi = min(r0 + D, TR), clo = max(c0, 0), chi = min(c0 + D, TC);
          hit = rhi > rlo && chi > clo;
          if (hit) {
            const unsigned rows = ((1u << rhi) - 1u) & ~((1u << rlo) - 1u);
            const unsigned cols = ((1u << chi) - 1u) & ~((1u << clo) - 1u);
            const unsigned spread = (cols & 1u) | ((cols & 2u) << 7) | ((cols & 4u) << 14) | ((cols & 8u) << 21);
            en.x = (int)(rows * spread);  // lane pr + 8 pc covered iff row pr and column pc are
            if (WIE) {
              en.y = ec.y - r0 - c0 * D;
              en.z = ec.z - r0 - c0 * D;
            } else {
              en.y = ec.y - r0 - mv * c0;
              en.z = r0 + c0 * D;
              en.w = ec.z;
            }
          }
        }
        const unsigned bal = __ballot_sync(FULL, hit);
        if (hit) lst[cnt + __popc(bal & ((1u << lane) - 1u))] = en;
        cnt += __popc(bal);
        if (cnt > LCAP - 32 - WB) flush();
      }
      flush();
    }
  };

  __syncthreads();  // win
  int countC = 0;
  for (int base = 0; base < total; base += NTC) {
    const int q = base + tid;
    bool hit = false;
    int4 ent = make_int4(0, 0, 0, 0);
    if (q < total) {
      // q / K and r2 / NJ by multiply-high with ceil(2^32 / divisor): exact
      // for dividends below 2^32 / divisor (here below NI NJ K < 2^20)
      const int r2 = K > 1 ? (int)__umulhi((unsigned)q, invK) : q, k = q - r2 * K;
      const int i2 = NJ > 1 ? (int)__umulhi((unsigned)r2, invNJ) : r2;
      const int i = i_lo + i2, j = j_lo + (r2 - i2 * NJ);
      const int g = i + A.M * j;
      // the count, the match index and the group weight are independent
      // loads: all three in flight before the count test (S holds K entries
      // per group whatever the count)
      const int nm = A.cnt ? __ldg(A.cnt + g) : K;
      const int eS = (int)__ldg(A.S + (size_t)g * K + k) - 1;
      const float gwv = WIE ? 0.f : __ldg(A.gw + g);
      if (k < nm) {
        const int e = eS;
        const int r0 = i * s + e % D2 - PR0, c0 = j * s + e / D2 - PC0;
        hit = r0 < CR && r0 + D > 0 && c0 < CC && c0 + D > 0;
        if (hit) {
          ent.x = (r0 + BIAS) | ((c0 + BIAS) << 16);
          if (WIE) {
            ent.y = (g * K + k) * (D * D);
            ent.z = g * (D * D);
          } else {
            ent.y = (int)((size_t)i * D + (size_t)mv * (j * D) + mn * k);
            ent.z = __float_as_int(gwv);
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

template <int D, int D2, bool WIE, bool KAHAN, int CAPC>
static cudaError_t launch_px_cap(const AggArgs& A, cudaStream_t st) {
  const size_t sm = (size_t)((D * D + 3) & ~3) * sizeof(float) + (size_t)(CAPC + (NTC / 32) * LCAP) * sizeof(int4);
  cudaError_t e = cudaFuncSetAttribute(k_aggregate_cta<D, D2, WIE, KAHAN, CAPC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  AggArgs B = A;
  int nt;
  tile_span(A.cols, A.n, CC, B.ct0, nt);
  if (nt == 0) return cudaSuccess;
  const int tiles = ((A.m + CR - 1) / CR) * nt;
  k_aggregate_cta<D, D2, WIE, KAHAN, CAPC><<<tiles, NTC, sm, st>>>(B);
  return cudaGetLastError();
}

// List capacity from the expected entries of a tile: (candidate references
// across the tile's reach) x K, about a quarter of which touch the tile.
template <int D, int D2, bool WIE, bool KAHAN = false>
static cudaError_t launch_px(const AggArgs& A, cudaStream_t st) {
  const long refs = (long)((CR + D + D2 - 2) / A.s + 1) * ((CC + D + D2 - 2) / A.s + 1);
  if (refs * A.K / 4 <= 1024 - NTC) return launch_px_cap<D, D2, WIE, KAHAN, 1024>(A, st);
  return launch_px_cap<D, D2, WIE, KAHAN, 2048>(A, st);
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
