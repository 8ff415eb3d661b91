// Deterministic owner-computes aggregation — denoiseAndAggregateGPU.m:186-208
// and denoiseAndAggregateWieFast.m:84-100.
//
// The reference adds every matched block, weighted, into U and W in the loop
// order (reference row y, reference column x, match i), each add rounded to
// single.  Here each output pixel is owned by one lane, which applies its
// contributions in exactly that order, so the result is bit-identical to the
// sequential loop and needs no atomics.
//
// One warp owns a tile of TR x TC pixels.  The warp walks the candidate
// contributions of the tile (every (reference, match) whose search window can
// reach it) in reference loop order, 32 at a time, tests them against the tile
// with a ballot and compacts the hits into a shared-memory list in the same
// order.  Each lane then walks the list for its own pixel.  Contributions
// falling outside the cropped image are never produced (the reference crops
// them away, :207-208).
#include "common.cuh"
#include "kernels.cuh"

namespace gbm3d {

constexpr int TR = 8, TC = 4;  // tile rows (fast axis) x cols

__host__ __device__ inline int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
__host__ __device__ inline int ceil_div(int a, int b) { return -floor_div(-a, b); }

static int list_max(int d, int d2, int K) {
  const int ni = (d + d2 - 2 + TR) / d + 2, nj = (d + d2 - 2 + TC) / d + 2;
  return ni * nj * K;
}

__global__ void __launch_bounds__(128) k_aggregate(AggArgs A, int lmax) {
  extern __shared__ int smi[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int d = A.d, dd = d * d, K = A.K;
  float* win = reinterpret_cast<float*>(smi);
  int* lst = smi + dd + warp * 2 * lmax;
  for (int t = threadIdx.x; t < dd; t += blockDim.x) win[t] = A.win[t];
  __syncthreads();
  const int tiles_r = (A.m + TR - 1) / TR, tiles_c = (A.n + TC - 1) / TC;
  const int tile = blockIdx.x * 4 + warp;
  if (tile >= tiles_r * tiles_c) return;
  const int R0 = (tile % tiles_r) * TR, C0 = (tile / tiles_r) * TC;
  const int h = A.d2 / 2;
  const int PR0 = R0 + h, PC0 = C0 + h;  // tile origin in the padded U of the reference
  const int i_lo = max(0, ceil_div(PR0 - d - A.d2 + 2, d)), i_hi = min(A.M - 1, floor_div(PR0 + TR - 1, d));
  const int j_lo = max(0, ceil_div(PC0 - d - A.d2 + 2, d)), j_hi = min(A.N - 1, floor_div(PC0 + TC - 1, d));
  const int NI = i_hi - i_lo + 1, NJ = j_hi - j_lo + 1;
  const int total = (NI > 0 && NJ > 0) ? NI * NJ * K : 0;
  const unsigned FULL = 0xffffffffu;
  int count = 0;
  for (int base = 0; base < total; base += 32) {
    const int q = base + lane;
    bool hit = false;
    int packed = 0, id = 0;
    if (q < total) {
      const int k = q % K, jj = (q / K) % NJ, ii = q / (K * NJ);
      const int i = i_lo + ii, j = j_lo + jj, g = i + A.M * j;
      const int nm = A.cnt ? A.cnt[g] : K;
      if (k < nm) {
        const int e = (int)A.S[(size_t)g * K + k] - 1;
        const int r0 = i * d + e % A.d2, c0 = j * d + e / A.d2;
        hit = r0 <= PR0 + TR - 1 && r0 + d - 1 >= PR0 && c0 <= PC0 + TC - 1 && c0 + d - 1 >= PC0;
        packed = r0 | (c0 << 16);
        id = g * K + k;
      }
    }
    const unsigned bal = __ballot_sync(FULL, hit);
    if (hit) {
      const int pos = count + __popc(bal & ((1u << lane) - 1u));
      lst[2 * pos] = packed;
      lst[2 * pos + 1] = id;
    }
    count += __popc(bal);
  }
  __syncwarp();
  const int pr = PR0 + (lane % TR), pc = PC0 + (lane / TR);
  const size_t mn = (size_t)A.m * A.n;
  float u = 0.f, w = 0.f;
  for (int e = 0; e < count; ++e) {
    const int packed = lst[2 * e];
    const unsigned rr = (unsigned)(pr - (packed & 0xffff)), cc = (unsigned)(pc - (packed >> 16));
    if (rr < (unsigned)d && cc < (unsigned)d) {
      const int id = lst[2 * e + 1];
      const int g = id / K, k = id % K;
      const float wk = win[rr + cc * d];
      float val, wv;
      if (!A.wiener) {
        const int i = g % A.M, j = g / A.M;
        const float blk = A.blocks[(size_t)(i * d + rr) + (size_t)A.m * (j * d + cc) + mn * k];
        const float wg = A.gw[g];
        val = (wg * blk) * wk;
        wv = wg * wk;
      } else {
        const float blk = A.blocks[(size_t)id * dd + rr + cc * d];
        wv = wk / A.gw[g];
        val = wv * blk;
      }
      u = u + val;
      w = w + wv;
    }
  }
  const int orow = R0 + lane % TR, ocol = C0 + lane / TR;
  if (orow < A.m && ocol < A.n) {
    A.U[orow + (size_t)A.m * ocol] = u;
    A.W[orow + (size_t)A.m * ocol] = w;
  }
}

// ---------------------------------------------------------------------------
// Strided-ownership version (D = 8, 16, 32).  A warp owns a 32 x 32 tile; lane
// (r, c) = (lane & 7, lane >> 3) owns the pixels (r + 8a, c + 4b), a < 4, b < 8.
// A D x D block at any offset covers D/8 rows and D/4 columns of every lane's
// pixels, so all lanes work on every contribution instead of the few whose
// pixel it happens to cover.  Per-pixel accumulators sit in shared memory,
// interleaved by lane (conflict-free).  Contributions are filtered in reference
// loop order into a chunked list whose entries carry the block's tile-relative
// origin, its data offset and its group weight; each pixel still receives its
// contributions in exactly the reference order.
// ---------------------------------------------------------------------------
constexpr int AT = 32;     // warp tile side
constexpr int LCAP = 256;  // list chunk capacity per warp

template <int D, bool WIE>
__global__ void __launch_bounds__(128) k_aggregate_tiled(AggArgs A) {
  extern __shared__ float sma[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* mask = sma;                                          // D*D
  float* acc = sma + D * D + warp * (2 * 32 * 32 + 4 * LCAP);  // [2][32 pixels][32 lanes]
  int4* lst = reinterpret_cast<int4*>(acc + 2 * 32 * 32);
  for (int t = threadIdx.x; t < D * D; t += blockDim.x) mask[t] = A.win[t];
  for (int t = lane; t < 2 * 32 * 32; t += 32) acc[t] = 0.f;
  __syncthreads();
  const int tiles_r = (A.m + AT - 1) / AT, tiles_c = (A.n + AT - 1) / AT;
  const int tile = blockIdx.x * 4 + warp;
  if (tile >= tiles_r * tiles_c) return;
  const int R0 = (tile % tiles_r) * AT, C0 = (tile / tiles_r) * AT;
  const int d2 = A.d2, K = A.K, h = d2 / 2;
  const int PR0 = R0 + h, PC0 = C0 + h;  // tile origin in the reference's padded U
  const int i_lo = max(0, ceil_div(PR0 - D - d2 + 2, D)), i_hi = min(A.M - 1, floor_div(PR0 + AT - 1, D));
  const int j_lo = max(0, ceil_div(PC0 - D - d2 + 2, D)), j_hi = min(A.N - 1, floor_div(PC0 + AT - 1, D));
  const int NI = i_hi - i_lo + 1, NJ = j_hi - j_lo + 1;
  const int total = (NI > 0 && NJ > 0) ? NI * NJ * K : 0;
  const size_t mn = (size_t)A.m * A.n;
  const int r = lane & 7, c = lane >> 3;
  const unsigned FULL = 0xffffffffu;

  auto walk = [&](int count) {
    for (int e = 0; e < count; ++e) {
      const int4 ent = lst[e];
      const int r0 = ent.x, c0 = ent.y;
      const float wgt = __int_as_float(ent.w);
      const int a_lo = max(0, (r0 - r + 7) >> 3), a_hi = min(3, (r0 + D - 1 - r) >> 3);
      const int b_lo = max(0, (c0 - c + 3) >> 2), b_hi = min(7, (c0 + D - 1 - c) >> 2);
      for (int a = a_lo; a <= a_hi; ++a) {
        const int rr = r + 8 * a - r0;
        for (int b = b_lo; b <= b_hi; ++b) {
          const int cc = c + 4 * b - c0;
          const float mk = mask[rr + cc * D];
          float val, wv;
          if (!WIE) {
            const float blk = A.blocks[(size_t)ent.z + rr + (size_t)A.m * cc];
            val = (wgt * blk) * mk;
            wv = wgt * mk;
          } else {
            const float blk = A.blocks[(size_t)ent.z * (D * D) + rr + cc * D];
            wv = mk / wgt;
            val = wv * blk;
          }
          float* p = acc + (a * 8 + b) * 32 + lane;
          p[0] = p[0] + val;
          p[32 * 32] = p[32 * 32] + wv;
        }
      }
    }
  };

  int count = 0;
  for (int base = 0; base < total; base += 32) {
    const int q = base + lane;
    bool hit = false;
    int4 ent = make_int4(0, 0, 0, 0);
    if (q < total) {
      const int k = q % K, rq = q / K, jj = rq % NJ, ii = rq / NJ;
      const int i = i_lo + ii, j = j_lo + jj, g = i + A.M * j;
      const int nm = A.cnt ? A.cnt[g] : K;
      if (k < nm) {
        const int e = (int)A.S[(size_t)g * K + k] - 1;
        const int r0 = i * D + e % d2 - PR0, c0 = j * D + e / d2 - PC0;
        hit = r0 < AT && r0 + D > 0 && c0 < AT && c0 + D > 0;
        if (hit) {
          ent.x = r0;
          ent.y = c0;
          // block data: step 1 reads the group tile of the image-shaped Vavg,
          // step 2 the filtered group (offset in units of D*D)
          ent.z = WIE ? g * K + k : 0;
          if (!WIE) {
            const size_t off = (size_t)i * D + (size_t)A.m * (j * D) + mn * k;
            ent.z = (int)off;  // fits: checked on the host (m*n*K < 2^31)
          }
          ent.w = __float_as_int(A.gw[g]);
        }
      }
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
  __syncwarp();
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 8; ++b) {
      const int orow = R0 + r + 8 * a, ocol = C0 + c + 4 * b;
      if (orow < A.m && ocol < A.n) {
        const float* p = acc + (a * 8 + b) * 32 + lane;
        A.U[orow + (size_t)A.m * ocol] = p[0];
        A.W[orow + (size_t)A.m * ocol] = p[32 * 32];
      }
    }
}

template <int D, bool WIE>
static cudaError_t launch_tiled(const AggArgs& A, cudaStream_t st) {
  const size_t sm = (size_t)(D * D + 4 * (2 * 32 * 32 + 4 * LCAP)) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_aggregate_tiled<D, WIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int tiles = ((A.m + AT - 1) / AT) * ((A.n + AT - 1) / AT);
  k_aggregate_tiled<D, WIE><<<(tiles + 3) / 4, 128, sm, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_aggregate(const AggArgs& A, cudaStream_t st) {
  const bool offsets_fit = (size_t)A.m * A.n * A.K < ((size_t)1 << 31) && (size_t)A.M * A.N * A.K < ((size_t)1 << 31);
  if (offsets_fit) {
#define GBM3D_AGG_CASE(DD)                                                           \
  if (A.d == DD) return A.wiener ? launch_tiled<DD, true>(A, st) : launch_tiled<DD, false>(A, st);
    GBM3D_AGG_CASE(8) GBM3D_AGG_CASE(16) GBM3D_AGG_CASE(32)
#undef GBM3D_AGG_CASE
  }
  const int lmax = list_max(A.d, A.d2, A.K);
  const size_t sm = (size_t)(A.d * A.d + 4 * 2 * lmax) * sizeof(int);
  cudaError_t e = cudaFuncSetAttribute(k_aggregate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int tiles = ((A.m + TR - 1) / TR) * ((A.n + TC - 1) / TC);
  k_aggregate<<<(tiles + 3) / 4, 128, sm, st>>>(A, lmax);
  return cudaGetLastError();
}

}  // namespace gbm3d
