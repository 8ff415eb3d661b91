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

cudaError_t launch_aggregate(const AggArgs& A, cudaStream_t st) {
  const int lmax = list_max(A.d, A.d2, A.K);
  const size_t sm = (size_t)(A.d * A.d + 4 * 2 * lmax) * sizeof(int);
  cudaError_t e = cudaFuncSetAttribute(k_aggregate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int tiles = ((A.m + TR - 1) / TR) * ((A.n + TC - 1) / TC);
  k_aggregate<<<(tiles + 3) / 4, 128, sm, st>>>(A, lmax);
  return cudaGetLastError();
}

}  // namespace gbm3d
