// Block matching — the search of matchBlocksCPU.m:21-116 and matchBlocksWie.m:21-92.
//
// One warp per reference block.  The block's search window (d+d2-1)^2 of the
// padded image sits in shared memory; lane a owns the d2 candidates with row
// offset a (one per column offset b) and streams the window rows a+r past its
// d2 accumulators, so every shared-memory read of a warp touches 32
// consecutive words.  The reference block itself is read from the window
// (it is the candidate at offset (d2/2, d2/2)) by warp-uniform broadcasts.
//
// Distances are exact FP32 sums of squared differences, row-major over the
// block: t = x - y; acc = fmaf(t, t, acc), in scalar instructions, which the
// scheduler spreads over both FP32 pipes (fmaheavy and fmalite); the paired
// f32x2 form of the same operations issues half as many instructions but runs
// on fmaheavy alone and measured 23 % slower.  The K best candidates are the K
// smallest (distance, column-major window index) pairs — the stable order of
// MATLAB's mink — found by a bitwise radix search for the K-th smallest
// distance with warp reductions, then an index-ordered pick among ties.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace gbm3d {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}
}  // namespace

bool encode_search_map(CUtensorMap* tm, const float* pad, int R, int Q, int P, int box_rows, int box_cols) {
  auto encode = encode_fn();
  if (!encode || (reinterpret_cast<uintptr_t>(pad) & 15) || (P & 3) || R < 1 || Q < 1 || P < R) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)R, (cuuint64_t)Q};
  const cuuint64_t strides[1] = {(cuuint64_t)P * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)box_rows, (cuuint32_t)box_cols};
  const cuuint32_t es[2] = {1, 1};
  return encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(pad), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Ipad of the reference for a circularly shifted image: rows (m+d2), cols
// (n+d2), column pitch P floats.  spin is the circshift applied to the image.
// A thread writes rows 4 t .. 4 t + 3 of column x as one 16-byte store (P is a
// multiple of 4; rows R .. P-1 of the pitch are never read as image rows).
__global__ void k_make_pad(const float* __restrict__ img, int m, int n, int h, int spin,
                           float* __restrict__ pad, int P, int R, int Q) {
  const int y0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int x = blockIdx.y;
  if (y0 >= P || x >= Q) return;
  // (pad_index(r) - spin) mod L without divisions when h <= L and 0 <= spin <= L
  // (r < L + 2h, so pad_index needs at most one wrap); the general form otherwise
  auto src = [&](int r, int L) {
    if (h <= L && (unsigned)spin <= (unsigned)L) {
      int t = r < h ? r + h : r - h;
      if (t >= L) t -= L;
      t -= spin;
      return t < 0 ? t + L : t;
    }
    return pmod(pad_index(r, L, h) - spin, L);
  };
  const float* col = img + (size_t)src(x, n) * m;
  const float4 v = make_float4(col[src(y0, m)], col[src(y0 + 1, m)], col[src(y0 + 2, m)], col[src(y0 + 3, m)]);
  *reinterpret_cast<float4*>(pad + y0 + (size_t)x * P) = v;
}

// Column pitch of a staged search window of WD rows: its first row sits up to
// 3 rows into a TMA box that starts on a 16-byte boundary.
__host__ __device__ constexpr int win_pitch(int wd) { return (wd + 3 + 3) & ~3; }
// Floats of one warp's window buffer (a multiple of 32: 128-byte aligned buffers).
__host__ __device__ constexpr int win_floats(int wd) { return (win_pitch(wd) * wd + 31) & ~31; }
constexpr long long MATCH_WAIT_CYCLES = 4000000000LL;  // ~2 s at 2 GHz

// The search of reference g by one warp: win holds win_floats(D + D2 - 1)
// floats of shared memory (128-byte aligned), lst 224 words (keys, indices, S
// and the bounded set), mbar the warp's mbarrier (phase: its parity).
template <int D, int D2>
__device__ __forceinline__ void match_ref(const MatchArgs& A, const CUtensorMap* tmap, const int g, float* win,
                                          uint32_t* lst, uint64_t* mbar, uint32_t& phase, const int lane) {
  constexpr int WD = D + D2 - 1;  // window rows/cols that candidates touch
  constexpr int WP = win_pitch(WD);
  constexpr int H = D2 / 2;
  const int i = g % A.M, j = g / A.M;

  // ---- stage the search window: one TMA copy (this GPU's search image, no
  // multicast) of a WP x WD box whose first row i s is rounded down to a
  // multiple of 4 (a 16-byte aligned coordinate); the window starts o rows
  // into each staged column.  Rows past the search image read as zero.
  const int y0 = i * A.s, o = y0 & 3;
  if (lane == 0) {
    tc::fence_proxy_async();  // this warp's earlier reads of the buffer come first
    tc::mbar_expect_tx(mbar, WP * WD * (int)sizeof(float));
    tc::tma_load_2d(win, tmap, y0 - o, j * A.s, mbar);
  }
  if (!tc::mbar_wait(mbar, phase, MATCH_WAIT_CYCLES)) {
    // the copy did not land in time: give it the full limit again before the
    // buffer is reused, report, and leave this reference's S unwritten
    tc::mbar_wait(mbar, phase, MATCH_WAIT_CYCLES);
    phase ^= 1u;
    if (lane == 0 && A.err) atomicOr(A.err, 4);
    return;
  }
  phase ^= 1u;
  const float* wv = win + o;

  // ---- exact SSD for the lane's candidates (a = lane, b = 0..D2-1) ----------
  // Candidate b sees t = x(r, c) - y, acc = fmaf(t, t, acc) in (r, c) order
  // (c = xw - b ascends with the window column xw).
  float acc[D2];
#pragma unroll
  for (int b = 0; b < D2; ++b) acc[b] = 0.f;
  const int a = lane < D2 ? lane : 0;
#pragma unroll 1
  for (int r = 0; r < D; ++r) {
    float xr[D];
#pragma unroll
    for (int c = 0; c < D; ++c) xr[c] = wv[(H + r) + (H + c) * WP];
    const float* wrow = wv + (a + r);
#pragma unroll
    for (int xw = 0; xw < WD; ++xw) {
      const float w = wrow[xw * WP];
#pragma unroll
      for (int b = 0; b < D2; ++b) {
        const int c = xw - b;
        if (c >= 0 && c < D) {
          const float t = xr[c] - w;
          acc[b] = fmaf(t, t, acc[b]);
        }
      }
    }
  }

  // ---- selection -------------------------------------------------------------
  const unsigned FULL = 0xffffffffu;
  uint32_t key[D2];
#pragma unroll
  for (int b = 0; b < D2; ++b) key[b] = lane < D2 ? __float_as_uint(acc[b]) : 0xffffffffu;
  const int K = A.K;
  uint32_t selmask = 0;
  int count = K;
  bool index_order = false;  // tolerance branch with numMin <= #found <= numMax
  int want = K;
  if (A.tol_branch) {
    // matchBlocksCPU.m:89-99: D = ssd/||xR||^2 compared with tol.
    float nR = 0.f;
    for (int c = 0; c < D; ++c)
      for (int r = 0; r < D; ++r) {
        const float xv = wv[(H + r) + (H + c) * WP];
        nR = fmaf(xv, xv, nR);
      }
    int nf = 0;
#pragma unroll
    for (int b = 0; b < D2; ++b)
      if (lane < D2 && __uint_as_float(key[b]) / nR < A.tol) { selmask |= 1u << b; ++nf; }
    const int found = __reduce_add_sync(FULL, nf);
    if (found > K) { want = K; selmask = 0; }
    else if (found < A.numMin) { want = A.numMin; selmask = 0; }
    else { index_order = true; count = found; }
    if (!index_order) count = want;
  }
  // Fast exact path: T = the want-th smallest of the 32 lane minima is >= the
  // want-th smallest key, so the selection lies in {key <= T}.  When that set
  // holds at most 64 keys, rank them by (key, index) directly.
  uint32_t* lkey = lst;
  uint32_t* lidx = lst + 32;
  uint32_t* lS = lst + 64;
  uint32_t* bkey = lst + 96;   // 64 keys and 64 indices of the bounded candidate set
  uint32_t* bidx = lst + 160;
  bool ranked = false;
  if (!index_order) {
    uint32_t lm = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < D2; ++b) lm = min(lm, key[b]);
    // bitonic sort of the lane minima across the warp (ascending by lane)
    uint32_t v = lm;
#pragma unroll
    for (int k2 = 2; k2 <= 32; k2 <<= 1)
#pragma unroll
      for (int j2 = k2 >> 1; j2 > 0; j2 >>= 1) {
        const uint32_t o = __shfl_xor_sync(FULL, v, j2);
        const bool up = ((lane & k2) == 0), lower = ((lane & j2) == 0);
        v = (lower == up) ? min(v, o) : max(v, o);
      }
    uint32_t T = __shfl_sync(FULL, v, want - 1);
    int cl = 0;
#pragma unroll
    for (int b = 0; b < D2; ++b) cl += key[b] <= T ? 1 : 0;
    int C = __reduce_add_sync(FULL, cl);
    if (T != 0xffffffffu && C > 64) {
      // Tighter bound (smooth images, where many keys tie with the lane
      // minima): T2 = the want-th smallest of the 64 values {lane minimum,
      // lane second minimum}, still >= the want-th smallest key.  With A the
      // sorted minima and B the sorted second minima, the want-th smallest of
      // A u B is the smallest max(A[i-1], B[want-1-i]) over i = 0..want.
      uint32_t m1 = 0xffffffffu, m2 = 0xffffffffu;
#pragma unroll
      for (int b = 0; b < D2; ++b) {
        const uint32_t kb = key[b];
        if (kb < m1) { m2 = m1; m1 = kb; } else if (kb < m2) m2 = kb;
      }
      uint32_t vb = m2;
#pragma unroll
      for (int k2 = 2; k2 <= 32; k2 <<= 1)
#pragma unroll
        for (int j2 = k2 >> 1; j2 > 0; j2 >>= 1) {
          const uint32_t o = __shfl_xor_sync(FULL, vb, j2);
          const bool up = ((lane & k2) == 0), lower = ((lane & j2) == 0);
          vb = (lower == up) ? min(vb, o) : max(vb, o);
        }
      const uint32_t a_prev = __shfl_sync(FULL, v, (lane + 31) & 31);          // A[lane - 1]
      const uint32_t b_pair = __shfl_sync(FULL, vb, (want - 1 - lane) & 31);  // B[want - 1 - lane]
      uint32_t cand = 0xffffffffu;
      if (lane <= want - 1)  // i = lane in 0 .. want - 1 (i = want is T itself)
        cand = max(lane == 0 ? 0u : a_prev, b_pair);
      T = min(T, __reduce_min_sync(FULL, cand));
      cl = 0;
#pragma unroll
      for (int b = 0; b < D2; ++b) cl += key[b] <= T ? 1 : 0;
      C = __reduce_add_sync(FULL, cl);
    }
    if (T != 0xffffffffu && C <= 64) {
      int pos = cl;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, pos, o);
        if (lane >= o) pos += t;
      }
      pos -= cl;
#pragma unroll
      for (int b = 0; b < D2; ++b)
        if (key[b] <= T) {
          bkey[pos] = key[b];
          bidx[pos] = (uint32_t)(a + b * D2);
          ++pos;
        }
      __syncwarp();
      for (int q = lane; q < C; q += 32) {
        const uint32_t kv = bkey[q], ix = bidx[q];
        int rank = 0;
        for (int t = 0; t < C; ++t) {
          const uint32_t k2 = bkey[t], i2 = bidx[t];
          rank += (k2 < kv || (k2 == kv && i2 < ix)) ? 1 : 0;
        }
        if (rank < want) lS[rank] = rank == 0 ? (uint32_t)(H + H * D2 + 1) : ix + 1;
      }
      ranked = true;
    }
  }
  if (!index_order && !ranked) {
    // radix search for v* = the want-th smallest key (keys are >= +0 floats)
    uint32_t p = 0;
#pragma unroll 1
    for (int bit = 30; bit >= 0; --bit) {
      const uint32_t t = p | ((1u << bit) - 1u);
      int c = 0;
#pragma unroll
      for (int b = 0; b < D2; ++b) c += key[b] <= t ? 1 : 0;
      if (__reduce_add_sync(FULL, c) < want) p |= 1u << bit;
    }
    int lt = 0;
#pragma unroll
    for (int b = 0; b < D2; ++b)
      if (key[b] < p) { selmask |= 1u << b; ++lt; }
    const int need = want - __reduce_add_sync(FULL, lt);
    // ties at v*: lowest column-major index first (b major, a = lane minor)
    int taken = 0;
    const unsigned below = (1u << lane) - 1u;
#pragma unroll
    for (int b = 0; b < D2; ++b) {
      const unsigned eq = __ballot_sync(FULL, key[b] == p);
      if (taken < need && eq) {
        const bool mine = (eq >> lane) & 1u;
        if (mine && taken + __popc(eq & below) < need) selmask |= 1u << b;
        taken += __popc(eq);
      }
    }
  }

  // ---- order the selection and write S ---------------------------------------
  if (!ranked) {
  int mine = __popc(selmask);
  int pos = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(FULL, pos, o);
    if (lane >= o) pos += v;
  }
  pos -= mine;
#pragma unroll
  for (int b = 0; b < D2; ++b)
    if ((selmask >> b) & 1u) {
      lkey[pos] = key[b];
      lidx[pos] = (uint32_t)(a + b * D2);
      ++pos;
    }
  __syncwarp();
  const uint32_t ref_idx = (uint32_t)(H + H * D2 + 1);  // matchBlocksCPU.m:103
  if (lane < count) {
    const uint32_t kv = lkey[lane], ix = lidx[lane];
    int rank = 0;
    for (int t = 0; t < count; ++t) {
      const uint32_t k2 = lkey[t], i2 = lidx[t];
      if (index_order) rank += i2 < ix ? 1 : 0;
      else rank += (k2 < kv || (k2 == kv && i2 < ix)) ? 1 : 0;
    }
    lS[rank] = rank == 0 ? ref_idx : ix + 1;
  }
  }
  __syncwarp();
  uint32_t* Sg = A.S + (size_t)g * K;
  if (lane < K) Sg[lane] = lane < count ? lS[lane] : 0u;
  if (lane == 0 && A.cnt) A.cnt[g] = count;

  // ---- optional gathers: Volume (matchBlocksCPU.m:107-114), V1/V2 (matchBlocksWie.m:85-89)
  if (A.volume) {
    const size_t mn = (size_t)A.m * A.n;
    float* vol0 = A.volume + (size_t)(i * D) + (size_t)A.m * (j * D);
    if (D == 8 && (A.m & 3) == 0 && (reinterpret_cast<uintptr_t>(A.volume) & 15) == 0) {
      // two slots per pass: lane = (slot parity, column c, half-column r0); each
      // lane stores four rows of one column as one 16-byte store (a block
      // column is 32 contiguous bytes of the volume, 16-byte aligned here)
      const int q = lane & 15, c = q >> 1, r0 = 4 * (q & 1);
      for (int k = lane >> 4; k < K; k += 2) {
        int aa = H, bb = H;
        if (k < count) {
          const int e = (int)lS[k] - 1;
          if ((unsigned)e < (unsigned)(D2 * D2)) { aa = e % D2; bb = e / D2; }
        }
        const float* ws = wv + aa + r0 + (bb + c) * WP;
        *reinterpret_cast<float4*>(vol0 + r0 + (size_t)A.m * c + mn * k) = make_float4(ws[0], ws[1], ws[2], ws[3]);
      }
    } else {
    // lane-parallel over the block: element t = lane + 32 u is row t % D, column t / D
    for (int k = 0; k < K; ++k) {
      int aa = H, bb = H;
      if (k < count) {
        const int e = (int)lS[k] - 1;
        if ((unsigned)e < (unsigned)(D2 * D2)) { aa = e % D2; bb = e / D2; }
      }
      const float* wsrc = wv + aa + bb * WP;
#pragma unroll
      for (int u = 0; u < (D * D + 31) / 32; ++u) {
        const int t = lane + 32 * u;
        if (t < D * D) {
          const int r = t % D, c = t / D;
          vol0[(size_t)r + (size_t)A.m * c + mn * k] = wsrc[r + c * WP];
        }
      }
    }
    }
  }
  if (A.V1 || A.V2) {
    const float* src2 = A.pad2 + (size_t)i * A.s + (size_t)j * A.s * A.P;
    for (int k = 0; k < K; ++k) {
      int e = (int)lS[k] - 1;
      if ((unsigned)e >= (unsigned)(D2 * D2)) e = H + H * D2;
      const int aa = e % D2, bb = e / D2;
      float* o1 = A.V1 ? A.V1 + (size_t)D * D * (k + (size_t)K * g) : nullptr;
      float* o2 = A.V2 ? A.V2 + (size_t)D * D * (k + (size_t)K * g) : nullptr;
      for (int t = lane; t < D * D; t += 32) {
        const int r = t % D, c = t / D;
        if (o1) o1[t] = wv[(aa + r) + (bb + c) * WP];
        if (o2) o2[t] = src2[(aa + r) + (size_t)(bb + c) * A.P];
      }
    }
  }
}

// Shared memory of a 4-warp CTA: the warps' window buffers, their lst words,
// their mbarriers.
template <int D, int D2>
struct MatchSmem {
  static constexpr int WF = win_floats(D + D2 - 1);
  static constexpr size_t LST = (size_t)4 * WF * sizeof(float);
  static constexpr size_t MBAR = LST + (size_t)4 * 224 * sizeof(uint32_t);
  static constexpr size_t BYTES = MBAR + 4 * sizeof(uint64_t);
};

// WIN: the group window of the strip form (A.g0, A.gn); without it the grid
// covers every group in order.
template <int D, int D2, bool WIN>
__global__ void __launch_bounds__(128, 7) k_match(const __grid_constant__ CUtensorMap tmap, MatchArgs A) {
  using SM = MatchSmem<D, D2>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = WIN ? window_group(blockIdx.x * 4 + warp, A.g0, A.gn, A.M * A.N) : blockIdx.x * 4 + warp;
  if (WIN ? g < 0 : g >= A.M * A.N) return;  // warp-uniform
  float* win = reinterpret_cast<float*>(smem_raw) + warp * SM::WF;
  uint32_t* lst = reinterpret_cast<uint32_t*>(smem_raw + SM::LST) + warp * 224;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + SM::MBAR) + warp;
  if (lane == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  __syncwarp();
  uint32_t phase = 0;
  match_ref<D, D2>(A, &tmap, g, win, lst, mbar, phase, lane);
}

// List mode: the references A.list[0 .. *A.list_count), grid-stride over the list.
template <int D, int D2>
__global__ void __launch_bounds__(128) k_match_list(const __grid_constant__ CUtensorMap tmap, MatchArgs A) {
  using SM = MatchSmem<D, D2>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* win = reinterpret_cast<float*>(smem_raw) + warp * SM::WF;
  uint32_t* lst = reinterpret_cast<uint32_t*>(smem_raw + SM::LST) + warp * 224;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + SM::MBAR) + warp;
  if (lane == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  __syncwarp();
  uint32_t phase = 0;
  const int n = *A.list_count;
  for (int t = blockIdx.x * 4 + warp; t < n; t += gridDim.x * 4) {
    const int g = A.list[t];
    if ((unsigned)g < (unsigned)(A.M * A.N)) match_ref<D, D2>(A, &tmap, g, win, lst, mbar, phase, lane);
    __syncwarp();  // the next reference restages win and lst
  }
}

template <int D, int D2, bool WIN>
static cudaError_t launch_match_t(const MatchArgs& A, cudaStream_t st) {
  constexpr int WD = D + D2 - 1;
  const size_t sm = MatchSmem<D, D2>::BYTES;
  CUtensorMap tm;
  if (!encode_search_map(&tm, A.pad, A.R, A.Q, A.P, win_pitch(WD), WD)) return cudaErrorInvalidValue;
  // The attribute belongs to the current device, so it is set before every
  // launch (a host-side call that costs well under a microsecond) rather than
  // remembered once per process: a second device, or another host thread on
  // it, would otherwise launch without it.
  cudaError_t e = cudaFuncSetAttribute(k_match<D, D2, WIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int G = A.gn > 0 ? A.gn : A.M * A.N;
  if (A.gn < 0) return cudaSuccess;  // an empty window
  k_match<D, D2, WIN><<<(G + 3) / 4, 128, sm, st>>>(tm, A);
  return cudaGetLastError();
}

template <int D, int D2>
static cudaError_t launch_match_list_t(const MatchArgs& A, cudaStream_t st) {
  constexpr int WD = D + D2 - 1;
  const size_t sm = MatchSmem<D, D2>::BYTES;
  CUtensorMap tm;
  if (!encode_search_map(&tm, A.pad, A.R, A.Q, A.P, win_pitch(WD), WD)) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_match_list<D, D2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int G = A.M * A.N;
  // enough warps for the rare references a list holds; the rest exit at once
  const int blocks = std::min((G + 3) / 4, 2 * 148);
  k_match_list<D, D2><<<blocks, 128, sm, st>>>(tm, A);
  return cudaGetLastError();
}

cudaError_t launch_match_list(int d, int d2, const MatchArgs& A, cudaStream_t st) {
  if (A.s < 1 || A.s > d || !A.list || !A.list_count) return cudaErrorInvalidValue;
#define GBM3D_MATCHL_CASE(DD, DD2) \
  if (d == DD && d2 == DD2) return launch_match_list_t<DD, DD2>(A, st);
  GBM3D_MATCHL_CASE(8, 16) GBM3D_MATCHL_CASE(8, 24) GBM3D_MATCHL_CASE(8, 32)
#undef GBM3D_MATCHL_CASE
  return cudaErrorInvalidValue;
}

bool match_supported(int d, int d2) {
  return (d == 8 || d == 16 || d == 32) && (d2 == 16 || d2 == 24 || d2 == 32);
}

cudaError_t launch_match(int d, int d2, const MatchArgs& A, cudaStream_t st) {
  if (A.s < 1 || A.s > d) return cudaErrorInvalidValue;
#define GBM3D_MATCH_CASE(DD, DD2) \
  if (d == DD && d2 == DD2) return A.gn ? launch_match_t<DD, DD2, true>(A, st) : launch_match_t<DD, DD2, false>(A, st);
  GBM3D_MATCH_CASE(8, 16) GBM3D_MATCH_CASE(8, 24) GBM3D_MATCH_CASE(8, 32)
  GBM3D_MATCH_CASE(16, 16) GBM3D_MATCH_CASE(16, 24) GBM3D_MATCH_CASE(16, 32)
  GBM3D_MATCH_CASE(32, 16) GBM3D_MATCH_CASE(32, 24) GBM3D_MATCH_CASE(32, 32)
#undef GBM3D_MATCH_CASE
  return cudaErrorInvalidValue;
}

// Gather the blocks a match set selects from another image's search image:
// the colour form matches on luma and filters every channel with those sets.
// vol is tile-space (vm = M d rows), block (i, j) slot k at rows i d, cols j d.
__global__ void k_gather_volume(const float* __restrict__ pad, int P, int M, int N, int s, int d, int d2, int K,
                                const uint32_t* __restrict__ S, const int32_t* __restrict__ cnt,
                                float* __restrict__ vol, int vm, int vn) {
  const size_t total = (size_t)M * N * K * d * d;
  const int h = d2 / 2;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(t % d), c = (int)((t / d) % d);
    const size_t gk = t / ((size_t)d * d);
    const int k = (int)(gk % K);
    const size_t g = gk / K;
    const int i = (int)(g % M), j = (int)(g / M);
    int e = (int)S[g * K + k] - 1;
    if ((cnt && k >= cnt[g]) || (unsigned)e >= (unsigned)(d2 * d2)) e = h + h * d2;
    const int a = e % d2, b = e / d2;
    vol[(size_t)(i * d + r) + (size_t)vm * (j * d + c) + (size_t)vm * vn * k] =
        pad[(size_t)(i * s + a + r) + (size_t)(j * s + b + c) * P];
  }
}

cudaError_t launch_gather_volume(const float* pad, int P, int M, int N, int s, int d, int d2, int K, const uint32_t* S,
                                 const int32_t* cnt, float* vol, cudaStream_t st) {
  k_gather_volume<<<1184, 256, 0, st>>>(pad, P, M, N, s, d, d2, K, S, cnt, vol, M * d, N * d);
  return cudaGetLastError();
}

cudaError_t launch_make_pad(const float* img, int m, int n, int d2, int spin, float* pad, int P,
                            cudaStream_t st) {
  const int R = m + d2, Q = n + d2;
  dim3 grid((P / 4 + 255) / 256, Q);
  if ((P & 3) || P < R || (reinterpret_cast<uintptr_t>(pad) & 15)) return cudaErrorInvalidValue;
  k_make_pad<<<grid, 256, 0, st>>>(img, m, n, d2 / 2, spin, pad, P, R, Q);
  return cudaGetLastError();
}

}  // namespace gbm3d
