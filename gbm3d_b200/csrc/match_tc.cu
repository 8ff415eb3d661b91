// Block matching, precision form: BF16 tensor-core distances + exact FP32 re-rank.
//
// For a reference block a and a candidate b (8 x 8 patches) with block means
// ma, mb and zero-mean residuals a' = a - ma, b' = b - mb,
//   ||a - b||^2 = 64 (ma - mb)^2 + ||a'||^2 + ||b'||^2 - 2 a'.b'
// (the residuals are orthogonal to the constant block).  ||a'||^2 is the same
// for every candidate of a reference, so the candidates are ranked by
// 64 (ma - mb)^2 + ||b'||^2 - 2 a'.b', where a'.b' is a bf16 x bf16 product
// accumulated in fp32 on the tensor cores (tcgen05.mma, accumulator in TMEM)
// and the other terms are fp32.  Removing each block's mean before the bf16
// rounding keeps the operands at the scale of the noise and texture, not of
// the grey level, which is what bounds the rounding error of a'.b'.  The 2K best by that approximate distance
// are then re-ranked by the exact FP32 sum of squared differences of the plain
// matcher (same operation order), and the K best by (exact distance, window
// index) are kept, so the match set equals the plain one whenever the true K
// best are among the approximate 2K best.
//
// Tile: 128 references = 8 reference rows x 16 reference columns (one per TMEM
// lane / thread).  Their search windows cover a PR x PC grid of candidate
// positions (PR = 7s + D2, PC = 15s + D2); the GEMM is A (128 refs x 64) times
// B^T (positions x 64), in chunks of 128 positions double-buffered in shared
// memory and in two TMEM accumulators of 128 columns, so the next chunk's MMA
// runs while the current one is read out.  Each thread keeps the 2K smallest
// approximate distances of its own window in a max-heap in shared memory: a
// position is tested against the heap's root with one compare, and the rare
// candidates that beat it are inserted in batches of 32 positions, so the
// warp's lanes diverge only in the short sift-down loop.
#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace gbm3d {

namespace {

constexpr int TD = 8;            // patch side (K dimension 64)
constexpr int TKD = TD * TD;     // 64
constexpr int TI = 8, TJ = 16;   // references per tile (rows x columns)
constexpr int NC = 128;          // positions per chunk (MMA N)
constexpr int CAND = 32;         // approximate candidates kept per reference (2K, K <= 16)
constexpr long long WAIT_CYCLES = 4000000000LL;  // ~2 s at 2 GHz

struct TcGeom {
  int PR, PC, NP;   // candidate-position grid of a tile
  int CH, CW;       // region (fp32 image) rows (padded even) and columns
  size_t off_img32, off_nb2, off_bm, off_A, off_B, off_heap, off_misc, bytes;
};

__host__ __device__ inline TcGeom tc_geom(int s, int d2) {
  TcGeom g;
  g.PR = s * (TI - 1) + d2;
  g.PC = s * (TJ - 1) + d2;
  g.NP = g.PR * g.PC;
  g.CH = (g.PR + TD - 1 + 1) & ~1;
  g.CW = g.PC + TD - 1;
  size_t o = 0;
  auto take = [&](size_t bytes, size_t align) {
    o = (o + align - 1) / align * align;
    const size_t at = o;
    o += bytes;
    return at;
  };
  g.off_A = take((size_t)128 * TKD * 2, 1024);
  g.off_B = take((size_t)2 * NC * TKD * 2, 1024);
  g.off_img32 = take((size_t)g.CH * g.CW * 4, 16);
  g.off_nb2 = take((size_t)2 * NC * 4, 16);             // ||b'||^2 of the two chunks in flight
  g.off_bm = take((size_t)2 * NC * 4, 16);              // block means of the two chunks in flight
  g.off_heap = take((size_t)2 * CAND * 128 * 4, 16);    // per-thread heaps: values, then positions
  g.off_misc = take(64, 16);
  g.bytes = o;
  return g;
}

template <int D2>
__global__ void __launch_bounds__(128) k_match_tc(MatchArgs A) {
  constexpr int H = D2 / 2;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int s = A.s;
  const TcGeom G = tc_geom(s, D2);
  float* img32 = reinterpret_cast<float*>(smem + G.off_img32);        // column-major CH x CW
  float* nb2 = reinterpret_cast<float*>(smem + G.off_nb2);            // ||b'||^2, chunk buffer b at b*NC
  float* bmean = reinterpret_cast<float*>(smem + G.off_bm);           // block means, same layout
  float* hv = reinterpret_cast<float*>(smem + G.off_heap);            // heap node q of thread t at q*128+t
  int* hp = reinterpret_cast<int*>(hv + CAND * 128);
  unsigned char* sA = smem + G.off_A;
  unsigned char* sB = smem + G.off_B;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + G.off_misc);    // [2]
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(mbar + 2);
  int* fail_s = reinterpret_cast<int*>(taddr_s + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles_i = (A.M + TI - 1) / TI;
  const int ti = blockIdx.x % tiles_i, tj = blockIdx.x / tiles_i;
  const int i0 = ti * TI, j0 = tj * TJ;
  // this thread's reference (TMEM lane tid): li fast
  const int li = tid % TI, lj = tid / TI;
  const int ri = i0 + li, rj = j0 + lj;
  const bool valid = ri < A.M && rj < A.N;

  if (warp == 0) tc::tmem_alloc(taddr_s, 2 * NC);
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
    tc::fence_mbar_init();
    *fail_s = 0;
  }

  // ---- region of the padded search image: pad rows i0*s .., cols j0*s .. ----
  const int R = A.m + D2, Q = A.n + D2;  // padded search-image extent
  const int y0 = i0 * s, x0 = j0 * s;
  for (int e = tid; e < G.CH * G.CW; e += 128) {
    const int y = e % G.CH, x = e / G.CH;
    float v = 0.f;
    if (y0 + y < R && x0 + x < Q && y < G.PR + TD - 1) v = A.pad[(size_t)(y0 + y) + (size_t)(x0 + x) * A.P];
    img32[e] = v;
  }
  __syncthreads();
  const int NPc = (G.NP + NC - 1) / NC * NC;
  // mean of the 8 x 8 block at (y, x) of the staged region
  auto block_mean = [&](int y, int x) -> float {
    float sum = 0.f;
#pragma unroll
    for (int cc = 0; cc < TD; ++cc)
#pragma unroll
      for (int r = 0; r < TD; ++r) sum += img32[(y + r) + (x + cc) * G.CH];
    return sum * (1.f / TKD);
  };
  // ---- A: this thread's reference block (at window offset (H, H)) ------------
  float amean;
  {
    const int ry = s * li + H, rx = s * lj + H;
    amean = block_mean(ry, rx);
    auto bf = [&](float x) -> uint32_t { return tc::bf16_bits(x - amean); };
#pragma unroll
    for (int r = 0; r < TD; ++r) {
      uint32_t w[4];
#pragma unroll
      for (int c = 0; c < TD; c += 2)
        w[c / 2] = bf(img32[(ry + r) + (rx + c) * G.CH]) | (bf(img32[(ry + r) + (rx + c + 1) * G.CH]) << 16);
      *reinterpret_cast<uint4*>(sA + tc::kmajor_offset(tid, r * TD, TKD)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
  // B chunk: thread t builds the row of position chunk*NC + t (k = r*8 + c):
  // the block's mean, its zero-mean residual in bf16 and the residual's
  // squared norm ||b'||^2 in fp32 (all 0 past the grid)
  auto build_B = [&](int chunk, int buf) {
    const int p = chunk * NC + tid;
    unsigned char* base = sB + (size_t)buf * NC * TKD * 2;
    const int pr = p % G.PR, pc = p / G.PR;
    const bool in = p < G.NP;
    const float mean = in ? block_mean(pr, pc) : 0.f;
    float acc = 0.f;
#pragma unroll
    for (int r = 0; r < TD; ++r) {
      uint32_t w[4];
#pragma unroll
      for (int c = 0; c < TD; c += 2) {
        uint32_t lo = 0, hi = 0;
        if (in) {
          const float x0v = img32[(pr + r) + (pc + c) * G.CH] - mean;
          const float x1v = img32[(pr + r) + (pc + c + 1) * G.CH] - mean;
          acc = fmaf(x0v, x0v, acc);
          acc = fmaf(x1v, x1v, acc);
          lo = tc::bf16_bits(x0v);
          hi = tc::bf16_bits(x1v);
        }
        w[c / 2] = lo | (hi << 16);
      }
      *reinterpret_cast<uint4*>(base + tc::kmajor_offset(tid, r * TD, TKD)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    nb2[buf * NC + tid] = acc;
    bmean[buf * NC + tid] = mean;
  };
  const int nch = NPc / NC;
  // chunks are visited from the middle of the position grid outwards: positions
  // near the windows' centres tend to match best, so the heap thresholds drop
  // early and few later positions need inserting.  Buffers follow the visit order.
  const int mid = nch / 2;
  auto chunk_of = [&](int k) { return k == 0 ? mid : ((k & 1) ? mid - (k + 1) / 2 : mid + k / 2); };
  build_B(chunk_of(0), 0);
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *taddr_s;
  constexpr uint32_t idesc = tc::idesc_bf16_f32(128, NC);
  auto issue = [&](int chunk) {  // chunk: position in the visit order (selects the buffers)
    const uint32_t a0 = tc::smem_u32(sA);
    const uint32_t b0 = tc::smem_u32(sB + (size_t)(chunk & 1) * NC * TKD * 2);
#pragma unroll
    for (int ks = 0; ks < TKD / 16; ++ks)
      tc::mma_bf16(tmem + (uint32_t)((chunk & 1) * NC), tc::desc_kmajor(a0 + ks * 256, 128, TKD * 16),
                   tc::desc_kmajor(b0 + ks * 256, 128, TKD * 16), idesc, ks > 0);
    tc::commit(&mbar[chunk & 1]);
  };
  if (tid == 0) issue(0);

  // running 2K smallest approximate distances of this thread's window: a
  // max-heap (root = the largest kept = the admission threshold)
#pragma unroll
  for (int q = 0; q < CAND; ++q) {
    hv[q * 128 + tid] = 3.0e38f;
    hp[q * 128 + tid] = -1;
  }
  float thr = 3.0e38f;
  const int wr0 = s * li, wc0 = s * lj;  // window origin in position coordinates
  // columns of position space any reference of this warp can use
  const int wpc_lo = s * (warp * 32 / TI), wpc_hi = s * (warp * 32 / TI + 32 / TI - 1) + D2 - 1;

  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) build_B(chunk_of(c + 1), (c + 1) & 1);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (*fail_s) break;
    if (tid == 0 && c + 1 < nch) issue(c + 1);
    const bool ok = tc::mbar_wait(&mbar[c & 1], (uint32_t)((c >> 1) & 1), WAIT_CYCLES);
    if (!ok) *fail_s = 1;
    tc::fence_after_sync();
    const int p0 = chunk_of(c) * NC;
    const int pc_first = p0 / G.PR, pc_last = (p0 + NC - 1) / G.PR;
    if (ok && pc_last >= wpc_lo && pc_first <= wpc_hi) {  // warp-uniform skip of chunks outside every window
      const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((c & 1) * NC);
#pragma unroll 1
      for (int q0 = 0; q0 < NC; q0 += 32) {
        // positions P0 .. P0+31: rows r0.. of column c0, then (after a wrap) rows 0.. of c0+1
        const int P0 = p0 + q0, r0 = P0 % G.PR, c0 = P0 / G.PR;
        const int L1 = min(32, G.PR - r0);
        auto bits = [](int lo, int hi) -> uint32_t {
          if (hi <= lo) return 0u;
          const int n = hi - lo;
          return (n >= 32 ? 0xffffffffu : ((1u << n) - 1u)) << lo;
        };
        uint32_t inm = 0;
        if ((unsigned)(c0 - wc0) < (unsigned)D2) inm |= bits(max(0, wr0 - r0), min(L1, wr0 + D2 - r0));
        if ((unsigned)(c0 + 1 - wc0) < (unsigned)D2) inm |= bits(L1 + wr0, min(32, L1 + wr0 + D2));
        if (!__any_sync(0xffffffffu, inm != 0)) continue;  // no reference of this warp sees these positions
        float v[32];
        tc::tmem_ld32(lane_base + q0, v);
        uint32_t qm = 0;
#pragma unroll
        for (int u = 0; u < 32; ++u) {
          const float dm = amean - bmean[(c & 1) * NC + q0 + u];
          v[u] = fmaf(-2.f, v[u], nb2[(c & 1) * NC + q0 + u]);  // approximate distance (less ||a'||^2)
          v[u] = fmaf((float)TKD * dm, dm, v[u]);
          qm |= (v[u] < thr ? 1u : 0u) << u;
        }
        qm &= inm;
        // insert the qualifying positions one at a time (lanes with none idle)
        while (__any_sync(0xffffffffu, qm != 0)) {
          if (qm) {
            const int u = __ffs(qm) - 1;
            qm &= qm - 1;
            float d = v[0];
#pragma unroll
            for (int k = 1; k < 32; ++k) d = (u == k) ? v[k] : d;
            if (d < thr) {  // replace the root, sift down
              int q = 0;
              while (true) {
                int ch = 2 * q + 1;
                if (ch >= CAND) break;
                float cv = hv[ch * 128 + tid];
                if (ch + 1 < CAND) {
                  const float cv2 = hv[(ch + 1) * 128 + tid];
                  if (cv2 > cv) {
                    cv = cv2;
                    ++ch;
                  }
                }
                if (cv <= d) break;
                hv[q * 128 + tid] = cv;
                hp[q * 128 + tid] = hp[ch * 128 + tid];
                q = ch;
              }
              hv[q * 128 + tid] = d;
              hp[q * 128 + tid] = P0 + u;
              thr = hv[tid];
            }
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  const bool failed = *fail_s != 0;
  if (failed && tid == 0 && A.err) atomicOr(A.err, 2);

  // ---- exact FP32 re-rank (the plain matcher's operation order) ----------------
  // The operand buffers are free now: exact keys and the selection go to
  // shared memory (element q of thread t at q * 128 + t) beside the heap.
  const int* cpS = hp;
  uint32_t* keyS = reinterpret_cast<uint32_t*>(sB);
  uint32_t* selS = reinterpret_cast<uint32_t*>(sA);
  if (valid && !failed) {
    const int ry = s * li + H, rx = s * lj + H;
    float xr[TKD];
#pragma unroll
    for (int r = 0; r < TD; ++r)
#pragma unroll
      for (int cc = 0; cc < TD; ++cc) xr[r * TD + cc] = img32[(ry + r) + (rx + cc) * G.CH];
#pragma unroll 1
    for (int q = 0; q < CAND; ++q) {
      const int p = cpS[q * 128 + tid];
      uint32_t key = 0xffffffffu;
      if (p >= 0) {
        const int pr = p % G.PR, pc = p / G.PR;
        const float* cand = img32 + pr + pc * G.CH;
        float acc = 0.f;
#pragma unroll
        for (int r = 0; r < TD; ++r)
#pragma unroll
          for (int cc = 0; cc < TD; ++cc) {
            const float t = xr[r * TD + cc] - cand[r + cc * G.CH];
            acc = fmaf(t, t, acc);
          }
        key = __float_as_uint(acc);
      }
      keyS[q * 128 + tid] = key;
    }
    const int K = A.K;
    for (int k = 0; k < K; ++k) selS[k * 128 + tid] = 0;
    // rank by (exact distance bits, column-major window index), ascending
#pragma unroll 1
    for (int q = 0; q < CAND; ++q) {
      const int p = cpS[q * 128 + tid];
      if (p < 0) continue;
      const uint32_t kq = keyS[q * 128 + tid];
      const uint32_t iq = (uint32_t)((p % G.PR - wr0) + (p / G.PR - wc0) * D2);
      int rank = 0;
#pragma unroll 4
      for (int t = 0; t < CAND; ++t) {
        const int pt = cpS[t * 128 + tid];
        const uint32_t kt = keyS[t * 128 + tid];
        const uint32_t it = pt < 0 ? 0xffffffffu : (uint32_t)((pt % G.PR - wr0) + (pt / G.PR - wc0) * D2);
        rank += (kt < kq || (kt == kq && it < iq)) ? 1 : 0;
      }
      if (rank < K) selS[rank * 128 + tid] = iq + 1;
    }
    selS[tid] = (uint32_t)(H + H * D2 + 1);  // S(1) is the reference itself (matchBlocksCPU.m:103)
    const int g = ri + A.M * rj;
    uint32_t* Sg = A.S + (size_t)g * K;
    for (int k = 0; k < K; ++k) Sg[k] = selS[k * 128 + tid];
    if (A.cnt) A.cnt[g] = K;
    if (A.volume) {  // tile-space (or image-shaped when s = d) gather, matchBlocksCPU.m:107-114
      const size_t mn = (size_t)A.m * A.n;
      for (int k = 0; k < K; ++k) {
        int e = (int)selS[k * 128 + tid] - 1;
        if ((unsigned)e >= (unsigned)(D2 * D2)) e = H + H * D2;
        const int py = wr0 + e % D2, px = wc0 + e / D2;
#pragma unroll
        for (int cc = 0; cc < TD; ++cc) {
          float* dst = A.volume + (size_t)(ri * TD) + (size_t)A.m * (rj * TD + cc) + mn * k;
          const float* src = img32 + py + (px + cc) * G.CH;
          *reinterpret_cast<float4*>(dst) = make_float4(src[0], src[1], src[2], src[3]);
          *reinterpret_cast<float4*>(dst + 4) = make_float4(src[4], src[5], src[6], src[7]);
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 2 * NC);
}

template <int D2>
cudaError_t launch_tc_t(const MatchArgs& A, cudaStream_t st) {
  const TcGeom G = tc_geom(A.s, D2);
  cudaError_t e = cudaFuncSetAttribute(k_match_tc<D2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G.bytes);
  if (e != cudaSuccess) return e;
  const int tiles = ((A.M + TI - 1) / TI) * ((A.N + TJ - 1) / TJ);
  k_match_tc<D2><<<tiles, 128, G.bytes, st>>>(A);
  return cudaGetLastError();
}

}  // namespace

bool match_tc_supported(int d, int d2, int s, int K, bool tol_branch) {
  if (d != TD || K < 1 || K > 16 || tol_branch || s < 1 || s > 4) return false;
  if (d2 != 16 && d2 != 24 && d2 != 32) return false;
  return tc_geom(s, d2).bytes <= 113 * 1024;  // two CTAs (and two 256-column TMEM allocations) per SM
}

cudaError_t launch_match_tc(int d, int d2, const MatchArgs& A, cudaStream_t st) {
  if (!match_tc_supported(d, d2, A.s, A.K, A.tol_branch != 0)) return cudaErrorInvalidValue;
  // the volume is written as float4 pairs: its row count must keep 16-byte alignment
  if (A.volume && (A.m % 4 != 0)) return cudaErrorInvalidValue;
  if (d2 == 32) return launch_tc_t<32>(A, st);
  if (d2 == 24) return launch_tc_t<24>(A, st);
  return launch_tc_t<16>(A, st);
}

}  // namespace gbm3d
