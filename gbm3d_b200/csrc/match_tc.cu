// Block matching on the tensor cores — the search of matchBlocksCPU.m:21-116
// (and of matchBlocksWie.m:21-92), with the distances of
// matchBlocksCPU.m:82-85, ||x - y||^2 = ||x||^2 + ||y||^2 - 2<x,y>, where the
// <x,y> term is a 16-bit GEMM (bf16 for the precision form, f16 for the tensor
// form) with fp32 accumulation on tcgen05, used to bound the candidates; the
// exact FP32 sums of squared differences then rank them in the exhaustive
// matcher's operation order, so the match sets are that matcher's own.
//
// Tile: 4 x 4 references (MMA N = 16) at stride s.  Their search windows
// cover a PR x PR grid of candidate positions, PR = 3 s + d2 <= 56, whose 8 x 8
// blocks lie in a 64 x 68 region of the search image, loaded by one TMA copy
// (the tensor map covers this GPU's search image; no multicast).  Centring
// every value on the region mean m0 (x' = x - m0), the positions are the MMA's
// A operand without an im2col copy: E(y, x) holds the 8 values x'(y, x..x+7)
// (16 bytes), stored row-major with 64 entries per row, so the A rows of a
// chunk of 128 positions (2 position rows of 64) are 128 consecutive entries
// and the K = 16 slice of block rows r, r+1 is the same array read from r rows
// further on (descriptor start + r * 1024 bytes, leading byte offset 1024
// between the two rows, stride byte offset 128 between 8-position groups).
// Four MMAs (r = 0, 2, 4, 6) give <x'_p, a_j> for all 128 positions p of a
// chunk and the 16 references j, accumulated in TMEM on top of a value per
// (p, j) written there first (below).  All chunks of a tile (at most 28 x 16
// fp32 columns) stay in TMEM.  TMEM column 16 c + 4 li + lj of chunk c holds
// reference (li, lj) (row li, column lj of the tile), so that the four
// references of one tile row are adjacent.
//
// The reference operand is centred on its own block mean as well (a_z = a -
// m0 - ma, a_z.1 = 0), which keeps the rounding error proportional to ||a_z||
// (noise and texture) instead of the grey level; then
//     D(p, j) = ||a_z||^2 + 64 ma^2 - 2 v(p, j),
//     v(p, j) = <x'_p, a_z> + ma sum(x'_p) - ||x'_p||^2 / 2,
// and the last two terms are what TMEM holds before the MMAs add the first.
// Only the order of v within one reference matters, so the per-reference
// constant is left out.
//
// Selection, per reference j: pass 1 takes the best v of every window column
// and row parity (64 groups of 16 positions at matchSize 32; TMEM lane =
// position, so a lane's column and parity are fixed); T = the K-th best of
// those group bests, so at least K positions have v >= T.  With
// |v - v_exact| <= k ||x'_p|| (16-bit rounding of both operands, fp32
// accumulation: k ~ 2u ||a_z||, u = 2^-9 for bf16, 2^-11 for f16), every
// position of the exact top K has
//     v + k ||x'_p|| >= T - k max_window ||x'|| - h
// (h bounds the FP32 rounding of the position sums and of the accumulation);
// pass 2 lists exactly those positions.  The listed candidates are re-ranked
// by the exact FP32 SSD (t = x - y, acc = fmaf(t, t, acc), row-major over the
// block, as the exhaustive matcher adds) and the K best by (distance,
// column-major window index) are kept, S(1) forced to the reference
// (matchBlocksCPU.m:103).  A reference with more than 64 candidates is appended
// to a global list that the exhaustive matcher finishes.
//
// Schedule: one persistent CTA of 16 warps per SM takes tiles from a device
// work queue.  Per tile t: tables, E and the reference operand; TMEM
// initialisation and the 112 MMAs (lane 0 of 8 warps issues, one commit each); while they
// run, the exact re-rank of tile t-1; then pass 1, thresholds and pass 2.  The
// region of tile t+2 is loaded by TMA meanwhile (three region buffers).
//
// Every wait (TMA, MMA) gives up after a bounded number of SM clocks (about
// two seconds unless the caller sets fewer), sets bit 1 of the status word
// and ends the CTA's work, after letting its own copies and MMAs in flight
// land with the full limit; TMEM is always released.
#include <cuda.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace gbm3d {

namespace {

typedef unsigned long long u64;

constexpr int TD = 8;           // patch side
constexpr int TT = 4;           // references per tile side
constexpr int NREF = TT * TT;   // 16 = MMA N
constexpr int XW = 64;          // position columns per E row
constexpr int PRMAX = 56;       // largest position grid side, 3 * 8 + 32
constexpr int RP = 68;          // region rows (TMA box, inner) = pitch in floats
constexpr int RC = 64;          // region columns (TMA box)
constexpr int CAP = 64;         // candidate list capacity per reference: a longer list goes
                                // to the exhaustive matcher (a tile waits for its slowest
                                // re-rank, so long lists are cheaper there)
constexpr int NT = 512;         // threads: 16 warps
constexpr int NB2P = 65;        // pitch of the position tables (bank-conflict free both ways)
constexpr int NRB = 3;          // region buffers (TMA two tiles ahead)
constexpr int RBYTES = RP * RC * 4;
constexpr long long WAIT_CYCLES = 4000000000LL;  // ~2 s at 2 GHz
constexpr int NISS = 8;         // warps whose lane 0 issues MMAs (chunks c = w, w + 8, ...), one commit each

constexpr int OFF_REG = 0;                                   // NRB regions of RP x RC floats, column-major
constexpr int OFF_E = 52224;                                 // 64 x 64 entries of 16 bytes (1024-aligned)
constexpr int OFF_B = OFF_E + 64 * XW * 16;                  // reference operand: 16 x 64 16-bit values
constexpr int TBL = 64 * NB2P * 4;                           // one [px * NB2P + py] table
constexpr int OFF_NB2 = OFF_B + NREF * 64 * 2;               // ||x'_p||^2
constexpr int OFF_NBS = OFF_NB2 + TBL;                       // ||x'_p||
constexpr int OFF_SB = OFF_NBS + TBL;                        // sum(x'_p)
constexpr int OFF_CB = OFF_SB + TBL;                         // group bests [ref][parity][64]; later S rows
constexpr int OFF_LST = OFF_CB + NREF * 2 * 64 * 4;          // candidate lists [ref][CAP]
constexpr int OFF_MISC = OFF_LST + NREF * CAP * 4;
constexpr int SMEM_BYTES = OFF_MISC + 1024;
static_assert(NRB * RBYTES <= OFF_E && OFF_E % 1024 == 0 && OFF_B % 128 == 0, "operand alignment");
static_assert(2 * 64 * NB2P * 4 <= 64 * XW * 16, "column sums fit in the E area");
static_assert(SMEM_BYTES <= 227 * 1024, "shared memory");

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Bitonic sort of one value per lane, ascending by lane.
template <class T>
__device__ __forceinline__ T warp_sort_asc(T v, int lane) {
#pragma unroll
  for (int k2 = 2; k2 <= 32; k2 <<= 1)
#pragma unroll
    for (int j2 = k2 >> 1; j2 > 0; j2 >>= 1) {
      const T o = __shfl_xor_sync(0xffffffffu, v, j2);
      const bool up = (lane & k2) == 0, lower = (lane & j2) == 0;
      v = (lower == up) ? (o < v ? o : v) : (o < v ? v : o);
    }
  return v;
}

template <bool HALF>
__device__ __forceinline__ uint32_t pack_op(float lo, float hi) {
  return HALF ? tc::f16x2_bits(lo, hi) : tc::bf16x2_bits(lo, hi);
}

// Per-position error factor of v for a reference with ||a_z|| = na:
// |v - v_exact| <= k ||x'_p|| with k = (2u + u^2 + 2^-14) na (operand rounding,
// u = 2^-9 for bf16, 2^-11 for f16; fp32 accumulation), rounded up.
template <bool HALF>
__device__ __forceinline__ float err_factor(float na) {
  return (HALF ? 1.05f / 1024.f : 1.05f / 256.f) * na;
}

// Bound on the FP32 rounding not covered by k ||x'_p||, in units of v, for a
// reference with ||a - m0||^2 = nat2, window maximum ||x'||^2 = nbw2 and tile
// maximum nbt.  Every addend of v, of the table sums and of the exact SSD is
// bounded by nat2 + nbw2 (|ma sum(x'_p)| <= (64 ma^2 + ||x'_p||^2) / 2 and
// ||x'_p|| ||a_z|| <= (||x'_p||^2 + ||a_z||^2) / 2), and each is rounded at most
// ~70 times at 2^-24: about 2^-17.4 (nat2 + nbw2) per value, counted twice
// (the K positions behind T and the candidate) plus the exact SSD's own
// 2^-18 D, covered by 2^-14.  The running sums of the position tables start
// up to 6 rows or columns outside the window, so their rounding is bounded by
// the tile maximum instead (about 2^-19.4 nbt; 2^-17 is taken).  All terms are
// relative: on a smooth image the bound shrinks with the distances it separates.
__device__ __forceinline__ float fp32_slack(float nat2, float nbw2, float nbt) {
  return (nat2 + nbw2) * (1.f / 16384.f) + nbt * (1.f / 131072.f) + (1.f / 64.f);
}

template <int D2, bool HALF>
__global__ void __launch_bounds__(NT, 1) k_match_tc(const __grid_constant__ CUtensorMap tmap, MatchArgs A) {
  constexpr int H = D2 / 2;
  constexpr int NC = D2 / 2;  // chunks of one reference's window rows of one parity
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* E = smem + OFF_E;
  unsigned char* Bq = smem + OFF_B;
  float* nb2 = reinterpret_cast<float*>(smem + OFF_NB2);
  float* nbs = reinterpret_cast<float*>(smem + OFF_NBS);
  float* sbt = reinterpret_cast<float*>(smem + OFF_SB);
  float* cb = reinterpret_cast<float*>(smem + OFF_CB);
  uint32_t* lst = reinterpret_cast<uint32_t*>(smem + OFF_LST);
  int* cnt = reinterpret_cast<int*>(smem + OFF_MISC);   // [16] list lengths
  float* thr = reinterpret_cast<float*>(cnt + 16);      // [16] pass-2 thresholds
  float* kf = thr + 16;                                 // [16] error factors k
  float* rma = kf + 16;                                 // [16] reference means ma, by TMEM column
  float* red = rma + 16;                                // [32] reductions
  uint64_t* mbar = reinterpret_cast<uint64_t*>(red + 32);  // [NRB] TMA, [1] MMA, [1] wait probe
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(mbar + NRB + 2);
  int* fail_s = reinterpret_cast<int*>(taddr_s + 1);
  int* tq = fail_s + 1;                                  // [NRB] tile of each region buffer (-1: none)
  int* nbt_s = tq + NRB;                                 // tile maximum of ||x'_p||^2 (float bits)

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned FULL = 0xffffffffu;
  const int s = A.s;
  const int PR = 3 * s + D2;      // position grid side
  const int VR = PR + TD - 1;     // region side the blocks touch
  const int NCH = (PR + 1) / 2;   // chunks of 2 position rows
  const int tiles_i = (A.M + TT - 1) / TT;
  const int ntiles = tiles_i * ((A.N + TT - 1) / TT);
  const long long wait = A.wait_cycles > 0 ? A.wait_cycles : WAIT_CYCLES;  // < 0: a probe, below
  // tiles come from a device work queue (A.work, zeroed before the launch):
  // each CTA takes the next tile when it prefetches its region
  auto tile_of = [&](int it) { return tq[it % NRB]; };
  auto region = [&](int it) { return reinterpret_cast<float*>(smem + OFF_REG + (it % NRB) * RBYTES); };

  if (warp == 0) tc::tmem_alloc(taddr_s, 512);
  if (tid == 0) {
    for (int b = 0; b < NRB; ++b) tc::mbar_init(&mbar[b], 1);
    tc::mbar_init(&mbar[NRB], NISS);
    tc::mbar_init(&mbar[NRB + 1], 1);  // never arrives: the wait probe
    tc::fence_mbar_init();
    *fail_s = 0;
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *taddr_s;
  uint32_t tma_phase = 0;    // bit b: parity of region buffer b's next completion
  uint32_t tma_pending = 0;  // bit b: a load into region buffer b is in flight
  uint32_t mma_phase = 0;
  bool mma_pending = false;
  auto issue_tma = [&](int it) {  // one thread takes the next tile, if any, and loads its region
    const int t = atomicAdd(A.work, 1);
    tq[it % NRB] = t < ntiles ? t : -1;
    if (t >= ntiles) return;
    const int i0 = (t % tiles_i) * TT, j0 = (t / tiles_i) * TT;
    tc::mbar_expect_tx(&mbar[it % NRB], RBYTES);
    tc::tma_load_2d(region(it), &tmap, i0 * s, j0 * s, &mbar[it % NRB]);
  };
  if (tid == 0) {
    issue_tma(0);
    issue_tma(1);
  }
  __syncthreads();
  for (int b = 0; b < 2; ++b)
    if (tq[b] >= 0) tma_pending |= 1u << b;

  // ---- exact re-rank of the tile of iteration `it` (warp j: reference j) -------
  auto rerank = [&](int it) {
    const float* reg = region(it);
    const int t = tile_of(it);
    const int i0 = (t % tiles_i) * TT, j0 = (t / tiles_i) * TT;
    const int j = warp, li = j & 3, lj = j >> 2;
    const int ri = i0 + li, rj = j0 + lj;
    if (ri >= A.M || rj >= A.N) return;
    const int g = ri + A.M * rj;
    const int C = cnt[j];
    const int K = A.K;
    const uint32_t center = (uint32_t)(H + H * D2 + 1);
    uint32_t* Sg = A.S + (size_t)g * K;
    uint32_t* sel = reinterpret_cast<uint32_t*>(cb) + j * 32;  // the group bests are no longer needed
    if (lane == 0 && A.cand_hist) atomicAdd(&A.cand_hist[min(C >> 3, 32)], 1);
    if (C > CAP) {
      if (lane == 0) A.ovf_list[atomicAdd(A.ovf_count, 1)] = g;
      return;
    }
    const int wy = s * li, wx = s * lj;  // window origin in position coordinates
    const float* xref = reg + (wx + H) * RP + wy + H;
    float xr[TD * TD];
#pragma unroll
    for (int r = 0; r < TD; ++r)
#pragma unroll
      for (int c = 0; c < TD; ++c) xr[r * TD + c] = xref[r + c * RP];
    auto exact_key = [&](int e) -> u64 {
      const uint32_t pos = lst[j * CAP + e];
      const int py = (int)(pos >> 6), pxx = (int)(pos & 63);
      const float* cand = reg + pxx * RP + py;
      float acc = 0.f;
#pragma unroll
      for (int h2 = 0; h2 < 2; ++h2) {  // block rows 4 h2 .. 4 h2 + 3: 32 loads in flight, then their sums
        float cv[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) cv[q] = cand[(4 * h2 + (q >> 3)) + (q & 7) * RP];
#pragma unroll
        for (int q = 0; q < 32; ++q) {  // element (r, c) = (4 h2 + q / 8, q % 8): row-major order
          const float tt = xr[32 * h2 + q] - cv[q];
          acc = fmaf(tt, tt, acc);
        }
      }
      const uint32_t ix = (uint32_t)((py - wy) + (pxx - wx) * D2);
      return ((u64)__float_as_uint(acc) << 32) | ix;
    };
    // keys (distance bits, window index) are distinct: a key's rank is the
    // number of keys below it (independent broadcasts, no sorting network)
    if (C <= 32) {
      const u64 k0 = lane < C ? exact_key(lane) : ~0ull;
      int r0 = 0;
#pragma unroll
      for (int i = 0; i < 32; ++i) r0 += __shfl_sync(FULL, k0, i) < k0 ? 1 : 0;
      if (lane < C && r0 < K) sel[r0] = r0 == 0 ? center : (uint32_t)k0 + 1u;
    } else {  // C <= CAP = 64: two keys per lane
      const u64 k0 = exact_key(lane);
      const u64 k1 = lane + 32 < C ? exact_key(lane + 32) : ~0ull;
      int r0 = 0, r1 = 0;
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const u64 o0 = __shfl_sync(FULL, k0, i), o1 = __shfl_sync(FULL, k1, i);
        r0 += (o0 < k0 ? 1 : 0) + (o1 < k0 ? 1 : 0);
        r1 += (o0 < k1 ? 1 : 0) + (o1 < k1 ? 1 : 0);
      }
      if (r0 < K) sel[r0] = r0 == 0 ? center : (uint32_t)k0 + 1u;
      if (lane + 32 < C && r1 < K) sel[r1] = r1 == 0 ? center : (uint32_t)k1 + 1u;
    }
    __syncwarp();
    if (lane < K) Sg[lane] = sel[lane];
    if (lane == 0 && A.cnt) A.cnt[g] = K;
    if (A.volume) {  // matchBlocksCPU.m:107-114 (tile-space when s != d)
      const size_t mn = (size_t)A.m * A.n;
      for (int k = 0; k < K; ++k) {
        int e = (int)sel[k] - 1;
        if ((unsigned)e >= (unsigned)(D2 * D2)) e = H + H * D2;
        const int a = e % D2, b = e / D2;
        const float* src = reg + (wx + b) * RP + wy + a;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int q = lane + 32 * u, r = q & 7, c = q >> 3;
          A.volume[(size_t)(ri * TD + r) + (size_t)A.m * (rj * TD + c) + mn * k] = src[r + c * RP];
        }
      }
    }
  };

  int it = 0;
  for (;; ++it) {
    if (tq[it % NRB] < 0) break;  // the queue is empty (uniform: written before a barrier)
    const float* reg = region(it);
    // a negative limit asks for one wait on a barrier that nothing completes
    // (the test of the give-up path): it runs out after |limit| clocks
    if (it == 0 && A.wait_cycles < 0 && !tc::mbar_wait(&mbar[NRB + 1], 0, -A.wait_cycles)) *fail_s = 1;
    // ---- the region of tile `it` has arrived ----------------------------------
    if (tc::mbar_wait(&mbar[it % NRB], (tma_phase >> (it % NRB)) & 1u, wait)) {
      tma_phase ^= 1u << (it % NRB);
      tma_pending &= ~(1u << (it % NRB));
    } else {
      *fail_s = 1;
    }
    __syncthreads();
    tc::fence_after_sync();  // the previous tile's TMEM reads are ordered before this tile's TMEM writes
    if (*fail_s) break;
    // centre m0: mean of the region the blocks touch (every warp adds the 16
    // warp sums itself, in the same order, so all threads hold the same m0)
    {
      float sum = 0.f;
      for (int x = warp; x < VR; x += NT / 32)
        for (int y = lane; y < VR; y += 32) sum += reg[x * RP + y];
      sum = warp_sum(sum);
      if (lane == 0) red[warp] = sum;
      if (tid == 0) *nbt_s = 0;
    }
    __syncthreads();
    float m0 = 0.f;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) m0 += red[w];
    m0 = m0 / (float)(VR * VR);
    // per position: ||x'||^2, ||x'|| and sum(x') as running sums, first over 8
    // rows (kept in the E area until E is built; the MMAs of the previous tile
    // are complete), then over 8 columns
    {
      float* cs = reinterpret_cast<float*>(E);   // [py * NB2P + x] sums of squares over rows py .. py+7
      float* cl = cs + 64 * NB2P;                // [py * NB2P + x] sums
      {
        // thread: column x, rows 7 sg .. 7 sg + 6
        const int x = tid & 63, sg = tid >> 6;
        const int y0 = 7 * sg;
        if (x < VR && y0 < PR) {
          const float* col = reg + x * RP + y0;
          float t[TD];
          float a = 0.f, l = 0.f;
#pragma unroll
          for (int r = 0; r < TD; ++r) {
            t[r] = col[r] - m0;
            a = fmaf(t[r], t[r], a);
            l += t[r];
          }
          cs[y0 * NB2P + x] = a;
          cl[y0 * NB2P + x] = l;
#pragma unroll
          for (int u = 1; u < 7; ++u) {
            const int y = y0 + u;
            if (y < PR) {
              const float tn = col[u + TD - 1] - m0, to = t[u - 1];
              a = fmaf(tn, tn, a) - to * to;
              l = (l + tn) - to;
              t[(u + TD - 1) & 7] = tn;  // t[u - 1] is not needed again
              cs[y * NB2P + x] = a;
              cl[y * NB2P + x] = l;
            }
          }
        }
      }
      __syncthreads();
      {
        // thread: row py, columns 7 sg .. 7 sg + 6
        const int py = tid & 63, sg = tid >> 6;
        const int x0 = 7 * sg;
        float amax = 0.f;
        if (py < PR && x0 < PR) {
          float qa[TD], ql[TD];
          float a = 0.f, l = 0.f;
#pragma unroll
          for (int c = 0; c < TD; ++c) {
            qa[c] = cs[py * NB2P + x0 + c];
            ql[c] = cl[py * NB2P + x0 + c];
            a += qa[c];
            l += ql[c];
          }
          nb2[x0 * NB2P + py] = a;
          nbs[x0 * NB2P + py] = sqrtf(fmaxf(a, 0.f));
          sbt[x0 * NB2P + py] = l;
          amax = fmaxf(amax, a);
#pragma unroll
          for (int u = 1; u < 7; ++u) {
            const int px = x0 + u;
            if (px < PR) {
              const float na = cs[py * NB2P + px + TD - 1], nl = cl[py * NB2P + px + TD - 1];
              a = (a + na) - qa[(u - 1) & 7];
              l = (l + nl) - ql[(u - 1) & 7];
              qa[(u + TD - 1) & 7] = na;
              ql[(u + TD - 1) & 7] = nl;
              nb2[px * NB2P + py] = a;
              nbs[px * NB2P + py] = sqrtf(fmaxf(a, 0.f));
              sbt[px * NB2P + py] = l;
              amax = fmaxf(amax, a);
            }
          }
        }
        // non-negative floats order as their bit patterns
        amax = warp_max(amax);
        if (lane == 0) atomicMax(nbt_s, __float_as_int(amax));
      }
      __syncthreads();  // cs, cl are overwritten by E below
    }
    // E: entry (y, x) = the 8 centred values of row y from column x.
    // Warp w builds columns 8 (w % 8) .. + 7 and rows 32 (w / 8) .. + 31; in one
    // store, lanes 8k .. 8k+7 write 8 consecutive entries of one row (no bank
    // conflicts) and the region reads (pitch 68) fall in 32 distinct banks.
    {
      const int x = 8 * (warp & 7) + (lane & 7);
#pragma unroll 1
      for (int jj = 0; jj < 8; ++jj) {
        const int y = 32 * (warp >> 3) + (lane >> 3) + 4 * jj;
        uint4 q = make_uint4(0, 0, 0, 0);  // entries past column 56 belong to no position of the grid
        if (x + 8 <= RC) {
          float v[8];
#pragma unroll
          for (int dx = 0; dx < 8; ++dx) v[dx] = reg[(x + dx) * RP + y] - m0;
          q = make_uint4(pack_op<HALF>(v[0], v[1]), pack_op<HALF>(v[2], v[3]), pack_op<HALF>(v[4], v[5]),
                         pack_op<HALF>(v[6], v[7]));
        }
        *reinterpret_cast<uint4*>(E + (y * XW + x) * 16) = q;
      }
    }
    // B: reference j = li + 4 lj centred on its own mean, in MMA column
    // n = 4 li + lj; block row r at (n/8 * 8 + r) * 128 + (n%8) * 16.
    // Warp j, lane = element r * 8 + c (two per lane).
    {
      const int j = warp, li = j & 3, lj = j >> 2, n = 4 * li + lj;
      const float* src = reg + (s * lj + H) * RP + s * li + H;
      float x2[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int e = lane + 32 * u, r = e >> 3, c = e & 7;
        x2[u] = src[r + c * RP] - m0;
      }
      const float ma = warp_sum(x2[0] + x2[1]) * (1.f / 64.f);
      float z2 = 0.f;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        x2[u] -= ma;
        z2 = fmaf(x2[u], x2[u], z2);
      }
      const float na = sqrtf(warp_sum(z2));
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const float nb = __shfl_down_sync(FULL, x2[u], 1);
        const uint32_t w = pack_op<HALF>(x2[u], nb);
        if ((lane & 1) == 0) {
          const int e = lane + 32 * u, r = e >> 3, c = e & 7;
          *reinterpret_cast<uint32_t*>(Bq + ((n >> 3) * 8 + r) * 128 + (n & 7) * 16 + c * 2) = w;
        }
      }
      if (lane == 0) {
        rma[n] = ma;
        kf[j] = err_factor<HALF>(na);
      }
    }
    __syncthreads();
    // ---- TMEM init ma sum(x'_p) - ||x'_p||^2 / 2, then the MMAs ----------------------
    {
      const int q = warp & 3;
      const int p = 32 * q + lane;
      const int py0 = p >> 6, px = p & 63;
      float ma[NREF];
#pragma unroll
      for (int n = 0; n < NREF; ++n) ma[n] = rma[n];
      for (int c = warp >> 2; c < NCH; c += 4) {
        const int py = 2 * c + py0;
        const bool in = py < PR && px < PR;
        const float h = in ? -0.5f * nb2[px * NB2P + py] : 0.f;
        const float sb = in ? sbt[px * NB2P + py] : 0.f;
        uint32_t v[NREF];
#pragma unroll
        for (int n = 0; n < NREF; ++n) v[n] = __float_as_uint(fmaf(ma[n], sb, h));
        tc::tmem_st16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(16 * c), v);
      }
      tc::tmem_wait_st();
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    // NISS threads issue the chunks' MMAs (disjoint TMEM columns; the four
    // K steps of a chunk in order from one thread), so no warp's re-rank
    // below waits for all 112 issues; NCH >= 10 > NISS, every issuer has one
    if (warp < NISS && lane == 0) {
      const uint32_t e0 = tc::smem_u32(E), b0 = tc::smem_u32(Bq);
      constexpr uint32_t idesc = HALF ? tc::idesc_f16_f32(128, NREF) : tc::idesc_bf16_f32(128, NREF);
      for (int c = warp; c < NCH; c += NISS) {
#pragma unroll
        for (int r = 0; r < TD; r += 2)
          tc::mma_bf16(tmem + (uint32_t)(16 * c), tc::desc_kmajor(e0 + (2 * c + r) * (XW * 16), XW * 16, 128),
                       tc::desc_kmajor(b0 + r * 128, 128, 1024), idesc, 1u);
      }
      tc::commit(&mbar[NRB]);
    }
    mma_pending = true;
    // ---- the previous tile's re-rank overlaps these MMAs ------------------------------
    if (it > 0) rerank(it - 1);
    __syncthreads();  // re-rank done: its region buffer, lists, counts and S rows are free
    // ---- prefetch two tiles ahead, then this tile's selection -------------------------
    if (tid == 0) issue_tma(it + 2);
    if (tid < NREF) cnt[tid] = 0;
    if (tc::mbar_wait(&mbar[NRB], mma_phase, wait)) {
      mma_phase ^= 1u;
      mma_pending = false;
    } else {
      *fail_s = 1;
    }
    tc::fence_after_sync();
    __syncthreads();
    if (tq[(it + 2) % NRB] >= 0) tma_pending |= 1u << ((it + 2) % NRB);
    if (*fail_s) break;
    // warp (q, li): TMEM lanes 32 q .. (positions of parity q / 2, columns
    // 32 (q & 1) ..), references (li, lj) for lj = 0..3 (TMEM columns 4 li ..),
    // over the NC chunks of their window rows of this parity
    const int q = warp & 3, li = warp >> 2;
    const int par = q >> 1, px = lane + 32 * (q & 1);
    const int c_lo = (s * li - par + 1) >> 1;  // first chunk with 2 c + par >= s li
    const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(4 * li);
    // pass 1: best v of each window column, per row parity
    {
      float best[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
#pragma unroll
      for (int c0 = 0; c0 < NC; c0 += 4) {
        uint32_t v[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u) tc::tmem_ld4_async(tbase + (uint32_t)(16 * (c_lo + c0 + u)), v[u]);
        tc::tmem_wait_ld();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          tc::reg_fence4(v[u]);
#pragma unroll
          for (int lj = 0; lj < 4; ++lj) best[lj] = fmaxf(best[lj], __uint_as_float(v[u][lj]));
        }
      }
#pragma unroll
      for (int lj = 0; lj < 4; ++lj) {
        const bool colok = px >= s * lj && px < s * lj + D2;
        cb[((li + 4 * lj) * 2 + par) * 64 + px] = colok ? best[lj] : -INFINITY;
      }
    }
    __syncthreads();
    // thresholds: warp j; lane l = window column l
    {
      const int j = warp, tli = j & 3, tlj = j >> 2;
      const int wy = s * tli, wx = s * tlj;
      // K-th largest of the 2 d2 group bests: sort each parity's d2 (descending
      // by lane), then max over i of min(A[i-1], B[K-1-i]) (A[-1] = B[-1] = +inf)
      float ga = -INFINITY, gb = -INFINITY, wmax = 0.f;
      if (lane < D2) {
        ga = cb[(j * 2) * 64 + wx + lane];
        gb = cb[(j * 2 + 1) * 64 + wx + lane];
        for (int r = 0; r < D2; ++r) wmax = fmaxf(wmax, nb2[(wx + lane) * NB2P + wy + r]);
      }
      ga = -warp_sort_asc(-ga, lane);  // descending
      gb = -warp_sort_asc(-gb, lane);
      const int K = A.K;
      const float a_prev = __shfl_sync(FULL, ga, (lane + 31) & 31);   // A[lane - 1]
      const float b_pair = __shfl_sync(FULL, gb, (K - 1 - lane) & 31);  // B[K - 1 - lane]
      float cand = -INFINITY;
      if (lane <= K) cand = fminf(lane == 0 ? INFINITY : a_prev, lane == K ? INFINITY : b_pair);
      const float T = warp_max(cand);
      const float nbw2 = warp_max(wmax);
      const float nat2 = nb2[(wx + H) * NB2P + wy + H];  // ||a - m0||^2
      if (lane == 0) thr[j] = T - kf[j] * sqrtf(nbw2) - fp32_slack(nat2, nbw2, __int_as_float(*nbt_s));
    }
    __syncthreads();
    // pass 2: list every window position with v + k ||x'_p|| >= threshold
    {
      float th[4], kk[4];
      bool colok[4];
#pragma unroll
      for (int lj = 0; lj < 4; ++lj) {
        th[lj] = thr[li + 4 * lj];
        kk[lj] = kf[li + 4 * lj];
        colok[lj] = px >= s * lj && px < s * lj + D2;
      }
#pragma unroll
      for (int c0 = 0; c0 < NC; c0 += 4) {
        uint32_t v[4][4];
        float nbp[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          tc::tmem_ld4_async(tbase + (uint32_t)(16 * (c_lo + c0 + u)), v[u]);
          nbp[u] = nbs[px * NB2P + 2 * (c_lo + c0 + u) + par];
        }
        tc::tmem_wait_ld();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          tc::reg_fence4(v[u]);
          const int py = 2 * (c_lo + c0 + u) + par;
#pragma unroll
          for (int lj = 0; lj < 4; ++lj) {
            if (colok[lj] && fmaf(kk[lj], nbp[u], __uint_as_float(v[u][lj])) >= th[lj]) {
              const int j = li + 4 * lj;
              const int slot = atomicAdd(&cnt[j], 1);
              if (slot < CAP) lst[j * CAP + slot] = (uint32_t)(py * 64 + px);
            }
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  const bool failed = *fail_s != 0;
  if (!failed && it > 0) rerank(it - 1);
  if (failed) {
    // a wait gave up: let this CTA's copies and MMAs in flight land (with the
    // full limit) before its shared memory and TMEM are released
    for (int b = 0; b < NRB; ++b)
      if ((tma_pending >> b) & 1u) tc::mbar_wait(&mbar[b], (tma_phase >> b) & 1u, WAIT_CYCLES);
    if (mma_pending) tc::mbar_wait(&mbar[NRB], mma_phase, WAIT_CYCLES);
    if (tid == 0 && A.err) atomicOr(A.err, 2);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

template <int D2, bool HALF>
cudaError_t launch_tc_t(const MatchArgs& A, cudaStream_t st) {
  // the search image: rows (inner) R of pitch P floats, columns Q; box RP x RC
  CUtensorMap tm;
  if (!encode_search_map(&tm, A.pad, A.R, A.Q, A.P, RP, RC)) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_match_tc<D2, HALF>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(A.ovf_count, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(A.work, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int tiles = ((A.M + TT - 1) / TT) * ((A.N + TT - 1) / TT);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_match_tc<D2, HALF><<<std::min(tiles, sms), NT, SMEM_BYTES, st>>>(tm, A);
  return cudaGetLastError();
}

}  // namespace

bool match_tc_supported(int d, int d2, int s, int K, bool tol_branch) {
  if (d != TD || K < 1 || K > 16 || tol_branch || s < 1 || s > TD) return false;
  if (d2 != 16 && d2 != 24 && d2 != 32) return false;
  return 3 * s + d2 <= PRMAX;
}

cudaError_t launch_match_tc(int d, int d2, const MatchArgs& A, bool f16, cudaStream_t st) {
  if (!match_tc_supported(d, d2, A.s, A.K, A.tol_branch != 0)) return cudaErrorInvalidValue;
  // TMA: 16-byte aligned base and pitch; the tile's first row i0 s = 4 ti s is
  // a multiple of 4 floats, so every box starts on a 16-byte boundary
  if ((reinterpret_cast<uintptr_t>(A.pad) & 15) || (A.P & 3) || !A.ovf_list || !A.ovf_count || !A.work || A.R < 1 ||
      A.Q < 1)
    return cudaErrorInvalidValue;
  if (f16) {
    if (d2 == 32) return launch_tc_t<32, true>(A, st);
    if (d2 == 24) return launch_tc_t<24, true>(A, st);
    return launch_tc_t<16, true>(A, st);
  }
  if (d2 == 32) return launch_tc_t<32, false>(A, st);
  if (d2 == 24) return launch_tc_t<24, false>(A, st);
  return launch_tc_t<16, false>(A, st);
}

}  // namespace gbm3d
