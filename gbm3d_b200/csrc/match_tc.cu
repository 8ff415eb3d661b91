// Block matching on the tensor cores — the search of matchBlocksCPU.m:21-116
// (and of matchBlocksWie.m:21-92), with the distances of
// matchBlocksCPU.m:82-85, ||x - y||^2 = ||x||^2 + ||y||^2 - 2<x,y>, where the
// <x,y> term is a bf16 GEMM with fp32 accumulation on tcgen05, used to bound
// the candidates; the exact FP32 sums of squared differences then rank them
// in the exhaustive matcher's operation order, so the match sets are that
// matcher's own.
//
// Tile: 4 x 4 references (MMA N = 16) at stride s.  Their search windows
// cover a PR x PR grid of candidate positions, PR = 3 s + d2 <= 56, whose 8 x 8
// blocks lie in a 64 x 68 region of the search image, loaded by one TMA copy
// (the tensor map covers this GPU's search image; no multicast).  Centring
// every value on the region mean m0 (x' = x - m0), the positions are the MMA's
// A operand without an im2col copy: E(y, x) holds the 8 values x'(y, x..x+7)
// in bf16 (16 bytes), stored row-major with 64 entries per row, so the A rows
// of a chunk of 128 positions (2 position rows of 64) are 128 consecutive
// entries and the K = 16 slice of block rows r, r+1 is the same array read
// from r rows further on (descriptor start + r * 1024 bytes, leading byte
// offset 1024 between the two rows, stride byte offset 128 between 8-position
// groups).  Four MMAs (r = 0, 2, 4, 6) give <x'_p, a_j> for all 128 positions
// p of a chunk and the 16 references j, accumulated in TMEM on top of a value
// per (p, j) written there first (below).  All chunks of a tile (at most 28 x
// 16 fp32 columns) stay in TMEM.
//
// The reference operand is centred on its own block mean as well (a_z = a -
// m0 - ma, a_z.1 = 0), which keeps the bf16 rounding error proportional to
// ||a_z|| (noise and texture) instead of the grey level; then
//     D(p, j) = ||a_z||^2 - 2 v(p, j),
//     v(p, j) = <x'_p, a_z> - (||x'_p||^2 - 2 ma sum(x'_p) + 64 ma^2) / 2,
// and the second term is what TMEM holds before the MMAs add the first.
//
// Selection, per reference j: pass 1 takes the best v of every window column
// and row parity (64 groups of 16 positions at matchSize 32; TMEM lane =
// position, so a lane's column and parity are fixed); T = the K-th best of
// those group bests, so at least K positions have v >= T.  With
// |v - v_exact| <= k ||x'_p|| (bf16 rounding of both operands, fp32
// accumulation: k ~ 2^-8 ||a_z||), every position of the exact top K has
//     v + k ||x'_p|| >= T - k max_window ||x'|| - h
// (h bounds the FP32 rounding of the exact sums); pass 2 lists exactly those
// positions.  The listed candidates (about 20-30) are re-ranked by the exact
// FP32 SSD (t = x - y, acc = fmaf(t, t, acc), row-major over the block, as
// the exhaustive matcher adds) and the K best by (distance, column-major
// window index) are kept, S(1) forced to the reference (matchBlocksCPU.m:103).
// A reference whose list overflows is appended to a global list that the
// exhaustive matcher finishes.
//
// Every wait (TMA, MMA) gives up after about two seconds of SM clock, sets
// bit 1 of the status word and skips the rest; TMEM is always released.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

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
constexpr int CAP = 256;        // candidate list capacity per reference
constexpr int NT = 512;         // threads: 16 warps
constexpr int NB2P = 65;        // pitch of the ||x'||^2 table (bank-conflict free both ways)
constexpr long long WAIT_CYCLES = 4000000000LL;  // ~2 s at 2 GHz

constexpr int OFF_REG = 0;                                   // RP x RC floats, column-major
constexpr int OFF_E = OFF_REG + RP * RC * 4;                 // 64 x 64 entries of 16 bytes
constexpr int OFF_B = OFF_E + 64 * XW * 16;                  // reference operand: 16 x 64 bf16
constexpr int TBL = 64 * NB2P * 4;                           // one [px * NB2P + py] table
constexpr int OFF_NB2 = OFF_B + NREF * 64 * 2;               // ||x'_p||^2
constexpr int OFF_NBS = OFF_NB2 + TBL;                       // ||x'_p||
constexpr int OFF_SB = OFF_NBS + TBL;                        // sum(x'_p)
constexpr int OFF_CB = OFF_SB + TBL;                         // group bests [ref][parity][64]
constexpr int OFF_LST = OFF_CB + NREF * 2 * 64 * 4;          // candidate lists [ref][CAP]
constexpr int OFF_MISC = OFF_LST + NREF * CAP * 4;
constexpr int SMEM_BYTES = OFF_MISC + 1024;
static_assert(OFF_E % 1024 == 0 && OFF_B % 128 == 0, "operand alignment");

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

template <int D2, bool HALF>
__global__ void __launch_bounds__(NT, 1) k_match_tc(const __grid_constant__ CUtensorMap tmap, MatchArgs A) {
  constexpr int H = D2 / 2;
  extern __shared__ __align__(1024) unsigned char smem[];
  float* reg = reinterpret_cast<float*>(smem + OFF_REG);
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
  float* rma = kf + 16;                                 // [16] reference means ma
  float* rcj = rma + 16;                                // [16] -32 ma^2
  float* red = rcj + 16;                                // [32] reductions
  uint64_t* mbar = reinterpret_cast<uint64_t*>(red + 32);  // [2] TMA, MMA
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(mbar + 2);
  int* fail_s = reinterpret_cast<int*>(taddr_s + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned FULL = 0xffffffffu;
  const int s = A.s;
  const int PR = 3 * s + D2;      // position grid side
  const int VR = PR + TD - 1;     // region side the blocks touch
  const int NCH = (PR + 1) / 2;   // chunks of 2 position rows
  const int tiles_i = (A.M + TT - 1) / TT;
  const int i0 = (blockIdx.x % tiles_i) * TT, j0 = (blockIdx.x / tiles_i) * TT;

  if (warp == 0) tc::tmem_alloc(taddr_s, 512);
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
    tc::fence_mbar_init();
    *fail_s = 0;
  }
  if (tid < NREF) cnt[tid] = 0;
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *taddr_s;

  // ---- region of the search image: rows i0 s .., columns j0 s .. (zero past its end)
  if (tid == 0) {
    tc::mbar_expect_tx(&mbar[0], RP * RC * 4);
    tc::tma_load_2d(reg, &tmap, i0 * s, j0 * s, &mbar[0]);
  }
  if (!tc::mbar_wait(&mbar[0], 0, WAIT_CYCLES)) *fail_s = 1;
  __syncthreads();
  const bool failed_load = *fail_s != 0;

  if (!failed_load) {
    // ---- centre m0: mean of the region the blocks touch --------------------
    float sum = 0.f;
    for (int e = tid; e < VR * VR; e += NT) {
      const int x = e / VR, y = e - x * VR;
      sum += reg[x * RP + y];
    }
    sum = warp_sum(sum);
    if (lane == 0) red[warp] = sum;
    __syncthreads();
    if (warp == 0) {
      const float t = warp_sum(lane < NT / 32 ? red[lane] : 0.f);
      if (lane == 0) red[16] = t / (float)(VR * VR);
    }
    __syncthreads();
    const float m0 = red[16];

    // ---- per position: ||x'||^2, ||x'|| and sum(x') from column sums over 8
    // rows (kept in the E area until E is built); 0 outside the grid
    float* cs = reinterpret_cast<float*>(E);       // [x * 64 + y] sums of squares
    float* cl = cs + 64 * 64;                      // [x * 64 + y] sums
    for (int e = tid; e < PR * VR; e += NT) {
      const int x = e / PR, y = e - x * PR;
      const float* col = reg + x * RP + y;
      float a = 0.f, l = 0.f;
#pragma unroll
      for (int r = 0; r < TD; ++r) {
        const float t = col[r] - m0;
        a = fmaf(t, t, a);
        l += t;
      }
      cs[x * 64 + y] = a;
      cl[x * 64 + y] = l;
    }
    __syncthreads();
    for (int e = tid; e < 64 * 64; e += NT) {
      const int px = e >> 6, py = e & 63;
      float a = 0.f, l = 0.f;
      if (py < PR && px < PR) {
#pragma unroll
        for (int c = 0; c < TD; ++c) {
          a += cs[(px + c) * 64 + py];
          l += cl[(px + c) * 64 + py];
        }
      }
      nb2[px * NB2P + py] = a;
      nbs[px * NB2P + py] = sqrtf(a);
      sbt[px * NB2P + py] = l;
    }
    __syncthreads();  // cs, cl are overwritten by E below

    // ---- E: entry (y, x) = the 8 centred values of row y from column x, bf16.
    // Warp w builds columns 8 (w % 8) .. + 7 and rows 32 (w / 8) .. + 31; in one
    // store, lanes 8k .. 8k+7 write 8 consecutive entries of one row (no bank
    // conflicts) and the region reads (pitch 68) fall in 32 distinct banks.
    {
      const int x = 8 * (warp & 7) + (lane & 7);
#pragma unroll 1
      for (int jj = 0; jj < 8; ++jj) {
        const int y = 32 * (warp >> 3) + (lane >> 3) + 4 * jj;
        float v[8];
#pragma unroll
        for (int dx = 0; dx < 8; ++dx) v[dx] = x + dx < RC ? reg[(x + dx) * RP + y] - m0 : 0.f;
        const uint4 q = make_uint4(pack_op<HALF>(v[0], v[1]), pack_op<HALF>(v[2], v[3]), pack_op<HALF>(v[4], v[5]),
                                   pack_op<HALF>(v[6], v[7]));
        *reinterpret_cast<uint4*>(E + (y * XW + x) * 16) = q;
      }
    }
    // ---- B: reference j = li + 4 lj centred on its own mean; block row r at
    // (j/8 * 8 + r) * 128 + (j%8) * 16.  Warp j, lane = element r * 8 + c (two per lane).
    {
      const int j = warp, li = j & 3, lj = j >> 2;
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
      // lanes 0..31 hold elements (r, c) = (lane / 8, lane % 8) and (4 + lane / 8, lane % 8)
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const float nb = __shfl_down_sync(FULL, x2[u], 1);
        const uint32_t w = pack_op<HALF>(x2[u], nb);
        if ((lane & 1) == 0) {
          const int e = lane + 32 * u, r = e >> 3, c = e & 7;
          *reinterpret_cast<uint32_t*>(Bq + ((j >> 3) * 8 + r) * 128 + (j & 7) * 16 + c * 2) = w;
        }
      }
      if (lane == 0) {
        rma[j] = ma;
        rcj[j] = -32.f * ma * ma;
        kf[j] = err_factor<HALF>(na);
      }
    }
    __syncthreads();
    // ---- TMEM: (2 ma sum(x'_p) - ||x'_p||^2 - 64 ma^2) / 2 for the 16
    // references in the 16 columns of every chunk
    {
      const int q = warp & 3;
      const int p = 32 * q + lane;
      const int py0 = p >> 6, px = p & 63;
      float ma[NREF], cj[NREF];
#pragma unroll
      for (int j = 0; j < NREF; ++j) {
        ma[j] = rma[j];
        cj[j] = rcj[j];
      }
      for (int c = warp >> 2; c < NCH; c += 4) {
        const int py = 2 * c + py0;
        const bool in = py < PR && px < PR;
        const float h = in ? -0.5f * nb2[px * NB2P + py] : 0.f;
        const float sb = in ? sbt[px * NB2P + py] : 0.f;
        uint32_t v[NREF];
#pragma unroll
        for (int j = 0; j < NREF; ++j) v[j] = __float_as_uint(fmaf(ma[j], sb, h + cj[j]));
        tc::tmem_st16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(16 * c), v);
      }
      tc::tmem_wait_st();
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t e0 = tc::smem_u32(E), b0 = tc::smem_u32(Bq);
      constexpr uint32_t idesc = HALF ? tc::idesc_f16_f32(128, NREF) : tc::idesc_bf16_f32(128, NREF);
      for (int c = 0; c < NCH; ++c) {
#pragma unroll
        for (int r = 0; r < TD; r += 2)
          tc::mma_bf16(tmem + (uint32_t)(16 * c), tc::desc_kmajor(e0 + (2 * c + r) * (XW * 16), XW * 16, 128),
                       tc::desc_kmajor(b0 + r * 128, 128, 1024), idesc, 1u);
      }
      tc::commit(&mbar[1]);
    }
    if (!tc::mbar_wait(&mbar[1], 0, WAIT_CYCLES)) *fail_s = 1;
    tc::fence_after_sync();
    __syncthreads();
  }
  const bool failed = *fail_s != 0;

  if (!failed) {
    // warp (q, h): TMEM lanes 32 q .. (positions of parity q / 2, columns
    // 32 (q & 1) ..), references j = li + 4 h (one window column range)
    const int q = warp & 3, h = warp >> 2;
    const int par = q >> 1, px = lane + 32 * (q & 1);
    const bool colok = px >= s * h && px < s * h + D2;
    const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(4 * h);

    // ---- pass 1: best v of each window column, per row parity -----------------
    float best[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < NCH; ++c) {
      const int py = 2 * c + par;
      if (py >= PR) break;
      float v[4];
      tc::tmem_ld4(tbase + (uint32_t)(16 * c), v);
      tc::tmem_wait_ld();
#pragma unroll
      for (int li = 0; li < 4; ++li)
        if (py >= s * li && py < s * li + D2) best[li] = fmaxf(best[li], v[li]);
    }
#pragma unroll
    for (int li = 0; li < 4; ++li) cb[((li + 4 * h) * 2 + par) * 64 + px] = colok ? best[li] : -INFINITY;
    __syncthreads();

    // ---- thresholds: warp j; lane l = window column l -------------------------
    {
      const int j = warp, li = j & 3, lj = j >> 2;
      const int wy = s * li, wx = s * lj;
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
      if (lane == 0) thr[j] = T - kf[j] * sqrtf(nbw2) - (nat2 + nbw2) * (1.f / 32768.f) - 8.f;
    }
    __syncthreads();

    // ---- pass 2: list every window position with v + k ||x'_p|| >= threshold --
    {
      float th[4], kk[4];
#pragma unroll
      for (int li = 0; li < 4; ++li) {
        th[li] = thr[li + 4 * h];
        kk[li] = kf[li + 4 * h];
      }
      for (int c = 0; c < NCH; ++c) {
        const int py = 2 * c + par;
        if (py >= PR) break;
        float v[4];
        tc::tmem_ld4(tbase + (uint32_t)(16 * c), v);
        const float nbp = nbs[px * NB2P + py];
        tc::tmem_wait_ld();
#pragma unroll
        for (int li = 0; li < 4; ++li) {
          if (colok && py >= s * li && py < s * li + D2 && fmaf(kk[li], nbp, v[li]) >= th[li]) {
            const int j = li + 4 * h;
            const int slot = atomicAdd(&cnt[j], 1);
            if (slot < CAP) lst[j * CAP + slot] = (uint32_t)(py * 64 + px);
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();

    // ---- exact re-rank: warp j --------------------------------------------------
    {
      const int j = warp, li = j & 3, lj = j >> 2;
      const int ri = i0 + li, rj = j0 + lj;
      if (ri < A.M && rj < A.N) {
        const int g = ri + A.M * rj;
        const int C = cnt[j];
        const int K = A.K;
        const uint32_t center = (uint32_t)(H + H * D2 + 1);
        uint32_t* Sg = A.S + (size_t)g * K;
        uint32_t* sel = reinterpret_cast<uint32_t*>(cb) + j * 32;  // the group bests are no longer needed
        if (C > CAP) {
          if (lane == 0) A.ovf_list[atomicAdd(A.ovf_count, 1)] = g;
        } else {
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
            for (int r = 0; r < TD; ++r)
#pragma unroll
              for (int c = 0; c < TD; ++c) {
                const float t = xr[r * TD + c] - cand[r + c * RP];
                acc = fmaf(t, t, acc);
              }
            const uint32_t ix = (uint32_t)((py - wy) + (pxx - wx) * D2);
            return ((u64)__float_as_uint(acc) << 32) | ix;
          };
          if (C <= 64) {
            // two sorted halves of up to 32 keys; an element's rank is its place
            // in its own half plus the other half's keys below it
            u64 k0 = lane < C ? exact_key(lane) : ~0ull;
            u64 k1 = lane + 32 < C ? exact_key(lane + 32) : ~0ull;
            k0 = warp_sort_asc(k0, lane);
            k1 = warp_sort_asc(k1, lane);
            auto below = [&](u64 x, u64 other) {  // keys of the sorted `other` half below x
              int lo = 0;
#pragma unroll
              for (int b = 16; b >= 1; b >>= 1) {
                const u64 o = __shfl_sync(FULL, other, lo + b - 1);
                if (o < x) lo += b;
              }
              const u64 o = __shfl_sync(FULL, other, lo & 31);
              return lo + ((lo < 32 && o < x) ? 1 : 0);
            };
            const int r0 = lane + below(k0, k1), r1 = lane + below(k1, k0);
            if (k0 != ~0ull && r0 < K) sel[r0] = r0 == 0 ? center : (uint32_t)k0 + 1u;
            if (k1 != ~0ull && r1 < K) sel[r1] = r1 == 0 ? center : (uint32_t)k1 + 1u;
          } else {
            u64* kb = reinterpret_cast<u64*>(E) + j * CAP;  // E is free once the MMAs are done
            for (int e = lane; e < C; e += 32) kb[e] = exact_key(e);
            __syncwarp();
            for (int e = lane; e < C; e += 32) {
              const u64 ke = kb[e];
              int rank = 0;
              for (int t = 0; t < C; ++t) rank += kb[t] < ke ? 1 : 0;
              if (rank < K) sel[rank] = rank == 0 ? center : (uint32_t)ke + 1u;
            }
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
                const int t = lane + 32 * u, r = t & 7, c = t >> 3;
                A.volume[(size_t)(ri * TD + r) + (size_t)A.m * (rj * TD + c) + mn * k] = src[r + c * RP];
              }
            }
          }
        }
      }
    }
  }
  if (failed && tid == 0 && A.err) atomicOr(A.err, 2);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

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

template <int D2, bool HALF>
cudaError_t launch_tc_t(const MatchArgs& A, cudaStream_t st) {
  auto encode = encode_fn();
  if (!encode) return cudaErrorNotSupported;
  // the search image: rows (inner) R of pitch P floats, columns Q; box RP x RC
  CUtensorMap tm;
  const cuuint64_t dims[2] = {(cuuint64_t)A.R, (cuuint64_t)A.Q};
  const cuuint64_t strides[1] = {(cuuint64_t)A.P * sizeof(float)};
  const cuuint32_t box[2] = {RP, RC};
  const cuuint32_t es[2] = {1, 1};
  if (encode(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(A.pad), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_match_tc<D2, HALF>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(A.ovf_count, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int tiles = ((A.M + TT - 1) / TT) * ((A.N + TT - 1) / TT);
  k_match_tc<D2, HALF><<<tiles, NT, SMEM_BYTES, st>>>(tm, A);
  return cudaGetLastError();
}

}  // namespace

bool match_tc_supported(int d, int d2, int s, int K, bool tol_branch) {
  if (d != TD || K < 1 || K > 16 || tol_branch || s < 1 || s > TD) return false;
  if (d2 != 16 && d2 != 24 && d2 != 32) return false;
  return 3 * s + d2 <= PRMAX;
}

cudaError_t launch_match_tc(int d, int d2, const MatchArgs& A, cudaStream_t st) {
  if (!match_tc_supported(d, d2, A.s, A.K, A.tol_branch != 0)) return cudaErrorInvalidValue;
  // TMA: 16-byte aligned base and pitch; the tile's first row i0 s = 4 ti s is
  // a multiple of 4 floats, so every box starts on a 16-byte boundary
  if ((reinterpret_cast<uintptr_t>(A.pad) & 15) || (A.P & 3) || !A.ovf_list || !A.ovf_count || A.R < 1 || A.Q < 1)
    return cudaErrorInvalidValue;
  if (d2 == 32) return launch_tc_t<32, false>(A, st);
  if (d2 == 24) return launch_tc_t<24, false>(A, st);
  return launch_tc_t<16, false>(A, st);
}

}  // namespace gbm3d
