// Learned pilot: a residual CNN that stands in for step 1 (the hard-
// thresholded estimate), with its training kernels.
//
// Network (8 layers of 3x3 convolutions, "same" zero padding):
//   input  2 channels: noisy / 255 and sigma / 255 (padded to 16 with zeros)
//   layers 1..7: conv -> 48 channels, + bias, ReLU      (bf16 activations)
//   layer  8: conv -> 1 channel (padded to 16), + bias = r
//   pilot = noisy - 255 r                                 (fp32)
// Activations are NHWC bf16 ([image][row][column][channel]).
//
// Forward convolution (and the data gradient, which is a forward convolution
// with flipped, transposed weights) is an implicit GEMM on the tcgen05 tensor
// cores: a CTA takes 128 consecutive pixels of one row (M = 128), the output
// channels are N, and the 9 taps x input channels are K, 16 per MMA.  The
// three input rows the tile needs sit in shared memory "pixel-major inside
// each 8-channel chunk" (element (p, c) at (c/8)*LBO + p*16 + (c%8)*2), so the
// operand of tap (dy, dx) is the same buffer read from pixel dx+1 of row dy+1:
// a descriptor start offset of 16 (dx+1) bytes, no data movement.  The
// weights of all 9 taps stay in shared memory for the CTA's whole run.
//
// The weight gradient is a reduction over pixels done on the FP32 CUDA cores
// (per-CTA partial sums, then a fixed-order sum across CTAs, so training is
// deterministic); the optimizer is Adam on FP32 master weights.
#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace gbm3d {

namespace {

constexpr int TP = 128;       // pixels per tile (MMA M)
constexpr int NPX = TP + 2;   // tile pixels with the left/right halo
constexpr int LBO_A = NPX * 16;
constexpr long long PWAIT = 4000000000LL;

enum { EPI_ACT = 0, EPI_OUT = 1, EPI_DX = 2 };

struct ConvArgs {
  const uint16_t* in;    // NHWC bf16, CIN channels
  const uint16_t* w;     // bf16 [9][COUT][CIN]
  const float* bias;     // COUT (EPI_ACT / EPI_OUT)
  uint16_t* out;         // NHWC bf16, COUT channels (EPI_ACT / EPI_DX)
  const uint16_t* mask;  // EPI_DX: activation whose ReLU gates the gradient (COUT channels)
  const float* img;      // EPI_OUT: noisy image (fp32, [image][row][column])
  float* pilot;          // EPI_OUT: noisy - 255 r
  int nimg, H, W;
  int* err;
};

__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(128) k_conv(ConvArgs A) {
  constexpr int KCH = CIN / 8;                 // 8-channel chunks of the input
  constexpr int ROWB = KCH * LBO_A;            // bytes of one input row buffer
  constexpr int WB = 9 * COUT * CIN * 2;       // weight bytes
  constexpr int TCOLS = COUT <= 32 ? 32 : 64;  // TMEM columns
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sX = smem;                    // 3 row buffers
  unsigned char* sW = smem + 3 * ROWB;         // 9 taps, K-major core matrices
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sW + WB);
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(mbar + 1);
  int* fail_s = reinterpret_cast<int*>(taddr_s + 1);
  const int tid = threadIdx.x, warp = tid >> 5;

  if (warp == 0) tc::tmem_alloc(taddr_s, TCOLS);
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
    *fail_s = 0;
  }
  // weights: tap t, row co, k = ci
  for (int e = tid; e < 9 * COUT * (CIN / 8); e += 128) {
    const int t = e / (COUT * (CIN / 8)), r = e % (COUT * (CIN / 8));
    const int co = r / (CIN / 8), j = r % (CIN / 8);
    const uint4 v = *reinterpret_cast<const uint4*>(A.w + ((size_t)t * COUT + co) * CIN + 8 * j);
    *reinterpret_cast<uint4*>(sW + (size_t)t * COUT * CIN * 2 + tc::kmajor_offset(co, 8 * j, CIN)) = v;
  }
  const int xt_n = (A.W + TP - 1) / TP;
  const int ntiles = A.nimg * A.H * xt_n;
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *taddr_s;
  constexpr uint32_t idesc = tc::idesc_bf16_f32(TP, COUT);
  uint32_t phase = 0;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int xt = tile % xt_n, y = (tile / xt_n) % A.H, n = tile / (xt_n * A.H);
    const int x0 = xt * TP;
    // ---- the three input rows y-1 .. y+1, pixels x0-1 .. x0+128, zero outside ----
    for (int e = tid; e < 3 * NPX * KCH; e += 128) {
      const int r = e / (NPX * KCH), q = (e / KCH) % NPX, j = e % KCH;
      const int yy = y + r - 1, xx = x0 + q - 1;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (yy >= 0 && yy < A.H && xx >= 0 && xx < A.W)
        v = *reinterpret_cast<const uint4*>(A.in + (((size_t)n * A.H + yy) * A.W + xx) * CIN + 8 * j);
      *reinterpret_cast<uint4*>(sX + r * ROWB + j * LBO_A + q * 16) = v;
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t xa = tc::smem_u32(sX), wa = tc::smem_u32(sW);
      int first = 1;
#pragma unroll 1
      for (int t = 0; t < 9; ++t) {
        const int dy = t / 3, dx = t % 3;  // row buffer dy, pixel offset dx (0..2 = -1..+1)
#pragma unroll
        for (int ks = 0; ks < CIN / 16; ++ks) {
          const uint64_t ad = tc::desc_kmajor(xa + dy * ROWB + dx * 16 + 2 * ks * LBO_A, LBO_A, 128);
          const uint64_t bd = tc::desc_kmajor(wa + t * COUT * CIN * 2 + 2 * ks * 128, 128, (CIN / 8) * 128);
          tc::mma_bf16(tmem, ad, bd, idesc, first ? 0u : 1u);
          first = 0;
        }
      }
      tc::commit(mbar);
    }
    const bool ok = tc::mbar_wait(mbar, phase, PWAIT);
    phase ^= 1u;
    if (!ok) *fail_s = 1;
    tc::fence_after_sync();
    // ---- epilogue: thread = pixel -------------------------------------------
    const int x = x0 + tid;
    const size_t pix = ((size_t)n * A.H + y) * A.W + x;
    float v[64];
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    tc::tmem_ld32(lane_base, v);
    if (COUT > 32) tc::tmem_ld32(lane_base + 32, v + 32);
    if (ok && x < A.W) {
      if (EPI == EPI_OUT) {
        A.pilot[pix] = A.img[pix] - 255.f * (v[0] + A.bias[0]);
      } else {
#pragma unroll
        for (int j = 0; j < COUT / 8; ++j) {
          uint32_t w4[4];
          uint4 mk = make_uint4(0, 0, 0, 0);
          if (EPI == EPI_DX) mk = *reinterpret_cast<const uint4*>(A.mask + pix * COUT + 8 * j);
          const uint32_t mkw[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
          for (int h = 0; h < 4; ++h) {
            float a = v[8 * j + 2 * h], b = v[8 * j + 2 * h + 1];
            if (EPI == EPI_ACT) {
              a = fmaxf(a + A.bias[8 * j + 2 * h], 0.f);
              b = fmaxf(b + A.bias[8 * j + 2 * h + 1], 0.f);
            } else {  // gradient through the ReLU of the layer that produced `mask`
              if (bf2f((uint16_t)(mkw[h] & 0xffffu)) <= 0.f) a = 0.f;
              if (bf2f((uint16_t)(mkw[h] >> 16)) <= 0.f) b = 0.f;
            }
            w4[h] = (uint32_t)tc::bf16_bits(a) | ((uint32_t)tc::bf16_bits(b) << 16);
          }
          *reinterpret_cast<uint4*>(A.out + pix * COUT + 8 * j) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (*fail_s) break;
  }
  if (*fail_s && tid == 0 && A.err) atomicOr(A.err, 2);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TCOLS);
}

template <int CIN, int COUT, int EPI>
cudaError_t launch_conv_t(const ConvArgs& A, int sms, cudaStream_t st) {
  const size_t sm = (size_t)3 * (CIN / 8) * LBO_A + (size_t)9 * COUT * CIN * 2 + 64;
  cudaError_t e = cudaFuncSetAttribute(k_conv<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int tiles = A.nimg * A.H * ((A.W + TP - 1) / TP);
  const int grid = tiles < 2 * sms ? tiles : 2 * sms;
  k_conv<CIN, COUT, EPI><<<grid, 128, sm, st>>>(A);
  return cudaGetLastError();
}

// ---- input packing, weight layouts -------------------------------------------------

// NHWC bf16, 16 channels: noisy / 255, sigma / 255, zeros.
__global__ void k_pack_input(const float* __restrict__ img, const float* __restrict__ sig, int nimg, int H, int W,
                             uint16_t* __restrict__ out) {
  const size_t total = (size_t)nimg * H * W;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const int n = (int)(p / ((size_t)H * W));
    const uint32_t a = tc::bf16_bits(img[p] * (1.f / 255.f)), b = tc::bf16_bits(sig[n] * (1.f / 255.f));
    uint4* o = reinterpret_cast<uint4*>(out + p * 16);
    o[0] = make_uint4(a | (b << 16), 0, 0, 0);
    o[1] = make_uint4(0, 0, 0, 0);
  }
}

// master fp32 W [9][co_r][ci_r] -> bf16 [9][COUT][CIN] zero padded; with
// transpose, the data-gradient weights [9][CIN][COUT] of tap 8-t (flipped).
__global__ void k_pack_weights(const float* __restrict__ w, int co_r, int ci_r, int COUT, int CIN, int transpose,
                               uint16_t* __restrict__ out) {
  const int total = 9 * COUT * CIN;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int t = e / (COUT * CIN), r = e % (COUT * CIN);
    float v = 0.f;
    if (!transpose) {
      const int co = r / CIN, ci = r % CIN;
      if (co < co_r && ci < ci_r) v = w[((size_t)t * co_r + co) * ci_r + ci];
      out[e] = tc::bf16_bits(v);
    } else {
      // out[t][a][b] = W[8 - t][co = b][ci = a]: rows a are the forward input
      // channels (COUT here is the forward CIN), K index b the forward outputs
      const int a = r / CIN, b = r % CIN;
      if (b < co_r && a < ci_r) v = w[((size_t)(8 - t) * co_r + b) * ci_r + a];
      out[e] = tc::bf16_bits(v);
    }
  }
}

// ---- training ----------------------------------------------------------------------------

// loss = mean((pilot - target)^2); gradient on the last layer's output
// channel 0: d loss / d r = -255 * 2 (pilot - target) / P, stored bf16 NHWC
// (16 channels).  Per-block partial losses go to part[blockIdx.x].
__global__ void k_loss_grad(const float* __restrict__ pilot, const float* __restrict__ target, size_t P,
                            uint16_t* __restrict__ dy, float* __restrict__ part) {
  __shared__ float red[256];
  float acc = 0.f;
  const float sc = -255.f * 2.f / (float)P;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < P; p += (size_t)gridDim.x * blockDim.x) {
    const float e = pilot[p] - target[p];
    acc = fmaf(e, e, acc);
    uint4* o = reinterpret_cast<uint4*>(dy + p * 16);
    o[0] = make_uint4(tc::bf16_bits(sc * e), 0, 0, 0);
    o[1] = make_uint4(0, 0, 0, 0);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Weight and bias gradients of one layer on the tensor cores.  For tap
// t = (dy, dx), dW_t[co][ci] = sum_p g[p][co] x[p + (dy-1, dx-1)][ci] is a
// GEMM with M = co (padded to 128), N = ci and the pixels as K.  A CTA takes
// tiles of 128 pixels of one row (persistent over tiles, fixed assignment):
// g's tile and the input rows y-1, y, y+1 (with a one-pixel halo) sit in
// shared memory in the forward's activation layout (pixel-major inside 8-channel
// chunks), which read with pixels as K is the MN-major operand layout (core
// matrix = 8 pixels x 8 channels; K-adjacent cores 128 bytes apart, channel-
// adjacent ones a chunk apart), and tap dx is the row buffer read from pixel dx
// (a 16-byte shift).  D of all 9 taps stays in TMEM over the CTA's tiles; the
// centre tap also multiplies an all-ones channel, which gives the bias
// gradient.  Each CTA writes its partial sums (bf16 products, fp32
// accumulation) to part[blockIdx.x]; k_reduce_partials adds them in order, so
// training stays deterministic.
constexpr int WG_LBO_G = TP * 16;  // bytes of one 8-channel chunk of the gradient tile
template <int CI_R, int CO_R, int CIN, int COUT>
__global__ void __launch_bounds__(128) k_dweight_tc(const uint16_t* __restrict__ x, const uint16_t* __restrict__ g,
                                                    int nimg, int H, int W, float* __restrict__ part,
                                                    int* __restrict__ err) {
  constexpr int XCH = CIN / 8 + 2;           // input chunks + the ones chunk + a zero chunk
  constexpr int ROWX = XCH * LBO_A;          // bytes of one input row buffer
  constexpr int NCOL = 9 * CIN + 16;         // TMEM columns of the 9 taps (the centre one is 16 wider)
  constexpr int TCOLS = NCOL <= 256 ? 256 : 512;
  constexpr int E = 9 * CO_R * CI_R;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sG = smem;                  // 16 chunks (M = 128)
  unsigned char* sX = smem + 16 * WG_LBO_G;  // 3 row buffers
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sX + 3 * ROWX);
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(mbar + 1);
  int* fail_s = reinterpret_cast<int*>(taddr_s + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto col_of = [](int t) { return t <= 4 ? t * CIN : 5 * CIN + 16 + (t - 5) * CIN; };

  if (warp == 0) tc::tmem_alloc(taddr_s, TCOLS);
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
    *fail_s = 0;
  }
  // gradient chunks past COUT stay zero (rows co >= COUT of the M = 128 operand)
  for (int e = tid; e < (16 - COUT / 8) * WG_LBO_G / 16; e += 128)
    reinterpret_cast<uint4*>(sG + (COUT / 8) * WG_LBO_G)[e] = make_uint4(0, 0, 0, 0);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *taddr_s;
  const int xt_n = (W + TP - 1) / TP;
  const int ntiles = nimg * H * xt_n;
  uint32_t phase = 0;
  bool any = false;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int xt = tile % xt_n, y = (tile / xt_n) % H, n = tile / (xt_n * H);
    const int x0 = xt * TP;
    if (any) {  // the previous tile's MMAs read the buffers about to be rewritten
      const bool ok = tc::mbar_wait(mbar, phase, PWAIT);
      phase ^= 1u;
      if (!ok) *fail_s = 1;
      tc::fence_after_sync();
      __syncthreads();
      if (*fail_s) break;
    }
    for (int e = tid; e < TP * (COUT / 8); e += 128) {
      const int j = e / TP, q = e % TP, xx = x0 + q;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (xx < W) v = *reinterpret_cast<const uint4*>(g + (((size_t)n * H + y) * W + xx) * COUT + 8 * j);
      *reinterpret_cast<uint4*>(sG + j * WG_LBO_G + q * 16) = v;
    }
    for (int e = tid; e < 3 * NPX * XCH; e += 128) {
      const int r = e / (NPX * XCH), j = (e / NPX) % XCH, q = e % NPX;
      const int yy = y + r - 1, xx = x0 + q - 1;
      const bool in = yy >= 0 && yy < H && xx >= 0 && xx < W;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (in && j < CIN / 8) v = *reinterpret_cast<const uint4*>(x + (((size_t)n * H + yy) * W + xx) * CIN + 8 * j);
      else if (in && j == CIN / 8) v.x = 0x3F80u;  // bf16 1.0 in the first channel of the ones chunk
      *reinterpret_cast<uint4*>(sX + r * ROWX + j * LBO_A + q * 16) = v;
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t ga = tc::smem_u32(sG), xa = tc::smem_u32(sX);
#pragma unroll 1
      for (int t = 0; t < 9; ++t) {
        const int dy = t / 3, dx = t % 3;
        const uint32_t idesc = tc::idesc_bf16_f32(TP, t == 4 ? CIN + 16 : CIN) | (1u << 15) | (1u << 16);
#pragma unroll
        for (int ks = 0; ks < TP / 16; ++ks) {
          const uint64_t ad = tc::desc_kmajor(ga + ks * 256, 128, WG_LBO_G);
          const uint64_t bd = tc::desc_kmajor(xa + dy * ROWX + dx * 16 + ks * 256, 128, LBO_A);
          tc::mma_bf16(tmem + (uint32_t)col_of(t), ad, bd, idesc, (any || ks > 0) ? 1u : 0u);
        }
      }
      tc::commit(mbar);
    }
    any = true;
  }
  if (any && !*fail_s) {
    if (!tc::mbar_wait(mbar, phase, PWAIT)) *fail_s = 1;
    tc::fence_after_sync();
  }
  __syncthreads();
  const bool failed = *fail_s != 0;
  // ---- partial sums out: thread = co (TMEM lane), 32 columns at a time -------
  float* out = part + (size_t)blockIdx.x * (E + CO_R);
  const int co = warp * 32 + lane;
  for (int c0 = 0; c0 < NCOL; c0 += 32) {
    float v[32];
    tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
    if (co < CO_R) {
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const int c = c0 + q;
        const float val = (any && !failed) ? v[q] : 0.f;
        int t, ci;
        if (c < 4 * CIN) { t = c / CIN; ci = c % CIN; }
        else if (c < 5 * CIN + 16) { t = 4; ci = c - 4 * CIN; }
        else if (c < NCOL) { t = 5 + (c - 5 * CIN - 16) / CIN; ci = (c - 5 * CIN - 16) % CIN; }
        else continue;
        if (ci < CI_R) out[((size_t)t * CO_R + co) * CI_R + ci] = val;
        else if (t == 4 && ci == CIN) out[E + co] = val;  // the ones channel: bias gradient
      }
    }
  }
  if (failed && tid == 0 && err) atomicOr(err, 2);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TCOLS);
}

template <int CI_R, int CO_R, int CIN, int COUT>
cudaError_t launch_dweight_tc(const uint16_t* x, const uint16_t* g, int nimg, int H, int W, float* part, int grid,
                              int* err, cudaStream_t st) {
  const size_t sm = (size_t)16 * WG_LBO_G + (size_t)3 * (CIN / 8 + 2) * LBO_A + 64;
  cudaError_t e = cudaFuncSetAttribute(k_dweight_tc<CI_R, CO_R, CIN, COUT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k_dweight_tc<CI_R, CO_R, CIN, COUT><<<grid, 128, sm, st>>>(x, g, nimg, H, W, part, err);
  return cudaGetLastError();
}

__global__ void k_reduce_partials(const float* __restrict__ part, int nparts, int len, float* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < len; e += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < nparts; ++k) s += part[(size_t)k * len + e];
    out[e] = s;
  }
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
  }
}

}  // namespace

// ---- host-side network driver ------------------------------------------------------------

// parameter layout of the fp32 master vector: per layer W [9][co][ci] then b [co]
static const int kLayerCI[PILOT_LAYERS] = {2, 48, 48, 48, 48, 48, 48, 48};
static const int kLayerCO[PILOT_LAYERS] = {48, 48, 48, 48, 48, 48, 48, 1};

int pilot_param_count() {
  int n = 0;
  for (int l = 0; l < PILOT_LAYERS; ++l) n += 9 * kLayerCO[l] * kLayerCI[l] + kLayerCO[l];
  return n;
}

int pilot_param_offset(int layer) {
  int n = 0;
  for (int l = 0; l < layer; ++l) n += 9 * kLayerCO[l] * kLayerCI[l] + kLayerCO[l];
  return n;
}

static int pad16(int c) { return c <= 16 ? 16 : 48; }

cudaError_t pilot_pack_weights(const float* master, uint16_t* const* wfwd, uint16_t* const* wbwd, cudaStream_t st) {
  for (int l = 0; l < PILOT_LAYERS; ++l) {
    const int ci = kLayerCI[l], co = kLayerCO[l], CIN = pad16(ci), COUT = pad16(co);
    const float* w = master + pilot_param_offset(l);
    k_pack_weights<<<64, 256, 0, st>>>(w, co, ci, COUT, CIN, 0, wfwd[l]);
    if (wbwd && wbwd[l]) k_pack_weights<<<64, 256, 0, st>>>(w, co, ci, CIN, COUT, 1, wbwd[l]);
  }
  return cudaGetLastError();
}

cudaError_t pilot_pack_input(const float* img, const float* sig, int nimg, int H, int W, uint16_t* out,
                             cudaStream_t st) {
  k_pack_input<<<1024, 256, 0, st>>>(img, sig, nimg, H, W, out);
  return cudaGetLastError();
}

// Forward: acts[0] = packed input (16 ch), acts[l] = output of layer l (48 ch) for l = 1..7.
cudaError_t pilot_forward(const PilotNet& P, const float* img, int nimg, int H, int W, uint16_t* const* acts,
                          float* pilot, int* err, int sms, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  for (int l = 0; l < PILOT_LAYERS && e == cudaSuccess; ++l) {
    ConvArgs A{};
    A.in = acts[l];
    A.w = P.wfwd[l];
    A.bias = P.master + pilot_param_offset(l) + 9 * kLayerCO[l] * kLayerCI[l];
    A.nimg = nimg;
    A.H = H;
    A.W = W;
    A.err = err;
    if (l == 0) {
      A.out = acts[1];
      e = launch_conv_t<16, 48, EPI_ACT>(A, sms, st);
    } else if (l < PILOT_LAYERS - 1) {
      A.out = acts[l + 1];
      e = launch_conv_t<48, 48, EPI_ACT>(A, sms, st);
    } else {
      A.img = img;
      A.pilot = pilot;
      e = launch_conv_t<48, 16, EPI_OUT>(A, sms, st);
    }
  }
  return e;
}

// Backward after pilot_forward: gradients of mean((pilot - target)^2) with
// respect to the master parameters into grad (fp32, same layout).  gA, gB are
// two NHWC bf16 gradient buffers of 48 channels; dy16 holds 16 channels.
cudaError_t pilot_backward(const PilotNet& P, const float* pilot, const float* target, int nimg, int H, int W,
                           uint16_t* const* acts, uint16_t* dy16, uint16_t* gA, uint16_t* gB, float* part,
                           int nparts, float* grad, float* loss_part, int* err, int sms, cudaStream_t st) {
  const size_t Pn = (size_t)nimg * H * W;
  k_loss_grad<<<256, 256, 0, st>>>(pilot, target, Pn, dy16, loss_part);
  const int grid = nparts;
  const uint16_t* g = dy16;  // gradient on the current layer's (pre-activation) output
  uint16_t* bufs[2] = {gA, gB};
  int which = 0;
  for (int l = PILOT_LAYERS - 1; l >= 0; --l) {
    float* gl = grad + pilot_param_offset(l);
    const int len = 9 * kLayerCO[l] * kLayerCI[l] + kLayerCO[l];
    cudaError_t ew;
    if (l == PILOT_LAYERS - 1)
      ew = launch_dweight_tc<48, 1, 48, 16>(acts[l], g, nimg, H, W, part, grid, err, st);
    else if (l == 0)
      ew = launch_dweight_tc<2, 48, 16, 48>(acts[0], g, nimg, H, W, part, grid, err, st);
    else
      ew = launch_dweight_tc<48, 48, 48, 48>(acts[l], g, nimg, H, W, part, grid, err, st);
    if (ew != cudaSuccess) return ew;
    k_reduce_partials<<<64, 256, 0, st>>>(part, grid, len, gl);
    if (l == 0) break;
    // data gradient into the input of layer l, gated by that input's ReLU (acts[l])
    ConvArgs A{};
    A.in = g;
    A.w = P.wbwd[l];
    A.out = bufs[which];
    A.mask = acts[l];
    A.nimg = nimg;
    A.H = H;
    A.W = W;
    A.err = err;
    cudaError_t e = (l == PILOT_LAYERS - 1) ? launch_conv_t<16, 48, EPI_DX>(A, sms, st)
                                            : launch_conv_t<48, 48, EPI_DX>(A, sms, st);
    if (e != cudaSuccess) return e;
    g = bufs[which];
    which ^= 1;
  }
  return cudaGetLastError();
}

cudaError_t pilot_adam(float* w, const float* g, float* m1, float* m2, int n, float lr, int step, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<128, 256, 0, st>>>(w, g, m1, m2, n, lr, b1, b2, 1e-8f, c1, c2);
  return cudaGetLastError();
}

}  // namespace gbm3d
