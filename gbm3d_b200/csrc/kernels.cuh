// Launch interfaces of the GBM3D kernels (host side of each .cu file).
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace gbm3d {

// ---- column windows (the strip form) ------------------------------------------
// A circular range of columns [lo, lo + len) of an axis of length L, every
// index taken modulo L; len < 0 (or >= L): the whole axis; len 0: none.  The
// strip form restricts each stage to the columns its consumers read.
struct ColRange {
  int lo = 0, len = -1;
  bool all(int L) const { return len < 0 || len >= L; }
};
// The tiles of T columns (the last one partial) that hold every column of r:
// tiles t0, t0 + 1, ..., nt of them, modulo the tile count.  Whole axis: 0, count.
inline void tile_span(const ColRange& r, int L, int T, int& t0, int& nt) {
  const int ntile = (L + T - 1) / T;
  if (r.all(L)) {
    t0 = 0;
    nt = ntile;
    return;
  }
  if (r.len == 0) {
    t0 = nt = 0;
    return;
  }
  const int lo = ((r.lo % L) + L) % L, last = lo + r.len - 1;  // last may pass L: it wraps
  t0 = lo / T;
  nt = last < L ? last / T - t0 + 1 : (ntile - t0) + (last - L) / T + 1;
  if (nt >= ntile) t0 = 0, nt = ntile;
}
// Groups g = i + M j of the group columns r (N of them): g0 and the count gn
// (0: every group; -1: none).
inline void group_span(const ColRange& r, int M, int N, int& g0, int& gn) {
  if (r.all(N)) {
    g0 = gn = 0;
    return;
  }
  if (r.len == 0) {
    g0 = 0, gn = -1;
    return;
  }
  g0 = (((r.lo % N) + N) % N) * M;
  gn = r.len * M;
}
// Group of window slot gl (g0 + gl modulo G), or -1 past the window.
__host__ __device__ __forceinline__ int window_group(int gl, int g0, int gn, int G) {
  if (gl >= (gn > 0 ? gn : G)) return -1;
  const int g = gl + g0;
  return g >= G ? g - G : g;
}

// ---- block matching (match.cu) ----------------------------------------------
struct MatchArgs {
  const float* pad;   // padded search image of the matched image, pitch P
  const float* pad2;  // padded search image gathered into V2 (may be null)
  int P;              // column pitch of pad/pad2 in floats
  int M, N, K;        // reference grid and group size
  int s;              // reference stride: reference (i, j) sits at (i s, j s)
  int numMin;         // tolerance branch: minimum group size
  float tol;          // tolerance on ssd/||xR||^2
  int tol_branch;     // numMin != numMax
  uint32_t* S;        // K x M x N
  int32_t* cnt;       // M x N (may be null)
  float* volume;      // m x n x K gather (may be null); block (i, j) at rows i d, cols j d
  int m, n;           // volume rows/cols: the image for s = d, (M d) x (N d) otherwise
  float* V1;          // d x d x K x M x N gathers (may be null)
  float* V2;
  int* err;           // status word (may be null): bit 1 a tensor-core matcher wait ran out, bit 2
                      // the exhaustive matcher's wait for its search-window copy ran out
  int R, Q;           // rows and columns of the search image (m + d2, n + d2)
  // tensor-core matcher: references whose candidate set overflowed its list
  // are appended here (count first zeroed) and searched exhaustively after it
  int* ovf_list;
  int* ovf_count;
  // list mode of the exhaustive matcher: only the references list[0 .. *list_count)
  const int* list;
  const int* list_count;
  // tensor-core matcher: work queue counter (zeroed by the launch), limit of
  // every wait in SM clocks (0: about two seconds), and an optional histogram
  // of candidates per reference (33 buckets of 8, the last for >= 256)
  int* work;
  long long wait_cycles;
  int* cand_hist;
  // exhaustive matcher: only the groups g0 .. g0 + gn - 1 (modulo M N); gn 0: all
  int g0, gn;
};
bool match_supported(int d, int d2);
// 2-D fp32 tensor map of a search image (R rows, the inner dimension, of
// pitch P floats; Q columns) with a box of box_rows x box_cols, zero fill past
// its end, no multicast.  False when the driver's encoder is unavailable or
// the image is not TMA-addressable (16-byte aligned base, P a multiple of 4).
bool encode_search_map(CUtensorMap* tm, const float* pad, int R, int Q, int P, int box_rows, int box_cols);
cudaError_t launch_match(int d, int d2, const MatchArgs& A, cudaStream_t st);
cudaError_t launch_make_pad(const float* img, int m, int n, int d2, int spin, float* pad, int P,
                            cudaStream_t st);
cudaError_t launch_gather_volume(const float* pad, int P, int M, int N, int s, int d, int d2, int K, const uint32_t* S,
                                 const int32_t* cnt, float* vol, cudaStream_t st);
// The exhaustive matcher on the references A.list[0 .. *A.list_count) only
// (grid-stride over the list; the count is read on the device).
cudaError_t launch_match_list(int d, int d2, const MatchArgs& A, cudaStream_t st);
// Tensor-core matcher (match_tc.cu): bf16 tensor-core distances bound the
// candidates, exact FP32 re-rank in the exhaustive matcher's operation order,
// so the match sets equal its own.  Top-K branch only (numMin = numMax),
// d = 8, K <= 16, stride 1..8.  References whose candidate list overflows go
// to A.ovf_list; launch_match_list(A with list = ovf_list) finishes them.
bool match_tc_supported(int d, int d2, int s, int K, bool tol_branch);
// f16 selects f16 operands (tensor form) instead of bf16 (precision form).
cudaError_t launch_match_tc(int d, int d2, const MatchArgs& A, bool f16, cudaStream_t st);

// ---- step 1: global 3D wavelet hard thresholding (wavelet.cu) ----------------
struct WaveletBank {
  AxisBank xy, z;
  int reach_a;  // largest analysis tap index on the spatial axes
  int reach_s;  // largest synthesis tap index on the spatial axes
};
struct LevelBands {
  float tau[8];  // hard threshold per band code (code 0 unused)
};
// Analysis of one level + hard threshold.  in: Ly x Lx x Lz, read at
// ((y-shift) mod Ly, (x-shift) mod Lx, (z-shift) mod Lz).  out: 8 bands, band
// code fy + 2 fx + 4 fz, each (Ly/2)(Lx/2)(Lz/2) floats.
// qcols: the coefficient columns (of Lx / 2) to produce.
cudaError_t launch_wav_analysis(const float* in, int Ly, int Lx, int Lz, int shift, float* out,
                                const WaveletBank& bk, const LevelBands& th, cudaStream_t st,
                                const ColRange& qcols = ColRange());
// Synthesis of one level: bands (codes 1..7) + approx -> out (Oy x Ox x Oz).
// mode 0: out[p] = v; with shift_out, the value for p lands at p - shift_out.
// Level-1 cycle-spin accumulation: first (store) / middle (add) / last
// (add, divide by cycle count, clamp at 0).
struct SynthOut {
  float* out;
  int shift;
  int first, last;
  float cycles;
};
// cols: the output columns (values computed for p, before the shift) to produce.
cudaError_t launch_wav_synthesis(const float* bands, const float* approx, int Oy, int Ox, int Oz,
                                 const SynthOut& o, const WaveletBank& bk, cudaStream_t st,
                                 const ColRange& cols = ColRange());
// medfilt3 of the volume (filtType 'median').
cudaError_t launch_medfilt3(const float* V, int m, int n, int K, float* out, cudaStream_t st);
// Aggregation weight 1/(TV(group)+eps) per group of the image-shaped Vavg.
// jcols: the group columns (of N) to weigh.
cudaError_t launch_ht_weights(const float* Vavg, int m, int n, int M, int N, int d, int K,
                              const int32_t* cnt, float* wgt, cudaStream_t st, const ColRange& jcols = ColRange());

// ---- step 2: empirical Wiener (wiener.cu) --------------------------------------
struct WienerArgs {
  // group sources: either gathered from padded images through S, or read from
  // V1/V2 arrays (d x d x K x M x N)
  const float* padP;  // pilot search image (pitch P) or null
  const float* padN;  // noisy search image
  int P, d2;
  const float* V1;
  const float* V2;
  const uint32_t* S;
  int M, N, K;
  int s;              // reference stride
  float s2[256];      // sigma^2 per DCT coefficient (d x d), single precision
  float T[256];       // DCT-II matrix (d x d, column-major)
  float Ti[256];      // inverse used by the inverse transform
  int clamp_one;      // legacy variant: clamp to [0,1]
  float win[256];     // aggregation window w (d x d), single precision
  float* out;         // weighted filtered groups fl(wv .* block), d x d x K x M x N
  float* wt;          // per-group weights wv = fl(w / n2), d x d x M x N
  float* n2;          // ||filt||^2 per group (sqrt then square, single)
  int g0, gn;         // only the groups g0 .. g0 + gn - 1 (modulo M N); gn 0: all
};
bool wiener_supported(int d, int K);
cudaError_t launch_wiener(int d, const WienerArgs& A, cudaStream_t st);

// ---- owner-ordered aggregation (aggregate.cu) ------------------------------------
struct AggArgs {
  const uint32_t* S;
  const int32_t* cnt;   // may be null (every group holds K)
  int M, N, d, d2, K;
  int s;                // reference stride (block of reference (i, j) lands at (i s + a, j s + b))
  int kahan;            // 1: Kahan-compensated FP32 sums (precision form; d = 8 only)
  int wiener;           // 0: step-1 weights (scalar x mask); 1: step-2 (precomputed)
  const float* blocks;  // step 1: tile-space Vavg ((M d) x (N d) x K); step 2: weighted values, d x d x K per group
  const float* gw;      // step 1: weight per group; step 2: weight table, d x d per group
  float win[1024];      // step 1: mask (d x d)
  int m, n;             // output size (m = (M-1) s + d, n = (N-1) s + d)
  float* U;             // m x n
  float* W;
  ColRange cols;        // output columns to produce (whole CTA tiles; the rest of U, W is left as it is)
  int ct0;              // first CTA column tile (set by the launcher from cols)
};
cudaError_t launch_aggregate(const AggArgs& A, cudaStream_t st);

// ---- global matching (global_match.cu) ----------------------------------------------
struct GlobalMatchArgs {
  const float* I;  // m x n single image (prefiltered when sigma > 30/255)
  int m, n, M, N, K, numMin;
  float tol;
  int tol_branch;
  uint32_t* S;    // K x M x N, 1-based positions in the m x n image
  int32_t* cnt;   // M x N (may be null)
};
bool global_match_supported(int d, int K);
cudaError_t launch_match_global(int d, const GlobalMatchArgs& A, cudaStream_t st);
// in-place sym4 prefilter; work holds 8 * m * n floats
cudaError_t launch_sym4_prefilter(float* I, int m, int n, float tau, float* work, cudaStream_t st);

// ---- video (video.cu) ---------------------------------------------------------------------
struct VideoMatchArgs {
  const float* pads[32];  // search images of the window's frames (pitch P), circshifted as matched
  int P, M, N, F, K;      // references M x N (stride d), window of F frames, group size K
  int m, n;               // frame size (volume rows / columns)
  uint32_t* S;            // K x M x N, 1-based index a + b d + f d^2 into the d x d x F window
  float* volume;          // m x n x K
};
bool video_match_supported(int d, int F, int K);
cudaError_t launch_match_video(int d, const VideoMatchArgs& A, cudaStream_t st);
struct VideoAggArgs {
  const uint32_t* S;
  const float* wgt;       // weight per group
  const float* vsum;      // denoised volume, m x n x K
  int M, N, d, K, F, m, n;
  double* U;              // m x n x F
  double* W;
};
cudaError_t launch_aggregate_video(const VideoAggArgs& A, cudaStream_t st);
cudaError_t launch_clamp01(float* v, size_t n, cudaStream_t st);

// ---- learned pilot (pilot.cu) ----------------------------------------------------------
constexpr int PILOT_LAYERS = 8;
struct PilotNet {
  const float* master;           // fp32 parameters: per layer W [9][co][ci] then b [co]
  uint16_t* wfwd[PILOT_LAYERS];  // bf16 [9][COUT][CIN], channels padded to 16 / 48
  uint16_t* wbwd[PILOT_LAYERS];  // bf16 data-gradient weights (flipped taps, transposed channels)
};
int pilot_param_count();
int pilot_param_offset(int layer);
cudaError_t pilot_pack_weights(const float* master, uint16_t* const* wfwd, uint16_t* const* wbwd, cudaStream_t st);
cudaError_t pilot_pack_input(const float* img, const float* sig, int nimg, int H, int W, uint16_t* out,
                             cudaStream_t st);
cudaError_t pilot_forward(const PilotNet& P, const float* img, int nimg, int H, int W, uint16_t* const* acts,
                          float* pilot, int* err, int sms, cudaStream_t st);
cudaError_t pilot_backward(const PilotNet& P, const float* pilot, const float* target, int nimg, int H, int W,
                           uint16_t* const* acts, uint16_t* dy16, uint16_t* gA, uint16_t* gB, float* part,
                           int nparts, float* grad, float* loss_part, int* err, int sms, cudaStream_t st);
cudaError_t pilot_adam(float* w, const float* g, float* m1, float* m2, int n, float lr, int step, cudaStream_t st);

// ---- tensor-core self-check (tc_check.cu) -------------------------------------------
cudaError_t launch_tc_gemm_check(const uint16_t* A, const uint16_t* B, float* C, int* err, cudaStream_t st);
// The same product with both operands staged MN-major (the layout the pilot's
// weight gradient reads activations in).
cudaError_t launch_tc_gemm_check_mn(const uint16_t* A, const uint16_t* B, float* C, int* err, int swap_offsets,
                                    cudaStream_t st);

}  // namespace gbm3d
