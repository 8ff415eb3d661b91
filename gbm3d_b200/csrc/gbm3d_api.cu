// C ABI of the GBM3D library (include/gbm3d.h) and the device pipeline that
// restates source/GBM3D.m:15-83.
//
// Data stays on the device for the whole two-step pipeline: the image is
// uploaded once (double), converted to single and mirror-padded on the
// device, and only U (and optionally U1) come back.  The per-function entry
// points (matchBlocksCPU, denoiseAndAggregateGPU, matchBlocksWie,
// denoiseAndAggregateWieFast, denoiseAndAggregateWie) copy their host
// arguments in and their results out, so a MEX gateway can call them with
// mxArray data directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/gbm3d.h"
#include "common.cuh"
#include "kernels.cuh"

using namespace gbm3d;

struct gbm3d_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t st = nullptr;
  std::string err;
  std::map<std::string, std::pair<void*, size_t>> bufs;
  bool timing = false;
  std::vector<cudaEvent_t> evpool;           // events reused across calls
  std::vector<std::pair<int, int>> records;  // (stage, index of start event; end = +1)
  // per-launch timing: kpool[0] marks the call's start, kpool[i] is recorded
  // right after launch i (krec[i-1] names it), so on the in-order stream the
  // launch's device time is elapsed(kpool[i-1], kpool[i])
  std::vector<cudaEvent_t> kpool;
  std::vector<std::string> krec;
  int launches = 0;
  int form = 0;         // 0 plain, 1 precision, 2 learned pilot, 3 tensor-core matching (current call's options)
  bool pilot_ready = false;  // pilot parameters loaded (gbm3d_pilot_set_params)
  // the last batch captured as one CUDA graph, and the geometry it was captured for
  std::string graph_key;
  cudaGraphExec_t graph_exec = nullptr;
  int pilot_step = 0;        // Adam steps taken
  int sms = 148;
  int* flag = nullptr;  // device status word (non-finite input)
  // asynchronous host-buffer calls (gbm3d_denoise_async): two device slots for
  // input and output, one copy stream per direction, and the events that
  // order the copies of a slot with the compute that uses it
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t in_ready[2] = {}, in_free[2] = {}, out_ready[2] = {}, out_free[2] = {};
  int slot = 0;
  bool async_pending = false;
  int* sticky = nullptr;  // OR of the status words of the asynchronous calls since the last synchronisation
  long long tc_wait = 0;  // wait limit of the tensor-core matcher in SM clocks (0: about two seconds; < 0: probe)
  bool tc_stats = false;  // accumulate the tensor-core matcher's candidate histogram
  int* tc_hist = nullptr; // 33 buckets on the device
  // batched form: items of one submission run on `lanes` streams at once, each
  // lane with its own buffers (named with the lane's prefix `ns`)
  int lanes = 1;
  std::vector<cudaStream_t> lane_st;
  std::vector<cudaEvent_t> lane_ev;  // [0] fork, [1 + l] lane l done
  std::string ns;
};

namespace {

struct Fail {
  int code;
};

void set_err(gbm3d_ctx* c, const std::string& s) {
  if (c) c->err = s;
}

void ck(gbm3d_ctx* c, cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    set_err(c, std::string(what) + ": " + cudaGetErrorString(e));
    throw Fail{e == cudaErrorMemoryAllocation ? GBM3D_ERR_NOMEM : GBM3D_ERR_CUDA};
  }
}

void argfail(gbm3d_ctx* c, const std::string& s, int code = GBM3D_ERR_ARG) {
  set_err(c, s);
  throw Fail{code};
}

// Device status word: bit 0 non-finite input (k_prep), bit 1 a tensor-core
// matcher wait (TMA copy or MMA) that ran out of its limit (the kernel gave up),
// bit 2 the exhaustive matcher's wait for a search-window copy (likewise).
void report_flag(gbm3d_ctx* c, int flag) {
  if (flag & 1) argfail(c, "input image holds NaN or Inf", GBM3D_ERR_NONFINITE);
  if (flag & 2) argfail(c, "tensor-core matcher: a TMA copy or MMA did not complete within its wait limit", GBM3D_ERR_CUDA);
  if (flag & 4) argfail(c, "matcher: a search-window TMA copy did not complete within its wait limit", GBM3D_ERR_CUDA);
}

template <class T>
T* buf(gbm3d_ctx* c, const char* cname, size_t count) {
  const size_t bytes = std::max<size_t>(count * sizeof(T), 256);
  const std::string name = c->ns.empty() ? std::string(cname) : c->ns + cname;
  auto it = c->bufs.find(name);
  if (it != c->bufs.end() && it->second.second >= bytes) return reinterpret_cast<T*>(it->second.first);
  if (it != c->bufs.end()) {
    cudaFree(it->second.first);
    c->bufs.erase(it);
  }
  void* p = nullptr;
  ck(c, cudaMalloc(&p, bytes), name.c_str());
  c->bufs[name] = {p, bytes};
  return reinterpret_cast<T*>(p);
}

void kevent(gbm3d_ctx* c, size_t idx) {
  while (c->kpool.size() <= idx) {
    cudaEvent_t e;
    ck(c, cudaEventCreate(&e), "cudaEventCreate");
    c->kpool.push_back(e);
  }
  ck(c, cudaEventRecord(c->kpool[idx], c->st), "cudaEventRecord");
}

void launched(gbm3d_ctx* c, cudaError_t e, const char* what) {
  ck(c, e, what);
  ++c->launches;
  if (c->timing) {
    c->krec.push_back(what);
    kevent(c, c->krec.size());
  }
}

// Stage timer: records a start/end event pair on the stream when timing is on.
// Stages: 0 prepare, 1 step-1 matching, 2 step-1 wavelet, 3 step-1 aggregation,
// 4 step-2 matching, 5 step-2 Wiener, 6 step-2 aggregation, 7 whole call.
struct StageTimer {
  gbm3d_ctx* c;
  int idx = -1;
  StageTimer(gbm3d_ctx* cc, int stage) : c(cc) {
    if (!c->timing) return;
    idx = (int)c->records.size() * 2;
    while ((int)c->evpool.size() < idx + 2) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      c->evpool.push_back(e);
    }
    c->records.push_back({stage, idx});
    cudaEventRecord(c->evpool[idx], c->st);
  }
  ~StageTimer() {
    if (idx >= 0) cudaEventRecord(c->evpool[idx + 1], c->st);
  }
};

// ---- small host helpers shared with the option layer --------------------------

void sine_window(int d, double lo, double hi, double* w) {
  std::vector<double> v(d);
  for (int i = 0; i < d; ++i) {
    double t = (d == 1) ? hi : (i == d - 1 ? hi : lo + i * (hi - lo) / (d - 1));
    v[i] = std::sin(M_PI * t);
  }
  for (int c = 0; c < d; ++c)
    for (int r = 0; r < d; ++r) w[r + c * d] = v[r] * v[c];
}

// dct(eye(d)) and inv() of it (denoiseAndAggregateWieFast.m:33-34)
void dct_matrices(int d, double* Tm, double* Ti) {
  for (int k = 0; k < d; ++k)
    for (int n = 0; n < d; ++n) {
      double ck = (k == 0) ? std::sqrt(1.0 / d) : std::sqrt(2.0 / d);
      Tm[k + n * d] = ck * std::cos(M_PI * (2 * n + 1) * k / (2.0 * d));
    }
  std::vector<double> a(d * 2 * d);
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < 2 * d; ++c) a[r * 2 * d + c] = c < d ? Tm[r + c * d] : (c - d == r ? 1.0 : 0.0);
  for (int col = 0; col < d; ++col) {
    int piv = col;
    for (int r = col + 1; r < d; ++r)
      if (std::fabs(a[r * 2 * d + col]) > std::fabs(a[piv * 2 * d + col])) piv = r;
    if (piv != col)
      for (int c = 0; c < 2 * d; ++c) std::swap(a[col * 2 * d + c], a[piv * 2 * d + c]);
    double p = a[col * 2 * d + col];
    for (int c = 0; c < 2 * d; ++c) a[col * 2 * d + c] /= p;
    for (int r = 0; r < d; ++r) {
      if (r == col) continue;
      double f = a[r * 2 * d + col];
      if (f == 0.0) continue;
      for (int c = 0; c < 2 * d; ++c) a[r * 2 * d + c] -= f * a[col * 2 * d + c];
    }
  }
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < d; ++c) Ti[r + c * d] = a[r * 2 * d + d + c];
}

Taps make_taps(const double* h, int len) {
  Taps t{};
  t.n = 0;
  for (int k = 0; k < len && k < GBM3D_MAX_TAPS; ++k)
    if (h[k] != 0.0) {
      t.k[t.n] = k;
      t.h[t.n] = (float)h[k];
      ++t.n;
    }
  return t;
}

WaveletBank make_bank(gbm3d_ctx* c, const gbm3d_filters* f) {
  if (f->len_xy < 1 || f->len_xy > GBM3D_MAX_TAPS || f->len_z < 1 || f->len_z > GBM3D_MAX_TAPS)
    argfail(c, "filter length out of range");
  WaveletBank b{};
  b.xy.a[0] = make_taps(f->a_lo_xy, f->len_xy);
  b.xy.a[1] = make_taps(f->a_hi_xy, f->len_xy);
  b.xy.s[0] = make_taps(f->s_lo_xy, f->len_xy);
  b.xy.s[1] = make_taps(f->s_hi_xy, f->len_xy);
  b.z.a[0] = make_taps(f->a_lo_z, f->len_z);
  b.z.a[1] = make_taps(f->a_hi_z, f->len_z);
  b.z.s[0] = make_taps(f->s_lo_z, f->len_z);
  b.z.s[1] = make_taps(f->s_hi_z, f->len_z);
  b.reach_a = b.reach_s = 0;
  for (int x = 0; x < 2; ++x) {
    for (int u = 0; u < b.xy.a[x].n; ++u) b.reach_a = std::max(b.reach_a, b.xy.a[x].k[u]);
    for (int u = 0; u < b.xy.s[x].n; ++u) b.reach_s = std::max(b.reach_s, b.xy.s[x].k[u]);
    for (int u = 0; u < b.z.a[x].n; ++u)
      if (b.z.a[x].k[u] > 1) argfail(c, "slot-axis filters longer than 2 taps are not supported", GBM3D_ERR_UNSUPPORTED);
    for (int u = 0; u < b.z.s[x].n; ++u)
      if (b.z.s[x].k[u] > 1) argfail(c, "slot-axis filters longer than 2 taps are not supported", GBM3D_ERR_UNSUPPORTED);
  }
  return b;
}

void bior(gbm3d_filters* f) {
  std::memset(f, 0, sizeof(*f));
  const double Ca = 0.016572815184060, Cb = 0.121533978016438, Cc = std::sqrt(2.0) / 2;
  const double lo[10] = {Ca, -Ca, -Cb, Cb, Cc, Cc, Cb, -Cb, -Ca, Ca};
  const double shi[10] = {-Ca, -Ca, Cb, Cb, -Cc, Cc, -Cb, -Cb, Ca, Ca};
  f->len_xy = 10;
  for (int k = 0; k < 10; ++k) {
    f->a_lo_xy[k] = lo[k];
    f->s_hi_xy[k] = shi[k];
  }
  f->a_hi_xy[4] = -Cc;
  f->a_hi_xy[5] = Cc;
  f->s_lo_xy[4] = Cc;
  f->s_lo_xy[5] = Cc;
  f->len_z = 2;
  f->a_lo_z[0] = Cc; f->a_lo_z[1] = Cc; f->a_hi_z[0] = -Cc; f->a_hi_z[1] = Cc;
  f->s_lo_z[0] = Cc; f->s_lo_z[1] = Cc; f->s_hi_z[0] = -Cc; f->s_hi_z[1] = Cc;
}

// sym4 x Haar bank of the video path (getWaveFilters3D('sym','db',4,1),
// waveTransforms3D/getWaveFilters3D.m:6-33; VBM3D synthesises with the same
// filters): the published symlet-4 decomposition pair on the spatial axes.
void sym4haar(gbm3d_filters* f) {
  std::memset(f, 0, sizeof(*f));
  static const double lo[8] = {-0.07576571478927333, -0.02963552764599851, 0.49761866763201545, 0.8037387518059161,
                               0.29785779560527736, -0.09921954357684722, -0.012603967262037833, 0.0322231006040427};
  const double Cc = std::sqrt(2.0) / 2;
  f->len_xy = 8;
  for (int k = 0; k < 8; ++k) {
    f->a_lo_xy[k] = f->s_lo_xy[k] = lo[k];
    f->a_hi_xy[k] = f->s_hi_xy[k] = (k % 2 ? 1.0 : -1.0) * lo[7 - k];  // Hi_d(k) = (-1)^(k+1) Lo_d(7-k), 0-based
  }
  f->len_z = 2;
  f->a_lo_z[0] = f->a_lo_z[1] = f->s_lo_z[0] = f->s_lo_z[1] = Cc;
  f->a_hi_z[0] = f->s_hi_z[0] = -Cc;
  f->a_hi_z[1] = f->s_hi_z[1] = Cc;
}

void haar3d(gbm3d_filters* f);
void bior(gbm3d_filters* f);

void bank_of_opts(const gbm3d_opts* o, gbm3d_filters* f) {
  if (o->wavelet == 1) haar3d(f);
  else if (o->wavelet == 2) sym4haar(f);
  else bior(f);
}

// 3D Haar bank: the two-tap Haar pair on all three axes (opts.wavelet = 1).
void haar3d(gbm3d_filters* f) {
  std::memset(f, 0, sizeof(*f));
  const double Cc = std::sqrt(2.0) / 2;
  f->len_xy = 2;
  f->len_z = 2;
  double* lo[4] = {f->a_lo_xy, f->s_lo_xy, f->a_lo_z, f->s_lo_z};
  double* hi[4] = {f->a_hi_xy, f->s_hi_xy, f->a_hi_z, f->s_hi_z};
  for (int q = 0; q < 4; ++q) {
    lo[q][0] = Cc; lo[q][1] = Cc;
    hi[q][0] = -Cc; hi[q][1] = Cc;
  }
}

void tau_table(int levels, int mode, double* tau) {
  for (int j = 0; j < 7; ++j)
    for (int i = 0; i < levels; ++i) {
      double base = 3.3 - 0.3 * i, v = 0;
      switch (mode) {
        case 1: v = base; break;
        case 2: v = j < 3 ? base : (j < 6 ? base + 0.5 : base + 1.0); break;
        case 3: v = j < 3 ? base : (j < 6 ? base + 0.25 : base + 1.5); break;
        case 4: v = j < 3 ? 2.9 : (j < 6 ? 2.9 + 0.5 : 2.9 + 1.0); break;
        default: v = 0;
      }
      tau[i + levels * j] = v;
    }
}

// band code (fy + 2 fx + 4 fz) -> detail column j of tau (getWaveFilters3Dbior.m:39-46)
const int kDetailJ[8] = {-1, 0, 1, 3, 2, 4, 5, 6};

// ---- glue kernels --------------------------------------------------------------

// double m x n -> mirror-padded single M x N (myMirrorPadImage.m:3-8 then
// single(), matchBlocksCPU.m:31); flags non-finite input.
__global__ void k_prep(const double* __restrict__ I, int m, int n, float* __restrict__ out, int Mp, int Np,
                       int* flag) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= Mp || c >= Np) return;
  const int sr = r < m ? r : m - 1 - (r - m), sc = c < n ? c : n - 1 - (c - n);
  const double v = I[sr + (size_t)sc * m];
  if (!isfinite(v)) atomicOr(flag, 1);
  out[r + (size_t)c * Mp] = (float)v;
}

__global__ void k_f32_to_f64(const float* __restrict__ a, double* __restrict__ b, size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}

// acc[p] (+)= (double) v[(r+s) mod Mp, (c+s) mod Np]: circshift(.,[-s,-s]) then
// the running sum over spins (GBM3D.m:53-57,78-83).
// (r + s) mod L for r in [0, L): one conditional subtraction when 0 <= s <= L.
__device__ __forceinline__ int shift_index(int r, int s, int L) {
  if ((unsigned)s <= (unsigned)L) {
    const int t = r + s;
    return t >= L ? t - L : t;
  }
  return pmod(r + s, L);
}

// Both accumulators of one spin (U and W): acc += v shifted back by the spin.
__global__ void k_or_flag(const int* __restrict__ flag, int* __restrict__ sticky) { *sticky |= *flag; }

__global__ void k_accum2(const float* __restrict__ u, const float* __restrict__ w, int Mp, int Np, int s,
                         double* __restrict__ ua, double* __restrict__ wa, int first) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= Mp || c >= Np) return;
  const size_t src = shift_index(r, s, Mp) + (size_t)shift_index(c, s, Np) * Mp;
  const double x = (double)u[src], y = (double)w[src];
  const size_t o = r + (size_t)c * Mp;
  ua[o] = first ? x : ua[o] + x;
  wa[o] = first ? y : wa[o] + y;
}

__global__ void k_accum(const float* __restrict__ v, int Mp, int Np, int s, double* __restrict__ acc, int first) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= Mp || c >= Np) return;
  const double x = (double)v[pmod(r + s, Mp) + (size_t)pmod(c + s, Np) * Mp];
  const size_t o = r + (size_t)c * Mp;
  acc[o] = first ? x : acc[o] + x;
}

__global__ void k_shift_copy(const float* __restrict__ v, int Mp, int Np, int s, float* __restrict__ out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= Mp || c >= Np) return;
  out[r + (size_t)c * Mp] = v[pmod(r + s, Mp) + (size_t)pmod(c + s, Np) * Mp];
}

__global__ void k_add_f(const float* __restrict__ v, double* __restrict__ acc, size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) acc[i] = acc[i] + (double)v[i];
}

// out = a ./ b on the padded grid (double), its single copy, and the m x n crop.
__global__ void k_ratio(const double* __restrict__ a, const double* __restrict__ b, int Mp, int Np,
                        double* __restrict__ full, float* __restrict__ full_f, double* __restrict__ crop,
                        int m, int n) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= Mp || c >= Np) return;
  const size_t o = r + (size_t)c * Mp;
  const double v = a[o] / b[o];
  if (full) full[o] = v;
  if (full_f) full_f[o] = (float)v;
  if (crop && r < m && c < n) crop[r + (size_t)c * m] = v;
}

dim3 grid2(int rows, int cols) { return dim3((rows + 255) / 256, cols); }

// Opponent colour transform (Y, U, V) = A (R, G, B) with
// A = [1/3 1/3 1/3; 1/2 0 -1/2; 1/4 -1/2 1/4], and its inverse
// R = Y + U + 2V/3, G = Y - 4V/3, B = Y - U + 2V/3.  The chroma channels are
// carried with an offset of 128 so that they stay non-negative through the
// clamps at 0 of both steps (the offset only moves the coarse approximation,
// which is never thresholded).
__global__ void k_opp(const double* __restrict__ R, const double* __restrict__ G, const double* __restrict__ B,
                      size_t n, double* __restrict__ Y, double* __restrict__ U, double* __restrict__ V, int inverse) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double a = R[i], b = G[i], c = B[i];
    if (!inverse) {
      Y[i] = (a + b + c) / 3.0;
      U[i] = (a - c) / 2.0 + 128.0;
      V[i] = (a - 2.0 * b + c) / 4.0 + 128.0;
    } else {  // (a, b, c) = (Y, U + 128, V + 128)
      const double u = b - 128.0, v = c - 128.0;
      Y[i] = a + u + 2.0 * v / 3.0;
      U[i] = a - 4.0 * v / 3.0;
      V[i] = a - u + 2.0 * v / 3.0;
    }
  }
}

// ---- validation ------------------------------------------------------------------

void check_opts(gbm3d_ctx* c, const gbm3d_opts* o) {
  if (!o) argfail(c, "opts is NULL");
  if (o->numMax < 1 || o->numMax > 32) argfail(c, "numMax must be in 1..32");
  if (o->numMin < 1 || o->numMin > o->numMax) argfail(c, "numMin must be in 1..numMax");
  if (o->matchSize < 2 || (o->matchSize & 1)) argfail(c, "matchSize must be even");
  if (o->refStride < 0 || o->refStride > o->blockSize) argfail(c, "refStride must be in 1..blockSize (0: blockSize)");
  if (o->refStrideWie < 0 || o->refStrideWie > o->blockSizeWie)
    argfail(c, "refStrideWie must be in 1..blockSizeWie (0: blockSizeWie)");
  if (o->filtType != 0 && o->filtType != 1) argfail(c, "unrecognized filtering");  // denoiseAndAggregateGPU.m:54
  if (o->wavelet < 0 || o->wavelet > 2)
    argfail(c, "wavelet must be 0 (bior1.5 x Haar), 1 (3D Haar) or 2 (sym4 x Haar)");
  if (o->form < 0 || o->form > 3)
    argfail(c, "form must be 0 (plain), 1 (precision), 2 (learned pilot) or 3 (tensor-core matching)");
  if (o->form == 2 && !c->pilot_ready) argfail(c, "learned pilot: no parameters loaded (gbm3d_pilot_set_params)");
  c->form = o->form;
}

void check_match(gbm3d_ctx* c, int d, int d2, int K) {
  if (!match_supported(d, d2))
    argfail(c, "unsupported (blockSize, matchSize) pair for block matching: (" + std::to_string(d) + "," +
                   std::to_string(d2) + ")", GBM3D_ERR_UNSUPPORTED);
  if (d2 * d2 < K) argfail(c, "numMax exceeds the number of candidates");
}

int pitch4(int rows) { return (rows + 3) & ~3; }

// Reference stride of step 1 / step 2 (0 selects the block size, the
// reference's tiling) and the reference-grid size along an axis of L pixels.
int stride1(const gbm3d_opts* o) { return o->refStride > 0 ? o->refStride : o->blockSize; }
int stride2(const gbm3d_opts* o) { return o->refStrideWie > 0 ? o->refStrideWie : o->blockSizeWie; }
int grid_count(int L, int d, int s) { return (L - d) / s + 1; }

// Match sets and counts that come from the caller are checked on the host
// before any kernel indexes memory with them.
void check_match_set(gbm3d_ctx* c, const uint32_t* S, const int32_t* cnt, size_t groups, int K, int d2) {
  const uint32_t hi = (uint32_t)d2 * (uint32_t)d2;
  for (size_t g = 0; g < groups; ++g) {
    int nm = K;
    if (cnt) {
      nm = cnt[g];
      if (nm < 1 || nm > K) argfail(c, "S_count entry out of range 1..numMax");
    }
    for (int k = 0; k < nm; ++k) {
      const uint32_t v = S[g * K + k];
      if (v < 1 || v > hi) argfail(c, "S holds an index outside the matchSize x matchSize window");
    }
  }
}

// ---- pipelines ----------------------------------------------------------------------

// Block matching on a single-precision image already on the device.
// References at stride s; the volume is m x n x K for s = d (image-shaped,
// the reference's layout) and (M d) x (N d) x K otherwise.
void run_match(gbm3d_ctx* c, const float* img, const float* img2, int m, int n, int spin, int d, int d2,
               int K, int numMin, double sigma, uint32_t* S, int32_t* cnt, float* volume, float* V1,
               float* V2, const char* tag, int s, int form, const ColRange& jcols = ColRange()) {
  const int P = pitch4(m + d2);
  const std::string t(tag);
  float* pad = buf<float>(c, (t + ".pad").c_str(), (size_t)P * (n + d2));
  launched(c, launch_make_pad(img, m, n, d2, spin, pad, P, c->st), "make_pad");
  float* pad2 = nullptr;
  if (img2) {
    pad2 = buf<float>(c, (t + ".pad2").c_str(), (size_t)P * (n + d2));
    launched(c, launch_make_pad(img2, m, n, d2, spin, pad2, P, c->st), "make_pad");
  }
  MatchArgs A{};
  A.pad = pad;
  A.pad2 = pad2;
  A.P = P;
  A.M = grid_count(m, d, s);
  A.N = grid_count(n, d, s);
  A.K = K;
  A.s = s;
  A.numMin = numMin;
  A.tol = (float)(0.005 * sigma * sigma * d * d);
  A.tol_branch = numMin != K;
  A.S = S;
  A.cnt = cnt;
  A.volume = volume;
  A.m = s == d ? m : A.M * d;
  A.n = s == d ? n : A.N * d;
  A.V1 = V1;
  A.V2 = V2;
  A.err = c->flag;
  A.R = m + d2;
  A.Q = n + d2;
  group_span(jcols, A.M, A.N, A.g0, A.gn);  // the exhaustive matcher's window (strip form)
  if (form == 1 || form == 3) {
    // tensor-core distances (precision and tensor forms): the V1/V2 gathers of
    // matchBlocksWie are not produced by the tensor-core matcher, so that
    // entry point keeps the exhaustive search (with the same match sets)
    if (!match_tc_supported(d, d2, s, K, A.tol_branch != 0))
      argfail(c, "tensor-core matching needs blockSize 8, numMin = numMax <= 16, refStride <= 8 and "
                 "3 refStride + matchSize <= 56", GBM3D_ERR_UNSUPPORTED);
    if (!V1 && !V2 && !img2) {
      A.ovf_list = buf<int>(c, "mtc.ovf", (size_t)A.M * A.N);
      A.ovf_count = buf<int>(c, "mtc.novf", 1);
      A.work = buf<int>(c, "mtc.work", 1);
      A.wait_cycles = c->tc_wait;
      A.cand_hist = c->tc_stats ? c->tc_hist : nullptr;
      // precision form: bf16 operands; tensor form: f16 (a tighter bound, the same match sets)
      launched(c, launch_match_tc(d, d2, A, form == 3, c->st), "match_tc");
      // references whose candidate list overflowed: the exhaustive search
      MatchArgs L = A;
      L.list = A.ovf_list;
      L.list_count = A.ovf_count;
      launched(c, launch_match_list(d, d2, L, c->st), "match_redo");
      return;
    }
  }
  launched(c, launch_match(d, d2, A, c->st), "match");
}

// denoiseAndAggregateGPU on device buffers: vol is (M d) x (N d) x K and
// U, W are float ((M-1) s + d) x ((N-1) s + d).
// The cycle-spun 3D wavelet hard threshold (or medfilt3) of an m x n x K
// volume: Vavg = max(mean over cycle spins, 0), returned in "ht.vsum".
// Strip form: the columns each stage of one step-1 spin produces.
struct Spin1Cols {
  ColRange match, weights, agg;  // group columns matched and weighed; pixel columns aggregated
  std::vector<ColRange> an, sy;  // per level: analysis coefficient columns, synthesis output columns
};
struct Spin2Cols {
  ColRange groups, agg;  // group columns matched and filtered; pixel columns aggregated
};

float* run_wavelet_ht(gbm3d_ctx* c, const float* vol, int m, int n, int K, int levels, int cycleSpin,
                      const double* tau, const WaveletBank& bk, int filtType, const Spin1Cols* w = nullptr) {
  float* vsum = buf<float>(c, "ht.vsum", (size_t)m * n * K);
  if (filtType == 1) {  // medfilt3 instead of the wavelet (denoiseAndAggregateGPU.m:49-52)
    StageTimer tw(c, 2);
    launched(c, launch_medfilt3(vol, m, n, K, vsum, c->st), "medfilt3");
  } else {
  const int q = 1 << levels;
  if (levels < 1 || levels > GBM3D_MAX_LEVELS) argfail(c, "levels out of range");
  if (m % q || n % q || K % q)
    argfail(c, "image size and numMax must be divisible by 2^levels for the 3D wavelet");
  if (cycleSpin < 1) argfail(c, "cycleSpin must be >= 1");
  std::vector<float*> coef(levels), rec(levels);
  for (int lv = 0; lv < levels; ++lv) {
    const size_t insz = (size_t)(m >> lv) * (n >> lv) * (K >> lv);
    coef[lv] = buf<float>(c, ("ht.coef" + std::to_string(lv)).c_str(), insz);  // 8 bands = input size
    if (lv > 0) rec[lv] = buf<float>(c, ("ht.rec" + std::to_string(lv)).c_str(), insz);
  }
  std::vector<LevelBands> th(levels);
  for (int lv = 0; lv < levels; ++lv) {
    th[lv].tau[0] = 0.f;
    for (int code = 1; code < 8; ++code) th[lv].tau[code] = (float)tau[lv + levels * kDetailJ[code]];
  }
  {
  StageTimer tw(c, 2);
  for (int s = 0; s < cycleSpin; ++s) {
    for (int lv = 0; lv < levels; ++lv) {
      const float* in = lv == 0 ? vol : coef[lv - 1];
      launched(c, launch_wav_analysis(in, m >> lv, n >> lv, K >> lv, lv == 0 ? s : 0, coef[lv], bk, th[lv], c->st,
                                      w ? w->an[lv] : ColRange()),
               "wav_analysis");
    }
    for (int lv = levels - 1; lv >= 0; --lv) {
      const float* approx = lv == levels - 1 ? coef[lv] : rec[lv + 1];
      SynthOut o{};
      if (lv == 0) {
        o.out = vsum;
        o.shift = s;
        o.first = s == 0;
        o.last = s == cycleSpin - 1;
        o.cycles = (float)cycleSpin;
      } else {
        o.out = rec[lv];
        o.shift = 0;
        o.first = 1;
        o.last = 0;
        o.cycles = 1.f;
      }
      launched(c, launch_wav_synthesis(coef[lv], approx, m >> lv, n >> lv, K >> lv, o, bk, c->st,
                                       w ? w->sy[lv] : ColRange()),
               "wav_synthesis");
    }
  }
  }
  }
  return vsum;
}

void run_ht(gbm3d_ctx* c, const float* vol, const uint32_t* S, const int32_t* cnt, int M, int N, int d,
            int d2, int K, int levels, int cycleSpin, const double* tau, const WaveletBank& bk, float* U,
            float* W, int filtType, int s, const Spin1Cols* w = nullptr) {
  const int m = M * d, n = N * d;
  float* vsum = run_wavelet_ht(c, vol, m, n, K, levels, cycleSpin, tau, bk, filtType, w);
  StageTimer tagg(c, 3);
  float* wgt = buf<float>(c, "ht.wgt", (size_t)M * N);
  launched(c, launch_ht_weights(vsum, m, n, M, N, d, K, cnt, wgt, c->st, w ? w->weights : ColRange()), "ht_weights");
  AggArgs A{};
  A.S = S;
  A.cnt = cnt;
  A.M = M;
  A.N = N;
  A.d = d;
  A.d2 = d2;
  A.K = K;
  A.wiener = 0;
  A.blocks = vsum;
  A.gw = wgt;
  std::vector<double> mk(d * d);
  sine_window(d, 0.1, 0.9, mk.data());
  for (int e = 0; e < d * d; ++e) A.win[e] = (float)mk[e];
  A.kahan = c->form == 1;
  A.s = s;
  A.m = (M - 1) * s + d;
  A.n = (N - 1) * s + d;
  A.U = U;
  A.W = W;
  if (w) A.cols = w->agg;
  launched(c, launch_aggregate(A, c->st), "aggregate");
}

void fill_wiener_consts(WienerArgs& A, int d, const double* sigma, int is_matrix, int variant) {
  std::vector<double> Tm(d * d), Ti(d * d), wk(d * d);
  dct_matrices(d, Tm.data(), Ti.data());
  sine_window(d, 0.2, 0.8, wk.data());  // w = outer(sin(pi*linspace(.2,.8,d))) (denoiseAndAggregateWieFast.m:73-76)
  for (int e = 0; e < d * d; ++e) A.win[e] = (float)wk[e];
  for (int e = 0; e < d * d; ++e) {
    A.T[e] = (float)Tm[e];
    A.Ti[e] = variant == 0 ? (float)Ti[e] : (float)Tm[(e / d) + (e % d) * d];
    const double s = is_matrix ? sigma[e] : sigma[0];
    A.s2[e] = (float)(s * s);
  }
  A.clamp_one = variant == 1;
}

// Strip form: cols the aggregated pixel columns and cnt the per-group counts
// (K inside the filtered window, 0 outside); A.g0 / A.gn set the window.
void run_wiener_agg(gbm3d_ctx* c, WienerArgs& A, int d, int d2, float* U, float* W,
                    const ColRange& cols = ColRange(), const int32_t* cnt = nullptr) {
  const int M = A.M, N = A.N, K = A.K;
  if (!wiener_supported(d, K))
    argfail(c, "unsupported (blockSizeWie, numMax) pair for the Wiener step", GBM3D_ERR_UNSUPPORTED);
  A.out = buf<float>(c, "wie.out", (size_t)d * d * K * M * N);
  A.wt = buf<float>(c, "wie.wt", (size_t)d * d * M * N);
  A.n2 = buf<float>(c, "wie.n2", (size_t)M * N);
  {
    StageTimer t(c, 5);
    launched(c, launch_wiener(d, A, c->st), "wiener");
  }
  StageTimer t(c, 6);
  AggArgs G{};
  G.S = A.S;
  G.cnt = cnt;
  G.M = M;
  G.N = N;
  G.d = d;
  G.d2 = d2;
  G.K = K;
  G.wiener = 1;
  G.blocks = A.out;
  G.gw = A.wt;
  G.s = A.s;
  G.kahan = c->form == 1;
  G.m = (M - 1) * A.s + d;
  G.n = (N - 1) * A.s + d;
  G.U = U;
  G.W = W;
  G.cols = cols;
  launched(c, launch_aggregate(G, c->st), "aggregate");
}

void to_host_double(gbm3d_ctx* c, const float* dsrc, size_t n, double* host) {
  double* tmp = buf<double>(c, "io.f64", n);
  k_f32_to_f64<<<(unsigned)((n + 255) / 256), 256, 0, c->st>>>(dsrc, tmp, n);
  launched(c, cudaGetLastError(), "f32_to_f64");
  ck(c, cudaMemcpyAsync(host, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, c->st), "D2H");
}

template <class F>
int guarded(gbm3d_ctx* c, F&& f) {
  if (!c) return GBM3D_ERR_ARG;
  c->err.clear();
  try {
    ck(c, cudaSetDevice(c->device), "cudaSetDevice");
    c->launches = 0;
    c->form = 0;
    c->records.clear();
    c->krec.clear();
    if (c->timing) kevent(c, 0);
    f();
    return GBM3D_OK;
  } catch (const Fail& e) {
    return e.code;
  } catch (const std::exception& e) {
    set_err(c, e.what());
    return GBM3D_ERR_CUDA;
  }
}

void opts_dims(const gbm3d_opts* o, int& d, int& dw, int& d2, int& K) {
  d = o->blockSize;
  dw = o->blockSizeWie;
  d2 = o->matchSize;
  K = o->numMax;
}

// The whole GBM3D.m pipeline on device buffers.
// ---- learned pilot state -----------------------------------------------------------

PilotNet pilot_net(gbm3d_ctx* c) {
  PilotNet P{};
  P.master = buf<float>(c, "pl.master", pilot_param_count());
  static const int co[PILOT_LAYERS] = {48, 48, 48, 48, 48, 48, 48, 16}, ci[PILOT_LAYERS] = {16, 48, 48, 48, 48, 48, 48, 48};
  for (int l = 0; l < PILOT_LAYERS; ++l) {
    P.wfwd[l] = buf<uint16_t>(c, ("pl.wf" + std::to_string(l)).c_str(), (size_t)9 * co[l] * ci[l]);
    P.wbwd[l] = buf<uint16_t>(c, ("pl.wb" + std::to_string(l)).c_str(), (size_t)9 * co[l] * ci[l]);
  }
  return P;
}

// NHWC activation buffers: acts[0] 16 channels, acts[1..7] 48 channels
void pilot_acts(gbm3d_ctx* c, size_t px, uint16_t** acts) {
  acts[0] = buf<uint16_t>(c, "pl.a0", px * 16);
  for (int l = 1; l < PILOT_LAYERS; ++l) acts[l] = buf<uint16_t>(c, ("pl.a" + std::to_string(l)).c_str(), px * 48);
}

void check_pilot_dims(gbm3d_ctx* c, int nimg, int H, int W) {
  if (!c->pilot_ready) argfail(c, "learned pilot: no parameters loaded (gbm3d_pilot_set_params)");
  if (nimg < 1 || H < 1 || W < 1 || (size_t)nimg * H * W > ((size_t)1 << 31)) argfail(c, "pilot: image sizes out of range");
}

// pilot (fp32, [image][row][column]) of nimg noisy images of H x W, sigma per image (device)
void run_pilot(gbm3d_ctx* c, const float* img, const float* sig, int nimg, int H, int W, float* out) {
  const size_t px = (size_t)nimg * H * W;
  uint16_t* acts[PILOT_LAYERS];
  pilot_acts(c, px, acts);
  launched(c, pilot_pack_input(img, sig, nimg, H, W, acts[0], c->st), "pilot_pack");
  launched(c, pilot_forward(pilot_net(c), img, nimg, H, W, acts, out, c->flag, c->sms, c->st), "pilot_conv");
}

__global__ void k_crop_f2d(const float* __restrict__ v, int Mp, double* __restrict__ out, int m, int n) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, col = blockIdx.y;
  if (r < m && col < n) out[r + (size_t)col * m] = (double)v[r + (size_t)col * Mp];
}

__global__ void k_fill_f(float* __restrict__ p, float v) { p[0] = v; }

// Strip form, step 2: count K for the groups of the filtered window (group
// columns lo .. lo + len - 1 modulo N), 0 elsewhere, so that the aggregation
// takes nothing from groups this call did not match.
__global__ void k_window_counts(int32_t* __restrict__ cnt, int M, int N, int lo, int len, int K) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= M * N) return;
  const int dj = g / M - lo;
  cnt[g] = (dj < 0 ? dj + N : dj) < len ? K : 0;
}

// ---- the strip form: which columns each stage must produce ---------------------------
//
// A caller that wants output columns [c_lo, c_hi) only (one GPU's share of a
// single image) runs every stage on the full-size buffers but restricted to the
// columns its consumers read, walking the dependencies back from the output:
// spin shifts (GBM3D.m:53-57,78-83), aggregation reach (a group's blocks land
// within its search window, denoiseAndAggregateGPU.m:70-89), search windows
// (matchBlocksCPU.m:57-79), and the 3D wavelet's circular filters per level
// and cycle spin (denoiseAndAggregateGPU.m:27-47).  Every produced column is
// computed from the same inputs as in the whole-image call, so the strip is
// bit-identical to the same columns of that call.  Sets are circular column
// masks; each stage gets the smallest circular range that covers its mask.
using ColMask = std::vector<char>;

ColRange cover(const ColMask& m) {
  const int L = (int)m.size();
  bool any = false;
  int best = 0, best_end = 0, run = 0;  // longest circular run of unneeded columns
  for (int t = 0; t < 2 * L; ++t) {
    if (m[t % L]) {
      any = true;
      run = 0;
    } else if (++run > best && run <= L) {
      best = run;
      best_end = t + 1;
    }
  }
  if (!any) return ColRange{0, 0};
  if (best == 0) return ColRange{0, -1};
  return ColRange{best_end % L, L - best};
}
// mark [a, b] (inclusive, any integers) modulo the mask length
void mark(ColMask& m, int a, int b) {
  const int L = (int)m.size();
  if (b - a + 1 >= L) {
    std::fill(m.begin(), m.end(), 1);
    return;
  }
  for (int x = a; x <= b; ++x) m[pmod(x, L)] = 1;
}
ColMask shifted(const ColMask& m, int s) {  // {(c + s) mod L : c in m}
  const int L = (int)m.size();
  ColMask o(L, 0);
  for (int c = 0; c < L; ++c)
    if (m[c]) o[pmod(c + s, L)] = 1;
  return o;
}
// Groups (of N, stride s, patch D) whose blocks can land on a needed pixel
// column: a block of group j starts at column j s - h + b, b in 0 .. d2 - 1.
ColMask groups_reaching(const ColMask& px, int N, int s, int D, int d2) {
  const int L = (int)px.size(), h = d2 / 2;
  std::vector<int> pre(L + 1, 0);
  for (int c = 0; c < L; ++c) pre[c + 1] = pre[c] + (px[c] ? 1 : 0);
  ColMask g(N, 0);
  for (int j = 0; j < N; ++j) {
    const int a = std::max(0, j * s - h - 1), b = std::min(L, j * s - h + d2 + D);
    g[j] = b > a && pre[b] > pre[a];
  }
  return g;
}

struct StripCols {
  std::vector<Spin1Cols> s1;
  std::vector<Spin2Cols> s2;
};

// Columns per stage for output columns [c_lo, c_hi) of the Mp x Np padded grid.
StripCols strip_cols(const gbm3d_opts* o, int Mp, int Np, int d, int dw, int d2, int st1, int st2, int c_lo,
                     int c_hi, const WaveletBank& bk) {
  (void)Mp;
  const int nS = o->nMatchSpins, nW = o->Wiener ? o->nMatchSpinsWie : 0, h = d2 / 2;
  const bool stale = o->form != 2 && o->Wiener && o->staleWeights && nW < nS;
  StripCols P;
  ColMask out(Np, 0);
  for (int x = c_lo; x < c_hi; ++x) out[x] = 1;
  ColMask u1 = out;  // step-1 estimate columns needed (its own strip, and the step-2 search windows)
  // step 2: spin shift -> aggregation -> groups -> pilot search windows
  const int N2 = grid_count(Np, dw, st2);
  for (int ii = 0; ii < nW; ++ii) {
    const int sp = o->matchSpinsWie[ii];
    const ColMask a2 = shifted(out, sp);
    const ColMask g2 = groups_reaching(a2, N2, st2, dw, d2);
    P.s2.push_back(Spin2Cols{cover(g2), cover(a2)});
    for (int j = 0; j < N2; ++j) {
      if (!g2[j]) continue;
      for (int q = std::max(0, j * st2 - 1); q < std::min(Np + d2, j * st2 + d2 + dw + 1); ++q)
        u1[pmod(pad_index(q, Np, h) - sp, Np)] = 1;
    }
  }
  if (o->form == 2) return P;  // the learned pilot runs on the whole image
  // step 1: spin shift -> aggregation -> groups -> denoised volume -> wavelet -> matched volume
  const int N1 = grid_count(Np, d, st1), n0 = N1 * d, levels = o->levels;
  for (int ii = 0; ii < nS; ++ii) {
    const int sp = o->matchSpins[ii];
    ColMask a1 = shifted(u1, sp);
    if (stale && ii >= nW) {  // this spin's weights also join the step-2 denominator
      const ColMask extra = shifted(out, sp);
      for (int x = 0; x < Np; ++x) a1[x] |= extra[x];
    }
    const ColMask g1 = groups_reaching(a1, N1, st1, d, d2);
    ColMask vs(n0, 0);  // denoised-volume (mosaic) columns the weights and the aggregation read
    for (int j = 0; j < N1; ++j)
      if (g1[j]) mark(vs, j * d, j * d + d - 1);
    ColMask vol(n0, 0);  // matched-volume columns
    Spin1Cols w;
    if (o->filtType == 1) {
      for (int x = 0; x < n0; ++x)
        if (vs[x]) mark(vol, x - 2, x + 2);
    } else {
      std::vector<ColMask> an(levels), sy(levels);
      for (int lv = 0; lv < levels; ++lv) {
        an[lv].assign(n0 >> (lv + 1), 0);
        sy[lv].assign(n0 >> lv, 0);
      }
      const int RS = bk.reach_s + 1, RA = bk.reach_a + 1;
      for (int sc = 0; sc < o->cycleSpin; ++sc) {
        // synthesis, level 0 up: outputs computed at p land at p - shift (shift sc at level 0)
        std::vector<ColMask> coef(levels);
        ColMask p = shifted(vs, sc);
        for (int lv = 0; lv < levels; ++lv) {
          for (int x = 0; x < (int)p.size(); ++x) sy[lv][x] |= p[x];
          ColMask q(n0 >> (lv + 1), 0);
          for (int x = 0; x < (int)p.size(); ++x)
            if (p[x]) mark(q, x / 2 - 2, (x + RS) / 2 + 2);
          coef[lv] = q;  // bands of level lv (and, at the top, the approximation)
          p = q;         // the approximation rec[lv + 1] the level below needs
        }
        // analysis, top level down: coefficient q reads inputs 2q - reach - shift .. 2q + 1 - shift
        ColMask need = coef[levels - 1];
        for (int lv = levels - 1; lv >= 0; --lv) {
          for (int x = 0; x < (int)need.size(); ++x) an[lv][x] |= need[x];
          const int sh = lv == 0 ? sc : 0;
          ColMask in(n0 >> lv, 0);
          for (int x = 0; x < (int)need.size(); ++x)
            if (need[x]) mark(in, 2 * x - RA - sh - 1, 2 * x + 2 - sh);
          if (lv == 0) {
            for (int x = 0; x < n0; ++x) vol[x] |= in[x];
          } else {
            need = coef[lv - 1];
            for (int x = 0; x < (int)in.size(); ++x) need[x] |= in[x];
          }
        }
      }
      for (int lv = 0; lv < levels; ++lv) {
        w.an.push_back(cover(an[lv]));
        w.sy.push_back(cover(sy[lv]));
      }
    }
    ColMask gm = g1;  // matched groups: the aggregated ones and every one the wavelet reads
    for (int x = 0; x < n0; ++x)
      if (vol[x]) gm[x / d] = 1;
    w.match = cover(gm);
    w.weights = cover(g1);
    w.agg = cover(a1);
    P.s1.push_back(w);
  }
  return P;
}

// Padded size along an axis of L pixels.  GBM3D.m:21-25 pads to a multiple of
// blockSize; with other strides, to the smallest size whose references of both
// steps end exactly at the border.  Such a size exists iff d = dw modulo
// gcd(st1, st2); then the search ends within lcm(st1, st2) steps.
int padded_size(const gbm3d_opts* o, int L, int d, int dw, int st1, int st2) {
  if (st1 == d && (!o->Wiener || (st2 == dw && d % dw == 0))) return (L + d - 1) / d * d;
  int p = std::max(L, std::max(d, dw));
  while ((p - d) % st1 != 0 || (o->Wiener && (p - dw) % st2 != 0)) ++p;
  return p;
}

// tau_in (levels x 7) and sigwie_in (blockSizeWie^2) replace sigma * getTau
// and the scalar Wiener sigma on the coloured-noise path (GBM3D.m:30-36);
// sigma is then what the matchers use, mean(sqrt(sigmaPSD)).
// strip (c_lo < c_hi): only output columns [c_lo, c_hi) of dU are exact (the
// strip form); the rest of dU holds whatever the restricted stages left there.
void pipeline(gbm3d_ctx* c, const double* dI, int m, int n, double sigma, const gbm3d_opts* o, double* dU,
              double* dU1, const double* tau_in = nullptr, const double* sigwie_in = nullptr, int c_lo = 0,
              int c_hi = 0) {
  check_opts(c, o);
  int d, dw, d2, K;
  opts_dims(o, d, dw, d2, K);
  check_match(c, d, d2, K);
  if (o->Wiener) check_match(c, dw, d2, K);
  if (m < 1 || n < 1 || m > 32000 || n > 32000) argfail(c, "image size out of range");
  if (!(sigma >= 0) || !std::isfinite(sigma)) argfail(c, "sigma must be a finite non-negative scalar");
  const int st1 = stride1(o), st2 = stride2(o);
  if (o->Wiener && (d - dw) % std::gcd(st1, st2) != 0)
    argfail(c, "no padded size lets both reference grids end at the border: blockSize - blockSizeWie must be "
               "a multiple of gcd(refStride, refStrideWie)", GBM3D_ERR_UNSUPPORTED);
  const int Mp = padded_size(o, m, d, dw, st1, st2), Np = padded_size(o, n, d, dw, st1, st2);
  if (Mp - m > m || Np - n > n) argfail(c, "image smaller than the padding it needs");
  if (Mp < d2 || Np < d2) argfail(c, "image smaller than matchSize");
  const int nS = o->nMatchSpins, nW = o->Wiener ? o->nMatchSpinsWie : 0;
  if (nS < 1 || nS > 8 || nW < 0 || nW > 8 || (o->Wiener && nW < 1)) argfail(c, "match spin count out of range");
  const size_t px = (size_t)Mp * Np;
  gbm3d_filters f;
  bank_of_opts(o, &f);
  const WaveletBank bk = make_bank(c, &f);
  std::vector<double> tau(o->levels * 7);
  tau_table(o->levels, o->tauMode, tau.data());
  for (auto& t : tau) t *= sigma;
  if (tau_in) std::copy(tau_in, tau_in + o->levels * 7, tau.begin());
  const bool strip = c_lo < c_hi;
  StripCols plan;
  if (strip) {
    if (o->form == 1 || o->form == 3)
      argfail(c, "the strip form runs the exhaustive matcher (forms 0 and 2)", GBM3D_ERR_UNSUPPORTED);
    if (c_lo < 0 || c_hi > n) argfail(c, "strip columns out of range");
    plan = strip_cols(o, Mp, Np, d, dw, d2, st1, st2, c_lo, c_hi, bk);
  }

  StageTimer tall(c, 7);
  float* If = buf<float>(c, "p.If", px);
  {
    StageTimer t(c, 0);
    ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
    k_prep<<<grid2(Mp, Np), 256, 0, c->st>>>(dI, m, n, If, Mp, Np, c->flag);
    launched(c, cudaGetLastError(), "prep");
  }

  float* Us = buf<float>(c, "p.Us", px);
  float* Ws = buf<float>(c, "p.Ws", px);
  double* Ua = buf<double>(c, "p.Ua", px);
  double* Wa = buf<double>(c, "p.Wa", px);
  double* U1d = buf<double>(c, "p.U1d", px);
  float* U1f = buf<float>(c, "p.U1f", px);
  const bool stale = o->form != 2 && o->Wiener && o->staleWeights && nW < nS;
  float* Wstale = stale ? buf<float>(c, "p.Wstale", px * (nS - nW)) : nullptr;
  if (o->form == 2) {
    // learned pilot in place of step 1: the padded image, column-major Mp x Np,
    // is the network's [Np rows][Mp columns] image
    float* sg = buf<float>(c, "pl.sig1", 1);
    k_fill_f<<<1, 1, 0, c->st>>>(sg, (float)sigma);
    launched(c, cudaGetLastError(), "fill");
    {
      StageTimer t(c, 2);
      run_pilot(c, If, sg, 1, Np, Mp, U1f);
    }
    if (dU1) {
      k_crop_f2d<<<grid2(m, n), 256, 0, c->st>>>(U1f, Mp, dU1, m, n);
      launched(c, cudaGetLastError(), "crop");
    }
    if (!o->Wiener) {
      k_crop_f2d<<<grid2(m, n), 256, 0, c->st>>>(U1f, Mp, dU, m, n);
      launched(c, cudaGetLastError(), "crop");
      return;
    }
  } else {
  // step 1: hard-thresholding estimate over the match spins
  const int M1 = grid_count(Mp, d, st1), N1 = grid_count(Np, d, st1);
  uint32_t* S1 = buf<uint32_t>(c, "p.S1", (size_t)K * M1 * N1);
  int32_t* cnt1 = buf<int32_t>(c, "p.cnt1", (size_t)M1 * N1);
  float* vol = buf<float>(c, "p.vol", (size_t)M1 * d * N1 * d * K);
  for (int ii = 0; ii < nS; ++ii) {
    const int s = o->matchSpins[ii];
    {
      StageTimer t(c, 1);
      // strip form: groups this spin does not match count 0, so the aggregation skips them
      if (strip) ck(c, cudaMemsetAsync(cnt1, 0, sizeof(int32_t) * M1 * N1, c->st), "memset");
      run_match(c, If, nullptr, Mp, Np, s, d, d2, K, o->numMin, sigma, S1, cnt1, vol, nullptr, nullptr, "m1", st1,
                o->form, strip ? plan.s1[ii].match : ColRange());
    }
    run_ht(c, vol, S1, cnt1, M1, N1, d, d2, K, o->levels, o->cycleSpin, tau.data(), bk, Us, Ws, o->filtType, st1,
           strip ? &plan.s1[ii] : nullptr);
    k_accum2<<<grid2(Mp, Np), 256, 0, c->st>>>(Us, Ws, Mp, Np, s, Ua, Wa, ii == 0);
    launched(c, cudaGetLastError(), "accum");
    if (stale && ii >= nW) {
      k_shift_copy<<<grid2(Mp, Np), 256, 0, c->st>>>(Ws, Mp, Np, s, Wstale + (size_t)(ii - nW) * px);
      launched(c, cudaGetLastError(), "shift_copy");
    }
  }
  k_ratio<<<grid2(Mp, Np), 256, 0, c->st>>>(Ua, Wa, Mp, Np, U1d, U1f, dU1, m, n);
  launched(c, cudaGetLastError(), "ratio");
  if (!o->Wiener) {
    k_ratio<<<grid2(Mp, Np), 256, 0, c->st>>>(Ua, Wa, Mp, Np, nullptr, nullptr, dU, m, n);
    launched(c, cudaGetLastError(), "ratio");
    return;
  }
  }

  // step 2: empirical Wiener estimate over the Wiener match spins
  const int M2 = grid_count(Mp, dw, st2), N2 = grid_count(Np, dw, st2);
  uint32_t* S2 = buf<uint32_t>(c, "p.S2", (size_t)K * M2 * N2);
  for (int ii = 0; ii < nW; ++ii) {
    const int s = o->matchSpinsWie[ii];
    {
      StageTimer t(c, 4);
      run_match(c, U1f, nullptr, Mp, Np, s, dw, d2, K, K, sigma, S2, nullptr, nullptr, nullptr, nullptr, "m2", st2,
                o->form, strip ? plan.s2[ii].groups : ColRange());
    }
    float* padP = buf<float>(c, "m2.pad", 1);  // the pilot search image run_match just built
    float* padN = buf<float>(c, "m2.padN", (size_t)pitch4(Mp + d2) * (Np + d2));
    launched(c, launch_make_pad(If, Mp, Np, d2, s, padN, pitch4(Mp + d2), c->st), "make_pad");
    WienerArgs A{};
    A.padP = padP;
    A.padN = padN;
    A.P = pitch4(Mp + d2);
    A.d2 = d2;
    A.S = S2;
    A.M = M2;
    A.N = N2;
    A.K = K;
    A.s = st2;
    double sg = sigma;
    fill_wiener_consts(A, dw, sigwie_in ? sigwie_in : &sg, sigwie_in ? 1 : 0, 0);
    int32_t* cnt2 = nullptr;
    if (strip) {
      const ColRange& gr = plan.s2[ii].groups;
      group_span(gr, M2, N2, A.g0, A.gn);
      cnt2 = buf<int32_t>(c, "p.cnt2", (size_t)M2 * N2);
      k_window_counts<<<(M2 * N2 + 255) / 256, 256, 0, c->st>>>(cnt2, M2, N2, pmod(gr.lo, N2),
                                                                 gr.all(N2) ? N2 : gr.len, K);
      launched(c, cudaGetLastError(), "window_counts");
    }
    run_wiener_agg(c, A, dw, d2, Us, Ws, strip ? plan.s2[ii].agg : ColRange(), cnt2);
    k_accum2<<<grid2(Mp, Np), 256, 0, c->st>>>(Us, Ws, Mp, Np, s, Ua, Wa, ii == 0);
    launched(c, cudaGetLastError(), "accum");
  }
  if (stale)
    for (int ii = nW; ii < nS; ++ii) {
      k_add_f<<<(unsigned)((px + 255) / 256), 256, 0, c->st>>>(Wstale + (size_t)(ii - nW) * px, Wa, px);
      launched(c, cudaGetLastError(), "add");
    }
  k_ratio<<<grid2(Mp, Np), 256, 0, c->st>>>(Ua, Wa, Mp, Np, nullptr, nullptr, dU, m, n);
  launched(c, cudaGetLastError(), "ratio");
}

}  // namespace

// =====================================================================================
extern "C" {

int gbm3d_version(void) { return 100; }

int gbm3d_ctx_create(int device, gbm3d_ctx** out) {
  if (!out) return GBM3D_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) return GBM3D_ERR_CUDA;
  if (device < 0 || device >= n) return GBM3D_ERR_ARG;
  gbm3d_ctx* c = new gbm3d_ctx();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->flag, sizeof(int)) != cudaSuccess) {
    delete c;
    return GBM3D_ERR_CUDA;
  }
  c->st = c->own;
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  *out = c;
  return GBM3D_OK;
}

void gbm3d_ctx_destroy(gbm3d_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->st);
  if (c->h2d) {
    cudaStreamSynchronize(c->h2d);
    cudaStreamSynchronize(c->d2h);
    cudaStreamDestroy(c->h2d);
    cudaStreamDestroy(c->d2h);
    for (int k = 0; k < 2; ++k)
      for (cudaEvent_t e : {c->in_ready[k], c->in_free[k], c->out_ready[k], c->out_free[k]})
        if (e) cudaEventDestroy(e);
  }
  if (c->sticky) cudaFree(c->sticky);
  if (c->tc_hist) cudaFree(c->tc_hist);
  for (cudaStream_t s : c->lane_st) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  for (cudaEvent_t e : c->lane_ev) cudaEventDestroy(e);
  for (auto& kv : c->bufs) cudaFree(kv.second.first);
  for (auto& e : c->evpool) cudaEventDestroy(e);
  for (auto& e : c->kpool) cudaEventDestroy(e);
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->flag) cudaFree(c->flag);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
}

int gbm3d_ctx_set_lanes(gbm3d_ctx* c, int lanes) {
  if (!c || lanes < 1 || lanes > 16) return GBM3D_ERR_ARG;
  c->lanes = lanes;
  return GBM3D_OK;
}

int gbm3d_ctx_set_stream(gbm3d_ctx* c, void* s) {
  if (!c) return GBM3D_ERR_ARG;
  c->st = s ? (cudaStream_t)s : c->own;
  return GBM3D_OK;
}

const char* gbm3d_last_error(const gbm3d_ctx* c) { return c ? c->err.c_str() : "null context"; }

int gbm3d_ctx_set_tc_wait(gbm3d_ctx* c, long long cycles) {
  if (!c) return GBM3D_ERR_ARG;
  c->tc_wait = cycles;
  return GBM3D_OK;
}

int gbm3d_ctx_tc_stats(gbm3d_ctx* c, int enable, int32_t* hist) {
  return guarded(c, [&] {
    if (!c->tc_hist) {
      ck(c, cudaMalloc(&c->tc_hist, 33 * sizeof(int)), "tc_hist");
      ck(c, cudaMemsetAsync(c->tc_hist, 0, 33 * sizeof(int), c->st), "memset");
    }
    if (hist) {
      ck(c, cudaMemcpyAsync(hist, c->tc_hist, 33 * sizeof(int), cudaMemcpyDeviceToHost, c->st), "D2H");
      ck(c, cudaMemsetAsync(c->tc_hist, 0, 33 * sizeof(int), c->st), "memset");
      ck(c, cudaStreamSynchronize(c->st), "synchronize");
    }
    c->tc_stats = enable != 0;
  });
}

int gbm3d_ctx_enable_timing(gbm3d_ctx* c, int on) {
  if (!c) return GBM3D_ERR_ARG;
  c->timing = on != 0;
  return GBM3D_OK;
}

int gbm3d_stage_times(const gbm3d_ctx* c, float* ms, int n) {
  if (!c || !ms || !c->timing) return 0;
  float acc[8] = {};
  for (const auto& r : c->records) {
    float t = 0.f;
    if (cudaEventSynchronize(c->evpool[r.second + 1]) != cudaSuccess ||
        cudaEventElapsedTime(&t, c->evpool[r.second], c->evpool[r.second + 1]) != cudaSuccess)
      return -1;
    acc[r.first] += t;
  }
  int k = 0;
  for (; k < n && k < 8; ++k) ms[k] = acc[k];
  return k;
}

int gbm3d_last_launch_count(const gbm3d_ctx* c) { return c ? c->launches : 0; }

int gbm3d_ctx_synchronize(gbm3d_ctx* c) {
  if (!c) return GBM3D_ERR_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess || cudaStreamSynchronize(c->st) != cudaSuccess) {
    c->err = "stream synchronisation failed";
    return GBM3D_ERR_CUDA;
  }
  if (c->async_pending) {  // gbm3d_denoise_async: its copies, then its status words
    c->async_pending = false;
    int flag = 0;
    if (cudaStreamSynchronize(c->h2d) != cudaSuccess || cudaStreamSynchronize(c->d2h) != cudaSuccess ||
        cudaMemcpy(&flag, c->sticky, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemset(c->sticky, 0, sizeof(int)) != cudaSuccess) {
      c->err = "stream synchronisation failed";
      return GBM3D_ERR_CUDA;
    }
    if (flag & 1) {
      c->err = "input image holds NaN or Inf (an asynchronous call since the last synchronisation)";
      return GBM3D_ERR_NONFINITE;
    }
    if (flag & 2) {
      c->err = "tensor-core matcher: a TMA copy or MMA did not complete within its wait limit";
      return GBM3D_ERR_CUDA;
    }
    if (flag & 4) {
      c->err = "matcher: a search-window TMA copy did not complete within its wait limit";
      return GBM3D_ERR_CUDA;
    }
  }
  return GBM3D_OK;
}

int gbm3d_kernel_time(const gbm3d_ctx* c, const char* name, float* total_ms) {
  if (!c || !name || !total_ms || !c->timing) return -1;
  float acc = 0.f;
  int n = 0;
  for (size_t i = 0; i < c->krec.size(); ++i) {
    if (c->krec[i] != name) continue;
    float t = 0.f;
    if (cudaEventSynchronize(c->kpool[i + 1]) != cudaSuccess ||
        cudaEventElapsedTime(&t, c->kpool[i], c->kpool[i + 1]) != cudaSuccess)
      return -1;
    acc += t;
    ++n;
  }
  *total_ms = acc;
  return n;
}

void gbm3d_default_opts(const char* profile, gbm3d_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  std::string p = profile ? profile : "default";
  o->numMax = 16;
  o->numMin = 16;
  o->levels = 3;
  o->cycleSpin = 2;
  o->tauMode = 1;
  o->blockSize = 16;
  o->blockSizeWie = 8;
  o->matchSize = 32;
  o->Wiener = 1;
  o->filtType = 0;
  o->staleWeights = 1;
  auto spins = [](int* dst, int& cnt, std::initializer_list<int> v) {
    cnt = 0;
    for (int s : v) dst[cnt++] = s;
  };
  if (p == "fast") {
    spins(o->matchSpins, o->nMatchSpins, {0, 4, 6});
    spins(o->matchSpinsWie, o->nMatchSpinsWie, {0});
  } else if (p == "superFast") {
    spins(o->matchSpins, o->nMatchSpins, {0, 4, 6});
    spins(o->matchSpinsWie, o->nMatchSpinsWie, {0});
    o->blockSize = 32;
    o->Wiener = 0;
  } else if (p == "accuracy") {
    spins(o->matchSpins, o->nMatchSpins, {0, 4, 6});
    spins(o->matchSpinsWie, o->nMatchSpinsWie, {0, 4, 6});
  } else {
    spins(o->matchSpins, o->nMatchSpins, {0, 4});
    spins(o->matchSpinsWie, o->nMatchSpinsWie, {0, 4});
  }
}

void gbm3d_get_tau(int levels, int mode, double* tau) {
  if (tau && levels > 0) tau_table(levels, mode, tau);
}

void gbm3d_bior_filters(gbm3d_filters* f) {
  if (f) bior(f);
}

// Psi / Psi2 (Ly x Lx x Lz x 8, column-major; band order LLL, HLL, LHL, LLH,
// HHL, HLH, LHH, HHH over (y, x, z), getWaveFilters3Dbior.m:39-58) back to
// separable 1D factors.  Known banks (bior1.5 x Haar, 3D Haar) are recognised
// to 1e-5 and returned exactly; any other separable bank is split at its
// largest |LLL| entry (a, a, c): lo = LLL(:,a,c)/LLL(a,a,c), vlo = LLL(a,a,:),
// hi = HLL(:,a,c)/vlo(c), vhi = LLH(a,a,:), and must rebuild Psi to 1e-4.
static void bank_of(const gbm3d_filters& f, int which, std::vector<double>& B) {
  const int L = f.len_xy, Lz = f.len_z;
  const double* xy[2] = {which ? f.s_lo_xy : f.a_lo_xy, which ? f.s_hi_xy : f.a_hi_xy};
  const double* z[2] = {which ? f.s_lo_z : f.a_lo_z, which ? f.s_hi_z : f.a_hi_z};
  static const int ord[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  B.assign((size_t)L * L * Lz * 8, 0.0);
  for (int b = 0; b < 8; ++b)
    for (int zz = 0; zz < Lz; ++zz)
      for (int x = 0; x < L; ++x)
        for (int y = 0; y < L; ++y)
          B[y + (size_t)L * (x + (size_t)L * (zz + (size_t)Lz * b))] = xy[ord[b][0]][y] * xy[ord[b][1]][x] * z[ord[b][2]][zz];
}

static double bank_err(const gbm3d_filters& f, const float* Psi, const float* Psi2) {
  std::vector<double> B;
  double e = 0.0;
  for (int w = 0; w < 2; ++w) {
    bank_of(f, w, B);
    const float* P = w ? Psi2 : Psi;
    for (size_t i = 0; i < B.size(); ++i) e = std::max(e, std::fabs(B[i] - (double)P[i]));
  }
  return e;
}

int gbm3d_filters_from_bank(const float* Psi, const float* Psi2, int L, int Lz, gbm3d_filters* out) {
  if (!Psi || !Psi2 || !out || L < 1 || L > 16 || Lz < 1 || Lz > 16) return GBM3D_ERR_ARG;
  gbm3d_filters f;
  bior(&f);
  if (f.len_xy == L && f.len_z == Lz && bank_err(f, Psi, Psi2) <= 1e-5) { *out = f; return GBM3D_OK; }
  haar3d(&f);
  if (f.len_xy == L && f.len_z == Lz && bank_err(f, Psi, Psi2) <= 1e-5) { *out = f; return GBM3D_OK; }
  std::memset(&f, 0, sizeof(f));
  f.len_xy = L;
  f.len_z = Lz;
  const size_t band = (size_t)L * L * Lz;
  for (int w = 0; w < 2; ++w) {
    const float* P = w ? Psi2 : Psi;
    int a = 0, c = 0;
    double best = -1.0;
    for (int zz = 0; zz < Lz; ++zz)
      for (int x = 0; x < L; ++x)
        for (int y = 0; y < L; ++y) {
          const double v = std::fabs((double)P[y + (size_t)L * (x + (size_t)L * zz)]);
          if (v > best) { best = v; a = y; c = zz; }
        }
    auto at = [&](int b, int y, int x, int zz) { return (double)P[y + (size_t)L * (x + (size_t)L * zz) + band * b]; };
    const double piv = at(0, a, a, c);
    if (piv == 0.0) return GBM3D_ERR_ARG;
    double* lo = w ? f.s_lo_xy : f.a_lo_xy;
    double* hi = w ? f.s_hi_xy : f.a_hi_xy;
    double* vlo = w ? f.s_lo_z : f.a_lo_z;
    double* vhi = w ? f.s_hi_z : f.a_hi_z;
    for (int zz = 0; zz < Lz; ++zz) {
      vlo[zz] = at(0, a, a, zz);
      vhi[zz] = at(3, a, a, zz);
    }
    if (vlo[c] == 0.0) return GBM3D_ERR_ARG;
    for (int y = 0; y < L; ++y) {
      lo[y] = at(0, y, a, c) / piv;
      hi[y] = at(1, y, a, c) / vlo[c];
    }
  }
  if (bank_err(f, Psi, Psi2) > 1e-4) return GBM3D_ERR_ARG;  // not separable
  *out = f;
  return GBM3D_OK;
}

int gbm3d_matchBlocksCPU(gbm3d_ctx* c, const double* I, int m, int n, double sigma, const gbm3d_opts* o,
                         uint32_t* S, int32_t* S_count, float* Volume) {
  return guarded(c, [&] {
    check_opts(c, o);
    const int d = o->blockSize, d2 = o->matchSize, K = o->numMax;
    check_match(c, d, d2, K);
    if (!I || !S) argfail(c, "I and S are required");
    if (m < d2 || n < d2 || m < d || n < d) argfail(c, "image smaller than matchSize");
    const int s = stride1(o);
    const int M = grid_count(m, d, s), N = grid_count(n, d, s);
    const size_t px = (size_t)m * n;
    const size_t vn = s == d ? px * K : (size_t)M * d * N * d * K;
    double* dI = buf<double>(c, "io.I", px);
    ck(c, cudaMemcpyAsync(dI, I, px * sizeof(double), cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
    float* If = buf<float>(c, "io.If", px);
    k_prep<<<grid2(m, n), 256, 0, c->st>>>(dI, m, n, If, m, n, c->flag);
    launched(c, cudaGetLastError(), "prep");
    uint32_t* dS = buf<uint32_t>(c, "io.S", (size_t)K * M * N);
    int32_t* dc = buf<int32_t>(c, "io.cnt", (size_t)M * N);
    float* dV = nullptr;
    if (Volume) {
      dV = buf<float>(c, "io.V", vn);
      ck(c, cudaMemsetAsync(dV, 0, vn * sizeof(float), c->st), "memset");
    }
    run_match(c, If, nullptr, m, n, 0, d, d2, K, o->numMin, sigma, dS, dc, dV, nullptr, nullptr, "m1", s, o->form);
    ck(c, cudaMemcpyAsync(S, dS, (size_t)K * M * N * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    if (S_count) ck(c, cudaMemcpyAsync(S_count, dc, (size_t)M * N * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    if (Volume) ck(c, cudaMemcpyAsync(Volume, dV, vn * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    int flag = 0;
    ck(c, cudaMemcpyAsync(&flag, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
    report_flag(c, flag);
  });
}

int gbm3d_matchBlocksGPU(gbm3d_ctx* c, const double* I, int m, int n, double sigma, const gbm3d_opts* o,
                         uint32_t* S, int32_t* S_count) {
  return guarded(c, [&] {
    check_opts(c, o);
    const int d = o->blockSize, K = o->numMax;
    if (!global_match_supported(d, K))
      argfail(c, "unsupported blockSize for the global matcher", GBM3D_ERR_UNSUPPORTED);
    if (!I || !S) argfail(c, "I and S are required");
    if (m < d || n < d || m < 16 || n < 16) argfail(c, "image too small for the global matcher");
    if ((sigma > 30.0 / 255.0) && (m % 8 || n % 8))
      argfail(c, "the sym4 prefilter needs image sides divisible by 8");
    const int M = m / d, N = n / d;
    const size_t px = (size_t)m * n;
    double* dI = buf<double>(c, "io.I", px);
    ck(c, cudaMemcpyAsync(dI, I, px * sizeof(double), cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
    float* If = buf<float>(c, "io.If", px);
    k_prep<<<grid2(m, n), 256, 0, c->st>>>(dI, m, n, If, m, n, c->flag);
    launched(c, cudaGetLastError(), "prep");
    if (sigma > 30.0 / 255.0) {  // matchBlocksGPU.m:34
      float* work = buf<float>(c, "gm.work", px * 8);
      ck(c, launch_sym4_prefilter(If, m, n, (float)(2 * sigma), work, c->st), "sym4 prefilter");
    }
    uint32_t* dS = buf<uint32_t>(c, "io.S", (size_t)K * M * N);
    int32_t* dc = buf<int32_t>(c, "io.cnt", (size_t)M * N);
    GlobalMatchArgs A{};
    A.I = If;
    A.m = m;
    A.n = n;
    A.M = M;
    A.N = N;
    A.K = K;
    A.numMin = o->numMin;
    A.tol = (float)(0.005 * sigma * sigma * d * d);
    A.tol_branch = o->numMin != K;
    A.S = dS;
    A.cnt = dc;
    launched(c, launch_match_global(d, A, c->st), "match_global");
    ck(c, cudaMemcpyAsync(S, dS, (size_t)K * M * N * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    if (S_count) ck(c, cudaMemcpyAsync(S_count, dc, (size_t)M * N * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    int flag = 0;
    ck(c, cudaMemcpyAsync(&flag, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
    report_flag(c, flag);
  });
}

int gbm3d_denoiseAndAggregateGPU(gbm3d_ctx* c, const float* Volume, const uint32_t* S, const int32_t* S_count,
                                 int M, int N, const double* tau, const gbm3d_filters* f, const gbm3d_opts* o,
                                 double* U, double* W) {
  return guarded(c, [&] {
    check_opts(c, o);
    if (!Volume || !S || !tau || !U || !W) argfail(c, "missing argument");
    const int d = o->blockSize, d2 = o->matchSize, K = o->numMax;
    if (M < 1 || N < 1) argfail(c, "empty match set");
    gbm3d_filters fb;
    if (f) fb = *f; else bior(&fb);
    const WaveletBank bk = make_bank(c, &fb);
    const int s = stride1(o);
    const int m = M * d, n = N * d;  // tile-space volume
    const size_t px = (size_t)m * n, po = (size_t)((M - 1) * s + d) * ((N - 1) * s + d);
    check_match_set(c, S, S_count, (size_t)M * N, K, d2);
    float* dV = buf<float>(c, "io.V", px * K);
    uint32_t* dS = buf<uint32_t>(c, "io.S", (size_t)K * M * N);
    int32_t* dc = nullptr;
    ck(c, cudaMemcpyAsync(dV, Volume, px * K * 4, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemcpyAsync(dS, S, (size_t)K * M * N * 4, cudaMemcpyHostToDevice, c->st), "H2D");
    if (S_count) {
      dc = buf<int32_t>(c, "io.cnt", (size_t)M * N);
      ck(c, cudaMemcpyAsync(dc, S_count, (size_t)M * N * 4, cudaMemcpyHostToDevice, c->st), "H2D");
    }
    float* dU = buf<float>(c, "io.U", po);
    float* dW = buf<float>(c, "io.W", po);
    run_ht(c, dV, dS, dc, M, N, d, d2, K, o->levels, o->cycleSpin, tau, bk, dU, dW, o->filtType, s);
    to_host_double(c, dU, po, U);
    ck(c, cudaStreamSynchronize(c->st), "sync");
    to_host_double(c, dW, po, W);
    ck(c, cudaStreamSynchronize(c->st), "sync");
  });
}

int gbm3d_matchBlocksWie(gbm3d_ctx* c, const double* I, const double* In, int m, int n, double sigma,
                         const gbm3d_opts* o, uint32_t* S, float* V1, float* V2) {
  return guarded(c, [&] {
    check_opts(c, o);
    const int d = o->blockSizeWie, d2 = o->matchSize, K = o->numMax;
    check_match(c, d, d2, K);
    if (!I || !In || !S) argfail(c, "missing argument");
    if (m < d2 || n < d2 || m < d || n < d) argfail(c, "image smaller than matchSize");
    const int s = stride2(o);
    const int M = grid_count(m, d, s), N = grid_count(n, d, s);
    const size_t px = (size_t)m * n, gs = (size_t)d * d * K * M * N;
    double* dI = buf<double>(c, "io.I", px);
    double* dIn = buf<double>(c, "io.In", px);
    ck(c, cudaMemcpyAsync(dI, I, px * 8, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemcpyAsync(dIn, In, px * 8, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
    float* If = buf<float>(c, "io.If", px);
    float* Inf = buf<float>(c, "io.Inf", px);
    k_prep<<<grid2(m, n), 256, 0, c->st>>>(dI, m, n, If, m, n, c->flag);
    launched(c, cudaGetLastError(), "prep");
    k_prep<<<grid2(m, n), 256, 0, c->st>>>(dIn, m, n, Inf, m, n, c->flag);
    launched(c, cudaGetLastError(), "prep");
    uint32_t* dS = buf<uint32_t>(c, "io.S", (size_t)K * M * N);
    float* d1 = V1 ? buf<float>(c, "io.V1", gs) : nullptr;
    float* d2p = V2 ? buf<float>(c, "io.V2", gs) : nullptr;
    run_match(c, If, V2 ? Inf : nullptr, m, n, 0, d, d2, K, K, sigma, dS, nullptr, nullptr, d1, d2p, "m2", s, o->form);
    ck(c, cudaMemcpyAsync(S, dS, (size_t)K * M * N * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    if (V1) ck(c, cudaMemcpyAsync(V1, d1, gs * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    if (V2) ck(c, cudaMemcpyAsync(V2, d2p, gs * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    int flag = 0;
    ck(c, cudaMemcpyAsync(&flag, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
    report_flag(c, flag);
  });
}

static int wiener_entry(gbm3d_ctx* c, const float* V1, const float* V2, const uint32_t* S, int M, int N,
                        const double* sigma, int is_matrix, const gbm3d_opts* o, double* U, double* W,
                        int variant) {
  return guarded(c, [&] {
    check_opts(c, o);
    if (!V1 || !V2 || !S || !sigma || !U || !W) argfail(c, "missing argument");
    const int d = o->blockSizeWie, d2 = o->matchSize, K = o->numMax;
    if (M < 1 || N < 1) argfail(c, "empty match set");
    if (d * d > 256) argfail(c, "blockSizeWie too large", GBM3D_ERR_UNSUPPORTED);
    const int s = stride2(o);
    const size_t gs = (size_t)d * d * K * M * N, px = (size_t)((M - 1) * s + d) * ((N - 1) * s + d);
    check_match_set(c, S, nullptr, (size_t)M * N, K, d2);
    float* d1 = buf<float>(c, "io.V1", gs);
    float* d2p = buf<float>(c, "io.V2", gs);
    uint32_t* dS = buf<uint32_t>(c, "io.S", (size_t)K * M * N);
    ck(c, cudaMemcpyAsync(d1, V1, gs * 4, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemcpyAsync(d2p, V2, gs * 4, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemcpyAsync(dS, S, (size_t)K * M * N * 4, cudaMemcpyHostToDevice, c->st), "H2D");
    WienerArgs A{};
    A.V1 = d1;
    A.V2 = d2p;
    A.S = dS;
    A.M = M;
    A.N = N;
    A.K = K;
    A.s = s;
    A.d2 = d2;
    fill_wiener_consts(A, d, sigma, is_matrix, variant);
    float* dU = buf<float>(c, "io.U", px);
    float* dW = buf<float>(c, "io.W", px);
    run_wiener_agg(c, A, d, d2, dU, dW);
    to_host_double(c, dU, px, U);
    ck(c, cudaStreamSynchronize(c->st), "sync");
    to_host_double(c, dW, px, W);
    ck(c, cudaStreamSynchronize(c->st), "sync");
  });
}

int gbm3d_denoiseAndAggregateWieFast(gbm3d_ctx* c, const float* V1, const float* V2, const uint32_t* S, int M,
                                     int N, const double* sigma, int is_matrix, const gbm3d_opts* o, double* U,
                                     double* W) {
  return wiener_entry(c, V1, V2, S, M, N, sigma, is_matrix, o, U, W, 0);
}

int gbm3d_denoiseAndAggregateWie(gbm3d_ctx* c, const float* V1, const float* V2, const uint32_t* S, int M, int N,
                                 double sigma, const gbm3d_opts* o, double* U, double* W) {
  return wiener_entry(c, V1, V2, S, M, N, &sigma, 0, o, U, W, 1);
}

int gbm3d_tc_selfcheck(gbm3d_ctx* c, const uint16_t* A, const uint16_t* B, float* C) {
  return gbm3d_tc_selfcheck_layout(c, 0, A, B, C);
}

int gbm3d_tc_selfcheck_layout(gbm3d_ctx* c, int mn_major, const uint16_t* A, const uint16_t* B, float* C) {
  return guarded(c, [&] {
    if (!A || !B || !C) argfail(c, "missing argument");
    uint16_t* dA = buf<uint16_t>(c, "tc.A", 128 * 64);
    uint16_t* dB = buf<uint16_t>(c, "tc.B", 256 * 64);
    float* dC = buf<float>(c, "tc.C", 128 * 256);
    ck(c, cudaMemcpyAsync(dA, A, 128 * 64 * 2, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemcpyAsync(dB, B, 256 * 64 * 2, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
    if (mn_major)
      launched(c, launch_tc_gemm_check_mn(dA, dB, dC, c->flag, mn_major == 2, c->st), "tc_gemm_check");
    else
      launched(c, launch_tc_gemm_check(dA, dB, dC, c->flag, c->st), "tc_gemm_check");
    ck(c, cudaMemcpyAsync(C, dC, 128 * 256 * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    int flag = 0;
    ck(c, cudaMemcpyAsync(&flag, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
    if (flag) argfail(c, "tensor-core matcher: a TMA copy or MMA did not complete within its wait limit", GBM3D_ERR_CUDA);
  });
}

}  // extern "C"

namespace {

// Colour GBM3D in the opponent space: block matching on the luma channel
// only, and every channel filtered (hard threshold, then Wiener) and
// aggregated with luma's match sets, each with its own noise level
// sigma_c = sigma |row c of A|.  dI / dU: three device planes (R, G, B),
// float64 column-major m x n.
void pipeline_rgb(gbm3d_ctx* c, const double* const* dI, int m, int n, double sigma, const gbm3d_opts* o,
                  double* const* dU) {
  check_opts(c, o);
  if (o->form == 2) argfail(c, "the learned pilot is trained on grey images", GBM3D_ERR_UNSUPPORTED);
  if (!o->Wiener) argfail(c, "the colour form runs both steps", GBM3D_ERR_UNSUPPORTED);
  int d, dw, d2, K;
  opts_dims(o, d, dw, d2, K);
  check_match(c, d, d2, K);
  check_match(c, dw, d2, K);
  if (m < 1 || n < 1 || m > 32000 || n > 32000) argfail(c, "image size out of range");
  const int st1 = stride1(o), st2 = stride2(o);
  if ((d - dw) % std::gcd(st1, st2) != 0)
    argfail(c, "no padded size lets both reference grids end at the border", GBM3D_ERR_UNSUPPORTED);
  auto padded = [&](int L) {
    if (st1 == d && st2 == dw && d % dw == 0) return (L + d - 1) / d * d;
    int p = std::max(L, std::max(d, dw));
    while ((p - d) % st1 != 0 || (p - dw) % st2 != 0) ++p;
    return p;
  };
  const int Mp = padded(m), Np = padded(n);
  if (Mp - m > m || Np - n > n) argfail(c, "image smaller than the padding it needs");
  if (Mp < d2 || Np < d2) argfail(c, "image smaller than matchSize");
  const int nS = o->nMatchSpins, nW = o->nMatchSpinsWie;
  if (nS < 1 || nS > 8 || nW < 1 || nW > 8) argfail(c, "match spin count out of range");
  const size_t px = (size_t)Mp * Np, pm = (size_t)m * n;
  const double csig[3] = {sigma * std::sqrt(1.0 / 3.0), sigma * std::sqrt(0.5), sigma * std::sqrt(0.375)};
  gbm3d_filters f;
  bank_of_opts(o, &f);
  const WaveletBank bk = make_bank(c, &f);
  std::vector<double> tau1(o->levels * 7);
  tau_table(o->levels, o->tauMode, tau1.data());
  const int P = pitch4(Mp + d2);

  // opponent planes, mirror padded to single
  double* opp[3];
  float* If[3];
  for (int ch = 0; ch < 3; ++ch) {
    opp[ch] = buf<double>(c, ("rgb.opp" + std::to_string(ch)).c_str(), pm);
    If[ch] = buf<float>(c, ("rgb.If" + std::to_string(ch)).c_str(), px);
  }
  ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
  k_opp<<<592, 256, 0, c->st>>>(dI[0], dI[1], dI[2], pm, opp[0], opp[1], opp[2], 0);
  launched(c, cudaGetLastError(), "opp");
  for (int ch = 0; ch < 3; ++ch) {
    k_prep<<<grid2(Mp, Np), 256, 0, c->st>>>(opp[ch], m, n, If[ch], Mp, Np, c->flag);
    launched(c, cudaGetLastError(), "prep");
  }
  float* Us = buf<float>(c, "p.Us", px);
  float* Ws = buf<float>(c, "p.Ws", px);
  double *Ua[3], *Wa[3];
  float* U1f[3];
  for (int ch = 0; ch < 3; ++ch) {
    Ua[ch] = buf<double>(c, ("rgb.Ua" + std::to_string(ch)).c_str(), px);
    Wa[ch] = buf<double>(c, ("rgb.Wa" + std::to_string(ch)).c_str(), px);
    U1f[ch] = buf<float>(c, ("rgb.U1f" + std::to_string(ch)).c_str(), px);
  }
  float* pad = buf<float>(c, "rgb.pad", (size_t)P * (Np + d2));
  float* pad2 = buf<float>(c, "rgb.pad2", (size_t)P * (Np + d2));

  // step 1: luma matching, per-channel 3D hard thresholding
  const int M1 = grid_count(Mp, d, st1), N1 = grid_count(Np, d, st1);
  uint32_t* S1 = buf<uint32_t>(c, "p.S1", (size_t)K * M1 * N1);
  int32_t* cnt1 = buf<int32_t>(c, "p.cnt1", (size_t)M1 * N1);
  float* vol = buf<float>(c, "p.vol", (size_t)M1 * d * N1 * d * K);
  for (int ii = 0; ii < nS; ++ii) {
    const int s = o->matchSpins[ii];
    for (int ch = 0; ch < 3; ++ch) {
      if (ch == 0) {
        StageTimer t(c, 1);
        run_match(c, If[0], nullptr, Mp, Np, s, d, d2, K, o->numMin, csig[0], S1, cnt1, vol, nullptr, nullptr, "m1",
                  st1, o->form);
      } else {
        launched(c, launch_make_pad(If[ch], Mp, Np, d2, s, pad, P, c->st), "make_pad");
        launched(c, launch_gather_volume(pad, P, M1, N1, st1, d, d2, K, S1, cnt1, vol, c->st), "gather");
      }
      std::vector<double> tau(tau1);
      for (auto& t : tau) t *= csig[ch];
      run_ht(c, vol, S1, cnt1, M1, N1, d, d2, K, o->levels, o->cycleSpin, tau.data(), bk, Us, Ws, o->filtType, st1);
      k_accum<<<grid2(Mp, Np), 256, 0, c->st>>>(Us, Mp, Np, s, Ua[ch], ii == 0);
      launched(c, cudaGetLastError(), "accum");
      k_accum<<<grid2(Mp, Np), 256, 0, c->st>>>(Ws, Mp, Np, s, Wa[ch], ii == 0);
      launched(c, cudaGetLastError(), "accum");
    }
  }
  for (int ch = 0; ch < 3; ++ch) {
    k_ratio<<<grid2(Mp, Np), 256, 0, c->st>>>(Ua[ch], Wa[ch], Mp, Np, nullptr, U1f[ch], nullptr, m, n);
    launched(c, cudaGetLastError(), "ratio");
  }

  // step 2: matching on the luma pilot, per-channel Wiener filtering
  const int M2 = grid_count(Mp, dw, st2), N2 = grid_count(Np, dw, st2);
  uint32_t* S2 = buf<uint32_t>(c, "p.S2", (size_t)K * M2 * N2);
  for (int ii = 0; ii < nW; ++ii) {
    const int s = o->matchSpinsWie[ii];
    {
      StageTimer t(c, 4);
      run_match(c, U1f[0], nullptr, Mp, Np, s, dw, d2, K, K, csig[0], S2, nullptr, nullptr, nullptr, nullptr, "m2",
                st2, o->form);
    }
    for (int ch = 0; ch < 3; ++ch) {
      launched(c, launch_make_pad(U1f[ch], Mp, Np, d2, s, pad, P, c->st), "make_pad");
      launched(c, launch_make_pad(If[ch], Mp, Np, d2, s, pad2, P, c->st), "make_pad");
      WienerArgs A{};
      A.padP = pad;
      A.padN = pad2;
      A.P = P;
      A.d2 = d2;
      A.S = S2;
      A.M = M2;
      A.N = N2;
      A.K = K;
      A.s = st2;
      fill_wiener_consts(A, dw, &csig[ch], 0, 0);
      run_wiener_agg(c, A, dw, d2, Us, Ws);
      k_accum<<<grid2(Mp, Np), 256, 0, c->st>>>(Us, Mp, Np, s, Ua[ch], ii == 0);
      launched(c, cudaGetLastError(), "accum");
      k_accum<<<grid2(Mp, Np), 256, 0, c->st>>>(Ws, Mp, Np, s, Wa[ch], ii == 0);
      launched(c, cudaGetLastError(), "accum");
    }
  }
  for (int ch = 0; ch < 3; ++ch) {
    k_ratio<<<grid2(Mp, Np), 256, 0, c->st>>>(Ua[ch], Wa[ch], Mp, Np, nullptr, nullptr, opp[ch], m, n);
    launched(c, cudaGetLastError(), "ratio");
  }
  k_opp<<<592, 256, 0, c->st>>>(opp[0], opp[1], opp[2], pm, dU[0], dU[1], dU[2], 1);
  launched(c, cudaGetLastError(), "opp");
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// ---- video (VBM3D.m, matchBlocksV.m, denoiseAndAggregateV.m) -----------------------

int video_frames(const gbm3d_opts* o) { return o->videoFrames > 0 ? o->videoFrames : 11; }

void check_video(gbm3d_ctx* c, const gbm3d_opts* o, int d, int F, int K) {
  if (o->numMin != o->numMax) argfail(c, "video matching: the tolerance branch is not supported", GBM3D_ERR_UNSUPPORTED);
  if (!video_match_supported(d, F, K))
    argfail(c, "video matching supports blockSize 8/16/32, an odd window of frames and numMax <= 32",
            GBM3D_ERR_UNSUPPORTED);
}

// matchBlocksV + denoiseAndAggregateV on one window whose F search images are
// built (pads); U, W: m x n x F double (device).
void video_window(gbm3d_ctx* c, float* const* pads, int P, int m, int n, int F, int d, int K, int levels,
                  int cycleSpin, const double* tau, const WaveletBank& bk, uint32_t* S, float* vol, double* U,
                  double* W) {
  const int M = m / d, N = n / d;
  VideoMatchArgs A{};
  for (int f = 0; f < F; ++f) A.pads[f] = pads[f];
  A.P = P;
  A.M = M;
  A.N = N;
  A.F = F;
  A.K = K;
  A.m = m;
  A.n = n;
  A.S = S;
  A.volume = vol;
  {
    StageTimer t(c, 1);
    launched(c, launch_match_video(d, A, c->st), "match_video");
  }
  float* vsum;
  {
    StageTimer t(c, 2);
    vsum = run_wavelet_ht(c, vol, m, n, K, levels, cycleSpin, tau, bk, 0);
    launched(c, launch_clamp01(vsum, (size_t)m * n * K, c->st), "clamp");  // Vavg = min(max(.,0),1)
  }
  StageTimer t(c, 3);
  float* wgt = buf<float>(c, "v.wgt", (size_t)M * N);
  launched(c, launch_ht_weights(vsum, m, n, M, N, d, K, nullptr, wgt, c->st), "ht_weights");
  VideoAggArgs G{};
  G.S = S;
  G.wgt = wgt;
  G.vsum = vsum;
  G.M = M;
  G.N = N;
  G.d = d;
  G.K = K;
  G.F = F;
  G.m = m;
  G.n = n;
  G.U = U;
  G.W = W;
  launched(c, launch_aggregate_video(G, c->st), "aggregate_video");
}

__global__ void k_video_accum(const double* __restrict__ U, const double* __restrict__ W, size_t n,
                              float* __restrict__ Y, float* __restrict__ nn) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    Y[i] = (float)((double)Y[i] + U[i]);  // the reference's Y and nn are single arrays
    nn[i] = (float)((double)nn[i] + W[i]);
  }
}

// out frame (k - hw) += (Y ./ nn)(r + s, c + s) of frame k (the shift back), cropped to m0 x n0
__global__ void k_video_out(const float* __restrict__ Y, const float* __restrict__ nn, int Mp, int Np, int m0,
                            int n0, int hw, int nOut, int s, double* __restrict__ acc, int first) {
  const size_t total = (size_t)m0 * n0 * nOut;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(p % m0), c = (int)((p / m0) % n0), k = (int)(p / ((size_t)m0 * n0)) + hw;
    const size_t o = (size_t)Mp * Np * k + pmod(r + s, Mp) + (size_t)Mp * pmod(c + s, Np);
    const double v = (double)(Y[o] / nn[o]);
    acc[p] = first ? v : acc[p] + v;
  }
}

__global__ void k_video_final(const double* __restrict__ acc, size_t n, double nS, double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)(float)(acc[i] / nS);
}

// VBM3D.m:20-63 on device frames I (m0 x n0 x Kf, float64 column-major, the
// reference's [0,1] scale): out (m0 x n0 x (Kf - nF + 1)).
void pipeline_video(gbm3d_ctx* c, const double* I, int m0, int n0, int Kf, double sigma, const gbm3d_opts* o,
                    double* out) {
  check_opts(c, o);
  const int d = o->blockSize, K = o->numMax, F = video_frames(o), hw = (F - 1) / 2;
  check_video(c, o, d, F, K);
  if (Kf < F) argfail(c, "fewer frames than the temporal window");
  if (m0 < 1 || n0 < 1 || m0 > 32000 || n0 > 32000) argfail(c, "frame size out of range");
  const int Mp = (m0 + d - 1) / d * d, Np = (n0 + d - 1) / d * d;
  if (Mp - m0 > m0 || Np - n0 > n0) argfail(c, "frame smaller than the padding it needs");
  const int nS = o->nMatchSpins;
  if (nS < 1 || nS > 8) argfail(c, "match spin count out of range");
  gbm3d_filters f;
  bank_of_opts(o, &f);
  const WaveletBank bk = make_bank(c, &f);
  std::vector<double> tau(o->levels * 7);
  tau_table(o->levels, o->tauMode, tau.data());
  for (auto& t : tau) t *= sigma;
  const size_t px = (size_t)Mp * Np, px0 = (size_t)m0 * n0;
  const int P = pitch4(Mp + d), nOut = Kf - F + 1;
  StageTimer tall(c, 7);
  float* fr = buf<float>(c, "v.frames", px * Kf);
  ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
  for (int k = 0; k < Kf; ++k) {
    k_prep<<<grid2(Mp, Np), 256, 0, c->st>>>(I + px0 * k, m0, n0, fr + px * k, Mp, Np, c->flag);
    launched(c, cudaGetLastError(), "prep");
  }
  float* Y = buf<float>(c, "v.Y", px * Kf);
  float* nn = buf<float>(c, "v.nn", px * Kf);
  double* U = buf<double>(c, "v.U", px * F);
  double* W = buf<double>(c, "v.W", px * F);
  double* acc = buf<double>(c, "v.acc", px0 * nOut);
  uint32_t* S = buf<uint32_t>(c, "v.S", (size_t)K * (Mp / d) * (Np / d));
  float* vol = buf<float>(c, "v.vol", px * K);
  std::vector<float*> pads(F);
  for (int q = 0; q < F; ++q) pads[q] = buf<float>(c, ("v.pad" + std::to_string(q)).c_str(), (size_t)P * (Np + d));
  for (int ii = 0; ii < nS; ++ii) {
    const int s = o->matchSpins[ii];
    ck(c, cudaMemsetAsync(Y, 0, px * Kf * sizeof(float), c->st), "memset");
    ck(c, cudaMemsetAsync(nn, 0, px * Kf * sizeof(float), c->st), "memset");
    for (int jj = hw; jj < Kf - hw; ++jj) {
      for (int q = 0; q < F; ++q)  // circshift(I3, [s, s, 0]) and matchBlocksV's search images
        launched(c, launch_make_pad(fr + px * (jj - hw + q), Mp, Np, d, s, pads[q], P, c->st), "make_pad");
      video_window(c, pads.data(), P, Mp, Np, F, d, K, o->levels, o->cycleSpin, tau.data(), bk, S, vol, U, W);
      k_video_accum<<<1184, 256, 0, c->st>>>(U, W, px * F, Y + px * (jj - hw), nn + px * (jj - hw));
      launched(c, cudaGetLastError(), "video_accum");
    }
    k_video_out<<<1184, 256, 0, c->st>>>(Y, nn, Mp, Np, m0, n0, hw, nOut, s, acc, ii == 0);
    launched(c, cudaGetLastError(), "video_out");
  }
  k_video_final<<<1184, 256, 0, c->st>>>(acc, px0 * nOut, (double)nS, out);
  launched(c, cudaGetLastError(), "video_out");
}

}  // namespace

extern "C" {

int gbm3d_vbm3d_device(gbm3d_ctx* c, const double* I, int m, int n, int frames, double sigma, const gbm3d_opts* o,
                       double* out) {
  return guarded(c, [&] {
    if (!I || !out) argfail(c, "missing argument");
    pipeline_video(c, I, m, n, frames, sigma, o, out);
  });
}

int gbm3d_matchBlocksV(gbm3d_ctx* c, const double* I, int m, int n, int frames, const gbm3d_opts* o, uint32_t* S,
                       float* Volume) {
  return guarded(c, [&] {
    check_opts(c, o);
    const int d = o->blockSize, K = o->numMax;
    check_video(c, o, d, frames, K);
    if (!I || !S) argfail(c, "I and S are required");
    if (m < 2 * d || n < 2 * d) argfail(c, "frames smaller than two blocks");
    const int M = m / d, N = n / d, P = pitch4(m + d);
    const size_t px = (size_t)m * n;
    double* dI = buf<double>(c, "io.I", px * frames);
    ck(c, cudaMemcpyAsync(dI, I, px * frames * 8, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
    float* fr = buf<float>(c, "io.If", px * frames);
    std::vector<float*> pads(frames);
    VideoMatchArgs A{};
    for (int q = 0; q < frames; ++q) {
      k_prep<<<grid2(m, n), 256, 0, c->st>>>(dI + px * q, m, n, fr + px * q, m, n, c->flag);
      launched(c, cudaGetLastError(), "prep");
      pads[q] = buf<float>(c, ("v.pad" + std::to_string(q)).c_str(), (size_t)P * (n + d));
      launched(c, launch_make_pad(fr + px * q, m, n, d, 0, pads[q], P, c->st), "make_pad");
      A.pads[q] = pads[q];
    }
    uint32_t* dS = buf<uint32_t>(c, "io.S", (size_t)K * M * N);
    float* dV = buf<float>(c, "io.V", px * K);
    ck(c, cudaMemsetAsync(dV, 0, px * K * 4, c->st), "memset");
    A.P = P;
    A.M = M;
    A.N = N;
    A.F = frames;
    A.K = K;
    A.m = m;
    A.n = n;
    A.S = dS;
    A.volume = dV;
    launched(c, launch_match_video(d, A, c->st), "match_video");
    ck(c, cudaMemcpyAsync(S, dS, (size_t)K * M * N * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    if (Volume) ck(c, cudaMemcpyAsync(Volume, dV, px * K * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    int flag = 0;
    ck(c, cudaMemcpyAsync(&flag, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
    report_flag(c, flag);
  });
}

int gbm3d_denoiseAndAggregateV(gbm3d_ctx* c, const float* Volume, const uint32_t* S, int M, int N, int frames,
                               const double* tau, const gbm3d_filters* filters, const gbm3d_opts* o, double* U,
                               double* W) {
  return guarded(c, [&] {
    check_opts(c, o);
    const int d = o->blockSize, K = o->numMax;
    check_video(c, o, d, frames, K);
    if (!Volume || !S || !tau || !U || !W) argfail(c, "missing argument");
    const int m = M * d, n = N * d;
    const size_t px = (size_t)m * n;
    for (size_t g = 0; g < (size_t)M * N * K; ++g)
      if (S[g] < 1 || S[g] > (uint32_t)(d * d * frames)) argfail(c, "S holds an index outside the d x d x frames window");
    gbm3d_filters fb;
    if (filters) fb = *filters;
    else sym4haar(&fb);
    const WaveletBank bk = make_bank(c, &fb);
    float* dV = buf<float>(c, "io.V", px * K);
    uint32_t* dS = buf<uint32_t>(c, "io.S", (size_t)K * M * N);
    ck(c, cudaMemcpyAsync(dV, Volume, px * K * 4, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemcpyAsync(dS, S, (size_t)K * M * N * 4, cudaMemcpyHostToDevice, c->st), "H2D");
    float* vsum = run_wavelet_ht(c, dV, m, n, K, o->levels, o->cycleSpin, tau, bk, 0);
    launched(c, launch_clamp01(vsum, px * K, c->st), "clamp");
    float* wgt = buf<float>(c, "v.wgt", (size_t)M * N);
    launched(c, launch_ht_weights(vsum, m, n, M, N, d, K, nullptr, wgt, c->st), "ht_weights");
    double* dU = buf<double>(c, "v.U", px * frames);
    double* dW = buf<double>(c, "v.W", px * frames);
    VideoAggArgs G{};
    G.S = dS;
    G.wgt = wgt;
    G.vsum = vsum;
    G.M = M;
    G.N = N;
    G.d = d;
    G.K = K;
    G.F = frames;
    G.m = m;
    G.n = n;
    G.U = dU;
    G.W = dW;
    launched(c, launch_aggregate_video(G, c->st), "aggregate_video");
    ck(c, cudaMemcpyAsync(U, dU, px * frames * 8, cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaMemcpyAsync(W, dW, px * frames * 8, cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
  });
}

int gbm3d_denoise_rgb_device(gbm3d_ctx* c, const double* R, const double* G, const double* B, int m, int n,
                             double sigma, const gbm3d_opts* o, double* UR, double* UG, double* UB) {
  return guarded(c, [&] {
    if (!R || !G || !B || !UR || !UG || !UB) argfail(c, "missing argument");
    const double* in[3] = {R, G, B};
    double* out[3] = {UR, UG, UB};
    pipeline_rgb(c, in, m, n, sigma, o, out);
  });
}

}  // extern "C"

namespace {

// Runs run_all() eagerly, or, with use_graph, replays the context's captured
// graph when its key matches; otherwise runs it eagerly (which sizes every
// workspace buffer and produces this call's result) and then captures the
// same launch sequence once for later calls with this key.
template <class F>
void run_graph(gbm3d_ctx* c, const std::string& key, bool use_graph, F&& run_all) {
  if (!use_graph) {
    run_all();
    return;
  }
  if (c->graph_exec && c->graph_key == key) {  // same geometry: replay
    ck(c, cudaGraphLaunch(c->graph_exec, c->st), "cudaGraphLaunch");
    c->launches = 1;
    return;
  }
  run_all();
  const bool tm = c->timing;
  c->timing = false;
  ck(c, cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
  cudaGraph_t g = nullptr;
  try {
    run_all();
  } catch (...) {
    cudaStreamEndCapture(c->st, &g);
    if (g) cudaGraphDestroy(g);
    c->timing = tm;
    throw;
  }
  c->timing = tm;
  ck(c, cudaStreamEndCapture(c->st, &g), "cudaStreamEndCapture");
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  c->graph_exec = nullptr;
  c->graph_key.clear();
  const cudaError_t e = cudaGraphInstantiate(&c->graph_exec, g, 0);
  cudaGraphDestroy(g);
  ck(c, e, "cudaGraphInstantiate");
  c->graph_key = key;
}

template <class T>
void key_add(std::string& key, const T& v) {
  key.append(reinterpret_cast<const char*>(&v), sizeof(T));
}

}  // namespace

extern "C" {

int gbm3d_denoise_batch(gbm3d_ctx* c, int nimg, const double* const* I, const int* m, const int* n,
                        const double* sigma, const gbm3d_opts* o, double* const* U, int use_graph) {
  return guarded(c, [&] {
    if (nimg < 1 || !I || !m || !n || !sigma || !U || !o) argfail(c, "missing argument");
    for (int k = 0; k < nimg; ++k)
      if (!I[k] || !U[k]) argfail(c, "missing image or output pointer");
    // largest images first: the workspace reaches its final size on the first ones
    std::vector<int> ord(nimg);
    for (int k = 0; k < nimg; ++k) ord[k] = k;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return (long)m[a] * n[a] > (long)m[b] * n[b]; });
    std::string key("batch");
    key_add(key, *o);
    for (int k = 0; k < nimg; ++k) {
      key_add(key, I[k]);
      key_add(key, U[k]);
      key_add(key, m[k]);
      key_add(key, n[k]);
      key_add(key, sigma[k]);
    }
    run_graph(c, key, use_graph != 0, [&] {
      for (int k : ord) pipeline(c, I[k], m[k], n[k], sigma[k], o, U[k], nullptr);
    });
  });
}

int gbm3d_denoise_mixed(gbm3d_ctx* c, const gbm3d_mixed_batch* b, const gbm3d_opts* o,
                        const gbm3d_opts* ov, int use_graph) {
  return guarded(c, [&] {
    if (!b || !o) argfail(c, "missing argument");
    if (b->n_grey < 0 || b->n_rgb < 0) argfail(c, "negative image count");
    if (b->n_grey > 0 && (!b->grey || !b->grey_m || !b->grey_n || !b->grey_sigma || !b->grey_out))
      argfail(c, "missing grey-image arrays");
    if (b->n_rgb > 0 && (!b->rgb || !b->rgb_m || !b->rgb_n || !b->rgb_sigma || !b->rgb_out))
      argfail(c, "missing colour-image arrays");
    if (b->video && (!ov || !b->video_out)) argfail(c, "video without options or output");
    for (int k = 0; k < b->n_grey; ++k)
      if (!b->grey[k] || !b->grey_out[k]) argfail(c, "missing grey image or output pointer");
    for (int k = 0; k < 3 * b->n_rgb; ++k)
      if (!b->rgb[k] || !b->rgb_out[k]) argfail(c, "missing colour plane or output pointer");
    if (b->n_grey == 0 && b->n_rgb == 0 && !b->video) argfail(c, "empty batch");
    std::vector<int> og(b->n_grey), orgb(b->n_rgb);
    for (int k = 0; k < b->n_grey; ++k) og[k] = k;
    for (int k = 0; k < b->n_rgb; ++k) orgb[k] = k;
    auto larger = [](const int* mm, const int* nn) {
      return [mm, nn](int x, int y) { return (long)mm[x] * nn[x] > (long)mm[y] * nn[y]; };
    };
    std::stable_sort(og.begin(), og.end(), larger(b->grey_m, b->grey_n));
    std::stable_sort(orgb.begin(), orgb.end(), larger(b->rgb_m, b->rgb_n));
    // each image's options: its own entry of grey_opts / rgb_opts, else opts
    auto grey_o = [&](int k) { return b->grey_opts ? b->grey_opts + k : o; };
    auto rgb_o = [&](int k) { return b->rgb_opts ? b->rgb_opts + k : o; };
    bool learned = o->form == 2;
    for (int k = 0; k < b->n_grey; ++k) learned |= grey_o(k)->form == 2;
    for (int k = 0; k < b->n_rgb; ++k) learned |= rgb_o(k)->form == 2;
    std::string key("mixed");
    key_add(key, *o);
    if (b->video) key_add(key, *ov);
    key_add(key, (int)(b->grey_opts != nullptr));
    key_add(key, (int)(b->rgb_opts != nullptr));
    for (int k = 0; k < b->n_grey; ++k) {
      if (b->grey_opts) key_add(key, b->grey_opts[k]);
      key_add(key, b->grey[k]);
      key_add(key, b->grey_out[k]);
      key_add(key, b->grey_m[k]);
      key_add(key, b->grey_n[k]);
      key_add(key, b->grey_sigma[k]);
    }
    for (int k = 0; k < b->n_rgb; ++k) {
      if (b->rgb_opts) key_add(key, b->rgb_opts[k]);
      for (int q = 0; q < 3; ++q) {
        key_add(key, b->rgb[3 * k + q]);
        key_add(key, b->rgb_out[3 * k + q]);
      }
      key_add(key, b->rgb_m[k]);
      key_add(key, b->rgb_n[k]);
      key_add(key, b->rgb_sigma[k]);
    }
    key_add(key, b->video);
    if (b->video) {
      key_add(key, b->video_out);
      key_add(key, b->video_m);
      key_add(key, b->video_n);
      key_add(key, b->video_frames);
      key_add(key, b->video_sigma);
    }
    // items (kind 0 grey, 1 colour, 2 video) in decreasing estimated work, each
    // given to the lane with the least work so far (longest processing time
    // first); a lane runs its items in that order on its own stream
    struct Item {
      int kind, k;
      double work;
    };
    std::vector<Item> items;
    for (int k : og) items.push_back({0, k, (double)b->grey_m[k] * b->grey_n[k]});
    for (int k : orgb) items.push_back({1, k, 3.0 * b->rgb_m[k] * b->rgb_n[k]});
    if (b->video) items.push_back({2, 0, 2.0 * b->video_m * b->video_n * b->video_frames});
    std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) { return x.work > y.work; });
    // the learned pilot's parameters live in unprefixed buffers: one lane
    const int L = std::max(1, std::min({c->lanes, (int)items.size(), learned ? 1 : 16}));
    key_add(key, L);
    std::vector<int> lane(items.size(), 0);
    {
      std::vector<double> load(L, 0.0);
      for (size_t t = 0; t < items.size(); ++t) {
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        lane[t] = l;
        load[l] += items[t].work;
      }
    }
    while ((int)c->lane_st.size() < L) {
      cudaStream_t st;
      ck(c, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
      c->lane_st.push_back(st);
    }
    while ((int)c->lane_ev.size() < L + 1) {
      cudaEvent_t e;
      ck(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
      c->lane_ev.push_back(e);
    }
    auto run_item = [&](const Item& it) {
      const int k = it.k;
      if (it.kind == 0)
        pipeline(c, b->grey[k], b->grey_m[k], b->grey_n[k], b->grey_sigma[k], grey_o(k), b->grey_out[k], nullptr);
      else if (it.kind == 1)
        pipeline_rgb(c, b->rgb + 3 * k, b->rgb_m[k], b->rgb_n[k], b->rgb_sigma[k], rgb_o(k), b->rgb_out + 3 * k);
      else
        pipeline_video(c, b->video, b->video_m, b->video_n, b->video_frames, b->video_sigma, ov, b->video_out);
    };
    run_graph(c, key, use_graph != 0, [&] {
      if (L == 1) {
        for (const Item& it : items) run_item(it);
        return;
      }
      // fork: every lane waits for the work already on the context stream
      cudaStream_t origin = c->st;
      struct Restore {  // the context's stream and buffer names, also when an item throws
        gbm3d_ctx* c;
        cudaStream_t st;
        ~Restore() {
          c->st = st;
          c->ns.clear();
        }
      } restore{c, origin};
      ck(c, cudaEventRecord(c->lane_ev[0], origin), "cudaEventRecord");
      for (int l = 0; l < L; ++l) ck(c, cudaStreamWaitEvent(c->lane_st[l], c->lane_ev[0], 0), "cudaStreamWaitEvent");
      for (size_t t = 0; t < items.size(); ++t) {
        c->st = c->lane_st[lane[t]];
        c->ns = "lane" + std::to_string(lane[t]) + ".";
        run_item(items[t]);
      }
      c->st = origin;
      c->ns.clear();
      // join: the context stream waits for every lane
      for (int l = 0; l < L; ++l) {
        ck(c, cudaEventRecord(c->lane_ev[1 + l], c->lane_st[l]), "cudaEventRecord");
        ck(c, cudaStreamWaitEvent(origin, c->lane_ev[1 + l], 0), "cudaStreamWaitEvent");
      }
    });
  });
}

int gbm3d_denoise_device(gbm3d_ctx* c, const double* I, int m, int n, double sigma, const gbm3d_opts* o,
                         double* U, double* U1) {
  return guarded(c, [&] {
    if (!I || !U) argfail(c, "missing argument");
    pipeline(c, I, m, n, sigma, o, U, U1);
  });
}

int gbm3d_denoise_strip_device(gbm3d_ctx* c, const double* I, int m, int n, double sigma, const gbm3d_opts* o,
                               int col_lo, int col_hi, double* U) {
  return guarded(c, [&] {
    if (!I || !U) argfail(c, "missing argument");
    if (m < 1 || n < 1 || m > 32000 || n > 32000) argfail(c, "image size out of range");
    if (col_lo < 0 || col_hi > n || col_lo >= col_hi) argfail(c, "strip columns must satisfy 0 <= col_lo < col_hi <= n");
    double* full = buf<double>(c, "strip.U", (size_t)m * n);
    pipeline(c, I, m, n, sigma, o, full, nullptr, nullptr, nullptr, col_lo, col_hi);
    ck(c, cudaMemcpyAsync(U, full + (size_t)col_lo * m, (size_t)m * (col_hi - col_lo) * sizeof(double),
                          cudaMemcpyDeviceToDevice, c->st),
       "D2D");
  });
}

int gbm3d_strip_work(const gbm3d_opts* o, int m, int n, int col_lo, int col_hi, double* frac) {
  if (!o || !frac || m < 1 || n < 1 || m > 32000 || n > 32000 || col_lo < 0 || col_hi > n || col_lo >= col_hi)
    return GBM3D_ERR_ARG;
  try {
    int d, dw, d2, K;
    opts_dims(o, d, dw, d2, K);
    const int st1 = stride1(o), st2 = stride2(o);
    if (!match_supported(d, d2) || o->levels < 1 || o->levels > GBM3D_MAX_LEVELS || o->cycleSpin < 1 ||
        o->nMatchSpins < 1 || o->nMatchSpins > 8 || (o->Wiener && (o->nMatchSpinsWie < 1 || o->nMatchSpinsWie > 8)) ||
        st1 < 1 || st1 > d || st2 < 1 || st2 > dw || (o->Wiener && (d - dw) % std::gcd(st1, st2) != 0))
      return GBM3D_ERR_ARG;
    const int Mp = padded_size(o, m, d, dw, st1, st2), Np = padded_size(o, n, d, dw, st1, st2);
    gbm3d_filters f;
    bank_of_opts(o, &f);
    const WaveletBank bk = make_bank(nullptr, &f);
    const StripCols P = strip_cols(o, Mp, Np, d, dw, d2, st1, st2, col_lo, col_hi, bk);
    const int N1 = grid_count(Np, d, st1), N2 = grid_count(Np, dw, st2);
    auto span = [](const ColRange& r, int N) { return r.all(N) ? N : r.len; };
    double a = 0, b = 0;
    for (const auto& w : P.s1) a += (double)span(w.match, N1) / N1;
    for (const auto& w : P.s2) b += (double)span(w.groups, N2) / N2;
    frac[0] = P.s1.empty() ? 0.0 : a / P.s1.size();
    frac[1] = P.s2.empty() ? 0.0 : b / P.s2.size();
    return GBM3D_OK;
  } catch (const Fail& e) {
    return e.code;
  }
}

static int denoise_host(gbm3d_ctx* c, const double* I, int m, int n, double sigma, const gbm3d_opts* o, double* U,
                        double* U1, const double* tau, const double* sigwie) {
  return guarded(c, [&] {
    if (!I || !U) argfail(c, "missing argument");
    if (m < 1 || n < 1 || m > 32000 || n > 32000) argfail(c, "image size out of range");
    const size_t px = (size_t)m * n;
    double* dI = buf<double>(c, "h.I", px);
    double* dU = buf<double>(c, "h.U", px);
    double* dU1 = U1 ? buf<double>(c, "h.U1", px) : nullptr;
    ck(c, cudaMemcpyAsync(dI, I, px * 8, cudaMemcpyHostToDevice, c->st), "H2D");
    pipeline(c, dI, m, n, sigma, o, dU, dU1, tau, sigwie);
    ck(c, cudaMemcpyAsync(U, dU, px * 8, cudaMemcpyDeviceToHost, c->st), "D2H");
    if (U1) ck(c, cudaMemcpyAsync(U1, dU1, px * 8, cudaMemcpyDeviceToHost, c->st), "D2H");
    int flag = 0;
    ck(c, cudaMemcpyAsync(&flag, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
    report_flag(c, flag);
  });
}

int gbm3d_denoise(gbm3d_ctx* c, const double* I, int m, int n, double sigma, const gbm3d_opts* o, double* U,
                  double* U1) {
  return denoise_host(c, I, m, n, sigma, o, U, U1, nullptr, nullptr);
}

int gbm3d_denoise_async(gbm3d_ctx* c, const double* I, int m, int n, double sigma, const gbm3d_opts* o,
                        double* U) {
  return guarded(c, [&] {
    if (!I || !U || !o) argfail(c, "missing argument");
    if (m < 1 || n < 1 || m > 32000 || n > 32000) argfail(c, "image size out of range");
    if (!c->h2d) {
      ck(c, cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking), "cudaStreamCreate");
      ck(c, cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking), "cudaStreamCreate");
      for (int k = 0; k < 2; ++k)
        for (cudaEvent_t* e : {&c->in_ready[k], &c->in_free[k], &c->out_ready[k], &c->out_free[k]})
          ck(c, cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
      ck(c, cudaMalloc(&c->sticky, sizeof(int)), "cudaMalloc");
      ck(c, cudaMemset(c->sticky, 0, sizeof(int)), "cudaMemset");
    }
    const size_t px = (size_t)m * n;
    const int k = c->slot;
    double* dI = buf<double>(c, k ? "a.I1" : "a.I0", px);
    double* dU = buf<double>(c, k ? "a.U1" : "a.U0", px);
    // H2D into this slot once the compute of the call two back has read it
    ck(c, cudaStreamWaitEvent(c->h2d, c->in_free[k], 0), "cudaStreamWaitEvent");
    ck(c, cudaMemcpyAsync(dI, I, px * 8, cudaMemcpyHostToDevice, c->h2d), "H2D");
    ck(c, cudaEventRecord(c->in_ready[k], c->h2d), "cudaEventRecord");
    // compute once the input is in and the D2H of the call two back has read the output slot
    ck(c, cudaStreamWaitEvent(c->st, c->in_ready[k], 0), "cudaStreamWaitEvent");
    ck(c, cudaStreamWaitEvent(c->st, c->out_free[k], 0), "cudaStreamWaitEvent");
    c->async_pending = true;
    pipeline(c, dI, m, n, sigma, o, dU, nullptr);
    k_or_flag<<<1, 1, 0, c->st>>>(c->flag, c->sticky);
    launched(c, cudaGetLastError(), "flag");
    ck(c, cudaEventRecord(c->in_free[k], c->st), "cudaEventRecord");
    ck(c, cudaEventRecord(c->out_ready[k], c->st), "cudaEventRecord");
    // D2H of the result
    ck(c, cudaStreamWaitEvent(c->d2h, c->out_ready[k], 0), "cudaStreamWaitEvent");
    ck(c, cudaMemcpyAsync(U, dU, px * 8, cudaMemcpyDeviceToHost, c->d2h), "D2H");
    ck(c, cudaEventRecord(c->out_free[k], c->d2h), "cudaEventRecord");
    c->slot = k ^ 1;
  });
}

// ---- learned pilot ---------------------------------------------------------------------

int gbm3d_pilot_param_count(void) { return pilot_param_count(); }

int gbm3d_pilot_set_params(gbm3d_ctx* c, const float* params) {
  return guarded(c, [&] {
    if (!params) argfail(c, "missing argument");
    const int np = pilot_param_count();
    PilotNet P = pilot_net(c);
    float* m1 = buf<float>(c, "pl.m1", np);
    float* m2 = buf<float>(c, "pl.m2", np);
    ck(c, cudaMemcpyAsync(const_cast<float*>(P.master), params, (size_t)np * 4, cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemsetAsync(m1, 0, (size_t)np * 4, c->st), "memset");
    ck(c, cudaMemsetAsync(m2, 0, (size_t)np * 4, c->st), "memset");
    launched(c, pilot_pack_weights(P.master, P.wfwd, P.wbwd, c->st), "pilot_weights");
    ck(c, cudaStreamSynchronize(c->st), "sync");
    c->pilot_ready = true;
    c->pilot_step = 0;
  });
}

int gbm3d_pilot_get_params(gbm3d_ctx* c, float* params) {
  return guarded(c, [&] {
    if (!params) argfail(c, "missing argument");
    if (!c->pilot_ready) argfail(c, "learned pilot: no parameters loaded (gbm3d_pilot_set_params)");
    PilotNet P = pilot_net(c);
    ck(c, cudaMemcpyAsync(params, P.master, (size_t)pilot_param_count() * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
  });
}

int gbm3d_pilot_forward(gbm3d_ctx* c, const float* img, const float* sigma, int nimg, int H, int W, float* pilot) {
  return guarded(c, [&] {
    if (!img || !sigma || !pilot) argfail(c, "missing argument");
    check_pilot_dims(c, nimg, H, W);
    run_pilot(c, img, sigma, nimg, H, W, pilot);
  });
}

// forward + loss + backward; with lr > 0 also one Adam step.  grad (host, may be
// null) receives the parameter gradients, loss (host, may be null) the loss.
static int pilot_train(gbm3d_ctx* c, const float* img, const float* target, const float* sigma, int nimg, int H,
                       int W, float lr, float* grad_host, float* loss) {
  return guarded(c, [&] {
    if (!img || !target || !sigma) argfail(c, "missing argument");
    check_pilot_dims(c, nimg, H, W);
    const size_t px = (size_t)nimg * H * W;
    const int np = pilot_param_count();
    PilotNet P = pilot_net(c);
    uint16_t* acts[PILOT_LAYERS];
    pilot_acts(c, px, acts);
    float* out = buf<float>(c, "pl.out", px);
    uint16_t* dy16 = buf<uint16_t>(c, "pl.dy16", px * 16);
    uint16_t* gA = buf<uint16_t>(c, "pl.gA", px * 48);
    uint16_t* gB = buf<uint16_t>(c, "pl.gB", px * 48);
    const int nparts = 2 * c->sms;
    float* part = buf<float>(c, "pl.part", (size_t)nparts * (9 * 48 * 48 + 48));
    float* grad = buf<float>(c, "pl.grad", np);
    float* lpart = buf<float>(c, "pl.lpart", 256);
    ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
    launched(c, pilot_pack_input(img, sigma, nimg, H, W, acts[0], c->st), "pilot_pack");
    launched(c, pilot_forward(P, img, nimg, H, W, acts, out, c->flag, c->sms, c->st), "pilot_conv");
    launched(c, pilot_backward(P, out, target, nimg, H, W, acts, dy16, gA, gB, part, nparts, grad, lpart, c->flag,
                               c->sms, c->st), "pilot_backward");
    if (lr > 0.f) {
      c->pilot_step += 1;
      launched(c, pilot_adam(const_cast<float*>(P.master), grad, buf<float>(c, "pl.m1", np), buf<float>(c, "pl.m2", np),
                             np, lr, c->pilot_step, c->st), "pilot_adam");
      launched(c, pilot_pack_weights(P.master, P.wfwd, P.wbwd, c->st), "pilot_weights");
    }
    float lp[256];
    ck(c, cudaMemcpyAsync(lp, lpart, sizeof(lp), cudaMemcpyDeviceToHost, c->st), "D2H");
    if (grad_host) ck(c, cudaMemcpyAsync(grad_host, grad, (size_t)np * 4, cudaMemcpyDeviceToHost, c->st), "D2H");
    int flag = 0;
    ck(c, cudaMemcpyAsync(&flag, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
    report_flag(c, flag);
    double s = 0.0;
    for (int i = 0; i < 256; ++i) s += lp[i];
    if (loss) *loss = (float)(s / (double)px);
  });
}

int gbm3d_pilot_train_step(gbm3d_ctx* c, const float* img, const float* target, const float* sigma, int nimg, int H,
                           int W, float lr, float* loss) {
  if (!(lr > 0.f)) {
    if (c) c->err = "lr must be positive";
    return GBM3D_ERR_ARG;
  }
  return pilot_train(c, img, target, sigma, nimg, H, W, lr, nullptr, loss);
}

int gbm3d_pilot_gradients(gbm3d_ctx* c, const float* img, const float* target, const float* sigma, int nimg, int H,
                          int W, float* grad, float* loss) {
  return pilot_train(c, img, target, sigma, nimg, H, W, 0.f, grad, loss);
}

int gbm3d_denoise_colored(gbm3d_ctx* c, const double* I, int m, int n, double sigma_match, const double* tau,
                          const double* sigmaWie, const gbm3d_opts* o, double* U, double* U1) {
  if (!tau || !sigmaWie) {
    if (c) c->err = "tau and sigmaWie are required";
    return GBM3D_ERR_ARG;
  }
  return denoise_host(c, I, m, n, sigma_match, o, U, U1, tau, sigmaWie);
}

}  // extern "C"

// ---- GBM3D_distributed on the device (source/GBM3D_distributed.m:54-120) ----------------
namespace {

// out(r, c) = circshift(I(r0 + (0..ny-1), c0 + (0..nx-1)), [s, s])(r, c)
//           = I(r0 + (r - s) mod ny, c0 + (c - s) mod nx)
__global__ void k_tile_in(const double* __restrict__ I, int m, int r0, int c0, int ny, int nx, int s,
                          double* __restrict__ out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= ny || c >= nx) return;
  out[r + (size_t)c * ny] = I[(size_t)(r0 + pmod(r - s, ny)) + (size_t)(c0 + pmod(c - s, nx)) * m];
}

// circshift(U, [-s, -s]) and circshift(W, [-s, -s]) of an ny x nx tile, single -> double
__global__ void k_tile_out(const float* __restrict__ U, const float* __restrict__ W, int ny, int nx, int s,
                           double* __restrict__ outU, double* __restrict__ outW) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= ny || c >= nx) return;
  const size_t src = (size_t)pmod(r + s, ny) + (size_t)pmod(c + s, nx) * ny;
  outU[r + (size_t)c * ny] = (double)U[src];
  outW[r + (size_t)c * ny] = (double)W[src];
}

// One item's stitch (GBM3D_distributed.m:69-71): U2 += U .* win, norm += win .* W
// over its ny x nx tile at (r0, c0), win = makeInterpWindow(ny, nx, k) built
// from the ramp linspace(0.01, 1, k) in makeInterpWindow.m's order.
__global__ void k_tile_stitch(const double* __restrict__ U, const double* __restrict__ W, int ny, int nx, int r0,
                              int c0, int k, const double* __restrict__ ramp, double* __restrict__ U2,
                              double* __restrict__ nrm, int m) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= ny || c >= nx) return;
  double w = 1.0;
  if (r < k) w *= ramp[r];
  if (c < k) w *= ramp[c];
  if (r >= ny - k) w *= ramp[ny - 1 - r];
  if (c >= nx - k) w *= ramp[nx - 1 - c];
  const size_t t = r + (size_t)c * ny, o = (size_t)(r0 + r) + (size_t)(c0 + c) * m;
  U2[o] = U2[o] + U[t] * w;
  nrm[o] = nrm[o] + w * W[t];
}

__global__ void k_div(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = a[i] / b[i];
}

void check_items(gbm3d_ctx* c, const int* items, int n_items, int m, int n, int tile) {
  if (!items || n_items < 0) argfail(c, "missing item table");
  for (int ii = 0; ii < n_items; ++ii) {
    const int* R = items + 5 * ii;
    const int ny = R[1] - R[0] + 1, nx = R[3] - R[2] + 1;
    if (R[0] < 1 || R[2] < 1 || R[1] > m || R[3] > n || ny < 1 || nx < 1 || ny > tile || nx > tile)
      argfail(c, "item " + std::to_string(ii) + ": tile bounds outside the image or larger than the tile size");
  }
}

}  // namespace

extern "C" {

int gbm3d_tiles_device(gbm3d_ctx* c, const double* I, const double* pilot, int m, int n, double sigma,
                       const double* tau, const gbm3d_opts* o, const int* items, int n_items, int tile, double* out) {
  return guarded(c, [&] {
    check_opts(c, o);
    if (!I || !out || (!pilot && !tau)) argfail(c, "missing argument");
    if (m < 1 || n < 1 || tile < 1) argfail(c, "image size out of range");
    check_items(c, items, n_items, m, n, tile);
    const bool step2 = pilot != nullptr;
    const int d = step2 ? o->blockSizeWie : o->blockSize, d2 = o->matchSize, K = o->numMax;
    check_match(c, d, d2, K);
    const int s = step2 ? stride2(o) : stride1(o);
    gbm3d_filters fb;
    bior(&fb);
    const WaveletBank bk = step2 ? WaveletBank{} : make_bank(c, &fb);
    const size_t slot = (size_t)tile * tile;
    ck(c, cudaMemsetAsync(c->flag, 0, sizeof(int), c->st), "memset");
    for (int ii = 0; ii < n_items; ++ii) {
      const int* R = items + 5 * ii;
      const int r0 = R[0] - 1, c0 = R[2] - 1, ny = R[1] - R[0] + 1, nx = R[3] - R[2] + 1, sp = R[4];
      if (ny < d2 || nx < d2 || ny < d || nx < d) argfail(c, "tile smaller than matchSize");
      const int M = grid_count(ny, d, s), N = grid_count(nx, d, s);
      const int uy = (M - 1) * s + d, ux = (N - 1) * s + d;
      if (uy != ny || ux != nx) argfail(c, "tile sides must be whole reference grids");
      const size_t px = (size_t)ny * nx;
      double* dT = buf<double>(c, "tl.I", px);
      k_tile_in<<<grid2(ny, nx), 256, 0, c->st>>>(I, m, r0, c0, ny, nx, sp, dT);
      launched(c, cudaGetLastError(), "tile_in");
      float* Tf = buf<float>(c, "tl.If", px);
      k_prep<<<grid2(ny, nx), 256, 0, c->st>>>(dT, ny, nx, Tf, ny, nx, c->flag);
      launched(c, cudaGetLastError(), "prep");
      uint32_t* dS = buf<uint32_t>(c, "tl.S", (size_t)K * M * N);
      float* dU = buf<float>(c, "tl.U", px);
      float* dW = buf<float>(c, "tl.W", px);
      if (!step2) {
        // [S, Volume] = matchBlocksCPU(Ilocal); [U, W] = denoiseAndAggregateGPU(...)
        int32_t* dc = buf<int32_t>(c, "tl.cnt", (size_t)M * N);
        const size_t vn = s == d ? px * K : (size_t)M * d * N * d * K;
        float* dV = buf<float>(c, "tl.V", vn);
        ck(c, cudaMemsetAsync(dV, 0, vn * sizeof(float), c->st), "memset");
        run_match(c, Tf, nullptr, ny, nx, 0, d, d2, K, o->numMin, sigma, dS, dc, dV, nullptr, nullptr, "tl1", s,
                  o->form);
        run_ht(c, dV, dS, dc, M, N, d, d2, K, o->levels, o->cycleSpin, tau, bk, dU, dW, o->filtType, s);
      } else {
        // [S, V1, V2] = matchBlocksWie(pilot tile, noisy tile); denoiseAndAggregateWieFast
        double* dP = buf<double>(c, "tl.P", px);
        k_tile_in<<<grid2(ny, nx), 256, 0, c->st>>>(pilot, m, r0, c0, ny, nx, sp, dP);
        launched(c, cudaGetLastError(), "tile_in");
        float* Pf = buf<float>(c, "tl.Pf", px);
        k_prep<<<grid2(ny, nx), 256, 0, c->st>>>(dP, ny, nx, Pf, ny, nx, c->flag);
        launched(c, cudaGetLastError(), "prep");
        const size_t gs = (size_t)d * d * K * M * N;
        float* d1 = buf<float>(c, "tl.V1", gs);
        float* d2p = buf<float>(c, "tl.V2", gs);
        run_match(c, Pf, Tf, ny, nx, 0, d, d2, K, K, sigma, dS, nullptr, nullptr, d1, d2p, "tl2", s, o->form);
        WienerArgs A{};
        A.V1 = d1;
        A.V2 = d2p;
        A.S = dS;
        A.M = M;
        A.N = N;
        A.K = K;
        A.s = s;
        A.d2 = d2;
        fill_wiener_consts(A, d, &sigma, 0, 0);
        run_wiener_agg(c, A, d, d2, dU, dW);
      }
      k_tile_out<<<grid2(ny, nx), 256, 0, c->st>>>(dU, dW, ny, nx, sp, out + 2 * slot * ii,
                                                  out + 2 * slot * ii + slot);
      launched(c, cudaGetLastError(), "tile_out");
    }
    int flag = 0;
    ck(c, cudaMemcpyAsync(&flag, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->st), "D2H");
    ck(c, cudaStreamSynchronize(c->st), "sync");
    report_flag(c, flag);
  });
}

int gbm3d_tiles_stitch_device(gbm3d_ctx* c, const double* tiles, const int* items, int n_items, int tile, int m,
                              int n, int k, const double* ramp, double* out) {
  return guarded(c, [&] {
    if (!tiles || !out || !ramp || k < 1 || k > 256) argfail(c, "missing argument");
    check_items(c, items, n_items, m, n, tile);
    const size_t px = (size_t)m * n, slot = (size_t)tile * tile;
    double* U2 = buf<double>(c, "st.U2", px);
    double* nrm = buf<double>(c, "st.norm", px);
    double* dr = buf<double>(c, "st.ramp", (size_t)k);
    ck(c, cudaMemcpyAsync(dr, ramp, (size_t)k * sizeof(double), cudaMemcpyHostToDevice, c->st), "H2D");
    ck(c, cudaMemsetAsync(U2, 0, px * sizeof(double), c->st), "memset");
    ck(c, cudaMemsetAsync(nrm, 0, px * sizeof(double), c->st), "memset");
    for (int ii = 0; ii < n_items; ++ii) {  // item order: every pixel adds its tiles in table order
      const int* R = items + 5 * ii;
      const int ny = R[1] - R[0] + 1, nx = R[3] - R[2] + 1;
      if (ny < 2 * k || nx < 2 * k) argfail(c, "tile shorter than two ramps");
      k_tile_stitch<<<grid2(ny, nx), 256, 0, c->st>>>(tiles + 2 * slot * ii, tiles + 2 * slot * ii + slot, ny, nx,
                                                     R[0] - 1, R[2] - 1, k, dr, U2, nrm, m);
      launched(c, cudaGetLastError(), "tile_stitch");
    }
    k_div<<<(unsigned)std::min<size_t>((px + 255) / 256, 4096), 256, 0, c->st>>>(U2, nrm, out, px);
    launched(c, cudaGetLastError(), "div");
    ck(c, cudaStreamSynchronize(c->st), "sync");
  });
}

}  // extern "C"
