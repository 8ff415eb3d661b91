// CPU ORACLE — test infrastructure only. Not part of the product.
//
// A C++ restatement of the GBM3D two-step denoising path of the MATLAB
// reference (toby-sanders/GBM3D). Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py load this library, always to
// check results against or as the timed CPU baseline, never as the product.
//
// PARITY UNPINNED: the reference is MATLAB-only, ships no tests, no golden
// vectors and no known-answer tests, and neither MATLAB nor Octave can run here.
// This restatement is cross-checked against a second, independent restatement
// that follows the reference's FFT route literally (oracle/fft_route.py, whose
// outputs are committed as tests/golden/*.npz) and against project
// known-answer tests (perfect reconstruction, padding, slot-1, tie order).
//
// Two precisions from one template:
//   T = float : "FP32 GPU order".  Every floating-point operation follows the
//               operation order of the CUDA kernels, so the CUDA path must be
//               bit-identical to this mode.
//   T = double: the same code in FP64, the reference run used to state error.
//
// Arithmetic conventions (shared with the CUDA kernels):
//   * a double operand that MATLAB mixes into single-precision arithmetic is
//     converted to single first (tau, eps, mask, sigma^2, DCT matrices);
//   * circular convolutions are computed directly from their definition
//     (what the reference computes through fftn/ifftn), taps with a zero
//     coefficient are skipped, and every multi-term sum is a serial fma chain
//     in a stated order;
//   * reductions (TV weight terms, Wiener gain norm) use a fixed 32-way
//     strided partial sum followed by an xor butterfly (red32 below);
//   * block distances are exact sums of squared differences, ranked by value
//     then by column-major window index (MATLAB mink's stable order).  The
//     reference divides all distances of one reference block by the same
//     positive ||xR||^2; that scaling cannot reorder them, so it is omitted
//     except where the tolerance branch compares against tol.
//
// Layouts are MATLAB column-major: image (r,c) at r + c*m.

#include <algorithm>
#include <cmath>
#include <numeric>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <class T> inline T fmaT(T a, T b, T c) { return std::fma(a, b, c); }

// ---------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------

// Row index into the reference's padded search image Ipad
// (source/matchBlocksCPU.m:57-61): Ipad = circshift(tile(I,2x2)(1:L+d2), d2/2).
// Rows 0..h-1 hold I rows h..2h-1 (not a periodic wrap), rows h..L+h-1 hold
// I rows 0..L-1, rows L+h..L+d2-1 hold I rows 0..h-1.
inline int pad_index(int r, int L, int h) { return r < h ? r + h : (r - h) % L; }

inline int pmod(int a, int L) { int r = a % L; return r < 0 ? r + L : r; }

// Fixed-order reduction: 32 strided partial sums, then xor butterfly.
template <class T, class F> T red32(int count, F value_at) {
  T p[32];
  for (int l = 0; l < 32; ++l) p[l] = T(0);
  for (int e = 0; e < count; ++e) p[e & 31] = p[e & 31] + value_at(e);
  for (int off = 16; off >= 1; off >>= 1) {
    T q[32];
    for (int l = 0; l < 32; ++l) q[l] = p[l] + p[l ^ off];
    for (int l = 0; l < 32; ++l) p[l] = q[l];
  }
  return p[0];
}

// sin window outer(sin(pi*linspace(lo,hi,d))) — denoiseAndAggregateGPU.m:65-67
// (lo,hi)=(.1,.9) and denoiseAndAggregateWieFast.m (lo,hi)=(.2,.8).
void sine_window(int d, double lo, double hi, double* w) {
  std::vector<double> v(d);
  for (int i = 0; i < d; ++i) {
    double t = (d == 1) ? hi : (i == d - 1 ? hi : lo + i * (hi - lo) / (d - 1));
    v[i] = std::sin(M_PI * t);
  }
  for (int c = 0; c < d; ++c)
    for (int r = 0; r < d; ++r) w[r + c * d] = v[r] * v[c];
}

// T = dct(eye(d)) (orthonormal DCT-II) and Tinv = inv(T) by Gauss-Jordan with
// partial pivoting — denoiseAndAggregateWieFast.m:33-34.
void dct_matrices(int d, double* Tm, double* Ti) {
  for (int k = 0; k < d; ++k)
    for (int n = 0; n < d; ++n) {
      double ck = (k == 0) ? std::sqrt(1.0 / d) : std::sqrt(2.0 / d);
      Tm[k + n * d] = ck * std::cos(M_PI * (2 * n + 1) * k / (2.0 * d));
    }
  std::vector<double> a(d * 2 * d);
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < 2 * d; ++c)
      a[r * 2 * d + c] = c < d ? Tm[r + c * d] : (c - d == r ? 1.0 : 0.0);
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

}  // namespace

// ---------------------------------------------------------------------------
// Public structs (mirrored in oracle/oracle.py)
// ---------------------------------------------------------------------------
extern "C" {

// Separable 3D filter bank: 1D filters for the two spatial axes and for the
// slot axis.  getWaveFilters3Dbior.m:12-58 builds Psi/Psi2 as outer products
// of exactly these factors.
typedef struct {
  int len_xy;
  double a_lo_xy[16], a_hi_xy[16], s_lo_xy[16], s_hi_xy[16];
  int len_z;
  double a_lo_z[16], a_hi_z[16], s_lo_z[16], s_hi_z[16];
} orc_filters;

typedef struct {
  int numMax, numMin, blockSize, blockSizeWie, matchSize;
  int levels, cycleSpin, tauMode, Wiener;
  int nSpins, spins[8];
  int nSpinsWie, spinsWie[8];
  int staleWeights;  // GBM3D.m:26-27,82 slice-reuse behaviour (1 = mirror it)
  int filtType;      // 0 'ht', 1 'median' (denoiseAndAggregateGPU.m:19,49)
  int refStride, refStrideWie;  // reference spacing per step; 0 = block size (the reference)
  int wavelet;                  // step-1 bank: 0 = bior1.5 x Haar (GBM3D.m:40), 1 = 3D Haar
} orc_opts;

}  // extern "C"

namespace {

// ---------------------------------------------------------------------------
// Block matching — matchBlocksCPU.m:21-116 and matchBlocksWie.m:21-92
// ---------------------------------------------------------------------------
template <class T>
struct MatchOut {
  uint32_t* S;     // K x refs (cell order i + M*j), 1-based window index
  int32_t* cnt;    // refs, numel(S{i,j})
  T* Volume;       // m x n x K, or null
  T* V1; T* V2;    // d x d x K x M x N, or null
};

// References sit at (i*s, j*s), s = refStride (the reference tiles with
// s = d).  Volume is image-shaped (m x n x K) when s = d, as in the reference,
// and tile-space (M*d x N*d x K) otherwise: group (i,j) always fills the tile
// rows i*d.., columns j*d...
template <class T>
void match_blocks(const T* I, const T* In, int m, int n, int d, int d2, int K,
                  int numMin, double tol, bool tol_branch, MatchOut<T> o, int stride) {
  const int h = d2 / 2, Wd = d + d2 - 1, s = stride;
  const int M = (m - d) / s + 1, N = (n - d) / s + 1;
  const int vm = s == d ? m : M * d, vn = s == d ? n : N * d;
  const uint32_t ref_idx = (uint32_t)(h + h * d2 + 1);  // matchBlocksCPU.m:103
#pragma omp parallel
  {
    std::vector<T> win(Wd * Wd), win2(In ? Wd * Wd : 0), ssd(d2 * d2);
    std::vector<std::pair<T, int>> keys(d2 * d2);
#pragma omp for schedule(dynamic, 16) collapse(2)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < M; ++i) {
        const int g = i + M * j;
        // local search window Itmp = Ipad(i*d + (0..Wd-1), j*d + (0..Wd-1))
        for (int c = 0; c < Wd; ++c) {
          int sc = pad_index(j * s + c, n, h);
          for (int r = 0; r < Wd; ++r) {
            int sr = pad_index(i * s + r, m, h);
            win[r + c * Wd] = I[sr + (size_t)sc * m];
            if (In) win2[r + c * Wd] = In[sr + (size_t)sc * m];
          }
        }
        // reference block xR = I(i*d.., j*d..) = Itmp(h.., h..)
        auto X = [&](int r, int c) { return win[(h + r) + (h + c) * Wd]; };
        // exact SSD for every offset (a,b); per candidate the sum runs over
        // block rows r (outer) and columns c (inner): t = x - y, acc = fma(t,t,acc).
        std::fill(ssd.begin(), ssd.end(), T(0));
        for (int r = 0; r < d; ++r)
          for (int c = 0; c < d; ++c) {
            const T xv = X(r, c);
            for (int b = 0; b < d2; ++b) {
              const T* wcol = &win[(b + c) * Wd + r];
              T* acc = &ssd[b * d2];
              for (int a = 0; a < d2; ++a) {
                T t = xv - wcol[a];
                acc[a] = fmaT(t, t, acc[a]);
              }
            }
          }
        for (int e = 0; e < d2 * d2; ++e) keys[e] = {ssd[e], e};
        auto less = [](const std::pair<T, int>& x, const std::pair<T, int>& y) {
          return x.first < y.first || (x.first == y.first && x.second < y.second);
        };
        std::vector<int> sel;
        if (!tol_branch) {
          std::partial_sort(keys.begin(), keys.begin() + K, keys.end(), less);
          for (int k = 0; k < K; ++k) sel.push_back(keys[k].second);
        } else {
          // matchBlocksCPU.m:89-99: find(D<tol), clamped to [numMin,numMax]
          // by mink.  D = ssd / ||xR||^2.
          T nR = T(0);
          for (int c = 0; c < d; ++c)
            for (int r = 0; r < d; ++r) nR = fmaT(X(r, c), X(r, c), nR);
          const T tolT = (T)tol;
          for (int e = 0; e < d2 * d2; ++e)
            if (ssd[e] / nR < tolT) sel.push_back(e);
          int want = -1;
          if ((int)sel.size() > K) want = K;
          else if ((int)sel.size() < numMin) want = numMin;
          if (want > 0) {
            std::partial_sort(keys.begin(), keys.begin() + want, keys.end(), less);
            sel.clear();
            for (int k = 0; k < want; ++k) sel.push_back(keys[k].second);
          }
        }
        const int cnt = (int)sel.size();
        uint32_t* Sg = o.S + (size_t)g * K;
        for (int k = 0; k < K; ++k) Sg[k] = k < cnt ? (uint32_t)(sel[k] + 1) : 0u;
        Sg[0] = ref_idx;
        if (o.cnt) o.cnt[g] = cnt;
        // gather (matchBlocksCPU.m:107-114, matchBlocksWie.m:85-89)
        for (int k = 0; k < K; ++k) {
          int a, b;
          bool real = k < cnt;
          if (real) { int e = (int)Sg[k] - 1; a = e % d2; b = e / d2; }
          else { a = h; b = h; }  // padding with the reference block (:114)
          for (int c = 0; c < d; ++c)
            for (int r = 0; r < d; ++r) {
              T v = win[(a + r) + (b + c) * Wd];
              if (o.Volume)
                o.Volume[(size_t)(i * d + r) + (size_t)(j * d + c) * vm + (size_t)k * vm * vn] = v;
              if (o.V1 && real) {
                size_t off = r + (size_t)d * (c + (size_t)d * (k + (size_t)K * (i + (size_t)M * j)));
                o.V1[off] = v;
                if (o.V2) o.V2[off] = win2[(a + r) + (b + c) * Wd];
              }
            }
        }
      }
  }
}

// ---------------------------------------------------------------------------
// 3D wavelet analysis / synthesis — myWavDec3DFFT.m:10-23, myWavRec3DGPUfast.m:10-40
// Volumes are (Ly, Lx, Lz) column-major (y fastest).
// ---------------------------------------------------------------------------
template <class T>
struct Bank1D {  // one axis: analysis lo/hi, synthesis lo/hi as T with tap lists
  std::vector<std::pair<int, T>> a[2], s[2];
};

template <class T>
Bank1D<T> make_bank(int len, const double* alo, const double* ahi, const double* slo, const double* shi) {
  Bank1D<T> b;
  const double* src[4] = {alo, ahi, slo, shi};
  for (int f = 0; f < 4; ++f)
    for (int k = 0; k < len; ++k)
      if (src[f][k] != 0.0) {
        auto& v = f < 2 ? b.a[f] : b.s[f - 2];
        v.push_back({k, (T)src[f][k]});
      }
  return b;
}

// analysis along one axis with decimation: out[q] = sum_k h[k] in[(2q-k) mod L]
// (taps k < L only: fftn(Psi,size) truncates a filter longer than the axis).
template <class T>
void analysis_axis(const std::vector<T>& in, int Ly, int Lx, int Lz, int axis,
                   const std::vector<std::pair<int, T>>& h, std::vector<T>& out) {
  int Oy = Ly, Ox = Lx, Oz = Lz;
  int L = axis == 0 ? Ly : axis == 1 ? Lx : Lz;
  if (axis == 0) Oy /= 2; else if (axis == 1) Ox /= 2; else Oz /= 2;
  out.assign((size_t)Oy * Ox * Oz, T(0));
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < Oz; ++z)
    for (int x = 0; x < Ox; ++x)
      for (int y = 0; y < Oy; ++y) {
        T acc = T(0);
        for (auto& t : h) {
          if (t.first >= L) continue;
          int yy = y, xx = x, zz = z;
          if (axis == 0) yy = pmod(2 * y - t.first, L);
          else if (axis == 1) xx = pmod(2 * x - t.first, L);
          else zz = pmod(2 * z - t.first, L);
          acc = fmaT(t.second, in[yy + (size_t)Ly * (xx + (size_t)Lx * zz)], acc);
        }
        out[y + (size_t)Oy * (x + (size_t)Ox * z)] = acc;
      }
}

// synthesis along one axis with upsampling, two bands (lo then hi):
// out[p] = sum_band sum_k g[k] up[(p+k) mod L], up[2q] = band[q].
template <class T>
void synthesis_axis(const std::vector<T>& lo, const std::vector<T>& hi, int Iy, int Ix, int Iz,
                    int axis, const Bank1D<T>& bk, std::vector<T>& out) {
  int Oy = Iy, Ox = Ix, Oz = Iz;
  if (axis == 0) Oy *= 2; else if (axis == 1) Ox *= 2; else Oz *= 2;
  int L = axis == 0 ? Oy : axis == 1 ? Ox : Oz;
  out.assign((size_t)Oy * Ox * Oz, T(0));
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < Oz; ++z)
    for (int x = 0; x < Ox; ++x)
      for (int y = 0; y < Oy; ++y) {
        int p = axis == 0 ? y : axis == 1 ? x : z;
        T acc = T(0);
        for (int band = 0; band < 2; ++band) {
          const std::vector<T>& src = band ? hi : lo;
          for (auto& t : bk.s[band]) {
            if (t.first >= L) continue;
            int pk = (p + t.first) % L;
            if (pk & 1) continue;
            int q = pk / 2, yy = y, xx = x, zz = z;
            if (axis == 0) yy = q; else if (axis == 1) xx = q; else zz = q;
            acc = fmaT(t.second, src[yy + (size_t)Iy * (xx + (size_t)Ix * zz)], acc);
          }
        }
        out[y + (size_t)Oy * (x + (size_t)Ox * z)] = acc;
      }
}

// band code = fy + 2 fx + 4 fz (1 = high-pass); reference detail index j
// (Psi(:,:,:,j+1), getWaveFilters3Dbior.m:39-46) for codes 1..7.
const int kDetailJ[8] = {-1, 0, 1, 3, 2, 4, 5, 6};

template <class T>
void wavelet_ht(std::vector<T>& V, int Ly, int Lx, int Lz, int levels, const double* tau,
                const Bank1D<T>& bxy, const Bank1D<T>& bz) {
  // analysis (myWavDec3DFFT.m:11-22) with hard threshold (denoiseAndAggregateGPU.m:35-39)
  std::vector<std::vector<T>> C(levels * 8);
  std::vector<int> dims(levels * 3);
  std::vector<T> U = V, tz[2], tx[2];
  int y = Ly, x = Lx, z = Lz;
  for (int lv = 0; lv < levels; ++lv) {
    dims[lv * 3] = y; dims[lv * 3 + 1] = x; dims[lv * 3 + 2] = z;
    for (int fz = 0; fz < 2; ++fz) analysis_axis(U, y, x, z, 2, bz.a[fz], tz[fz]);
    for (int fz = 0; fz < 2; ++fz)
      for (int fx = 0; fx < 2; ++fx) {
        analysis_axis(tz[fz], y, x, z / 2, 1, bxy.a[fx], tx[fx]);
        for (int fy = 0; fy < 2; ++fy) {
          int code = fy + 2 * fx + 4 * fz;
          auto& out = C[lv * 8 + code];
          analysis_axis(tx[fx], y, x / 2, z / 2, 0, bxy.a[fy], out);
          if (code) {
            T t = (T)tau[lv + levels * kDetailJ[code]];
            for (auto& v : out) v = v * (T)(std::fabs(v) > t ? 1 : 0);
          }
        }
      }
    U = C[lv * 8];
    y /= 2; x /= 2; z /= 2;
  }
  // synthesis (myWavRec3DGPUfast.m:10-40): per level y-pass, x-pass, z-pass
  std::vector<T> R = C[(levels - 1) * 8];  // coarsest approximation
  for (int lv = levels - 1; lv >= 0; --lv) {
    int oy = dims[lv * 3], ox = dims[lv * 3 + 1], oz = dims[lv * 3 + 2];
    int iy = oy / 2, ix = ox / 2, iz = oz / 2;
    auto band = [&](int code) -> const std::vector<T>& { return code ? C[lv * 8 + code] : R; };
    std::vector<T> Y[4], X[2], out;
    for (int fz = 0; fz < 2; ++fz)
      for (int fx = 0; fx < 2; ++fx)
        synthesis_axis(band(0 + 2 * fx + 4 * fz), band(1 + 2 * fx + 4 * fz), iy, ix, iz, 0, bxy, Y[fx + 2 * fz]);
    for (int fz = 0; fz < 2; ++fz) synthesis_axis(Y[0 + 2 * fz], Y[1 + 2 * fz], oy, ix, iz, 1, bxy, X[fz]);
    synthesis_axis(X[0], X[1], oy, ox, iz, 2, bz, out);
    R.swap(out);
  }
  V.swap(R);
}

// getBM3DAggWeights(3,1) (getBM3DAggWeights.m:11-19) on one group Vavg tile,
// then weight = 1/(D + eps) (denoiseAndAggregateGPU.m:75).
template <class T>
T ht_weight(const T* Vt, size_t sy, size_t sx, size_t sz, int d, int Nm) {
  auto at = [&](int r, int c, int k) { return Vt[r * sy + c * sx + k * sz]; };
  auto d3 = [](T u0, T u1, T u2, T u3) {
    T a0 = u1 - u0, a1 = u2 - u1, a2 = u3 - u2;
    T b0 = a1 - a0, b1 = a2 - a1;
    return b1 - b0;
  };
  const int dm = d - 3;
  T tx = red32<T>(d * dm * Nm, [&](int e) {
    int r = e % d, c = (e / d) % dm, k = e / (d * dm);
    return std::fabs(d3(at(r, c, k), at(r, c + 1, k), at(r, c + 2, k), at(r, c + 3, k)));
  });
  T ty = red32<T>(dm * d * Nm, [&](int e) {
    int r = e % dm, c = (e / dm) % d, k = e / (dm * d);
    return std::fabs(d3(at(r, c, k), at(r + 1, c, k), at(r + 2, c, k), at(r + 3, c, k)));
  });
  T tz = red32<T>(d * d * (Nm - 1), [&](int e) {
    int r = e % d, c = (e / d) % d, k = e / (d * d);
    return std::fabs(at(r, c, k + 1) - at(r, c, k));
  });
  T Wt = tx * T(0.25) + ty * T(0.25);
  Wt = Wt + tz;
  T eps = (T)2.220446049250313e-16;
  return T(1) / (Wt + eps);
}

// Owner-ordered aggregation shared by both steps: contributions are applied in
// the reference's loop order (ref row y, ref col x, match i), each add rounded
// in T.  value(g, k, r, c) and wval(g, r, c) give the per-pixel terms.
template <class T, class FV, class FW>
void aggregate(int M, int N, int d, int d2, int K, int stride, const uint32_t* S, const int32_t* cnt,
               FV value, FW wval, double* U, double* W) {
  const int s = stride;
  // output (M-1)s+d x (N-1)s+d; the reference (s = d) writes M*d x N*d
  const int m = (M - 1) * s + d, n = (N - 1) * s + d, h = d2 / 2, P = m + d2, Q = n + d2;
  std::vector<T> Up((size_t)P * Q, T(0)), Wp((size_t)P * Q, T(0));
  int nth = 1;
#ifdef _OPENMP
  nth = omp_get_max_threads();
#endif
#pragma omp parallel num_threads(nth)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    const int c0 = (int)((long)Q * t / nth), c1 = (int)((long)Q * (t + 1) / nth);
    for (int y = 0; y < M; ++y)
      for (int x = 0; x < N; ++x) {
        if (x * s + d2 + d - 1 <= c0 || x * s >= c1) continue;
        const int g = y + M * x;
        const int nm = cnt ? cnt[g] : K;
        for (int i = 0; i < nm; ++i) {
          int e = (int)S[(size_t)g * K + i] - 1, a = e % d2, b = e / d2;
          int R0 = y * s + a, C0 = x * s + b;
          for (int c = 0; c < d; ++c) {
            int C = C0 + c;
            if (C < c0 || C >= c1) continue;
            for (int r = 0; r < d; ++r) {
              size_t p = (size_t)(R0 + r) + (size_t)C * P;
              Up[p] = Up[p] + value(g, i, r, c);
              Wp[p] = Wp[p] + wval(g, r, c);
            }
          }
        }
      }
  }
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < m; ++r) {
      U[r + (size_t)c * m] = (double)Up[(r + h) + (size_t)(c + h) * P];
      W[r + (size_t)c * m] = (double)Wp[(r + h) + (size_t)(c + h) * P];
    }
}

template <class T>
void ht_aggregate(std::vector<T>& sum, int M, int N, int d, int d2, int K, int s, const uint32_t* S,
                  const int32_t* cnt, double* U, double* W);

// denoiseAndAggregateGPU.m:11-92 (filtType 'ht')
template <class T>
void denoise_ht(const T* Volume, int M, int N, int d, int d2, int K, const uint32_t* S,
                const int32_t* cnt, int levels, int cycleSpin, const double* tau,
                const orc_filters* f, double* U, double* W, int stride) {
  const int m = M * d, n = N * d;
  const size_t vol = (size_t)m * n * K;
  Bank1D<T> bxy = make_bank<T>(f->len_xy, f->a_lo_xy, f->a_hi_xy, f->s_lo_xy, f->s_hi_xy);
  Bank1D<T> bz = make_bank<T>(f->len_z, f->a_lo_z, f->a_hi_z, f->s_lo_z, f->s_hi_z);
  std::vector<T> sum(vol, T(0)), V(vol);
  for (int spin = 0; spin < cycleSpin; ++spin) {
    // Vrec = circshift(Volume,[spin,spin,spin])
#pragma omp parallel for collapse(2)
    for (int z = 0; z < K; ++z)
      for (int x = 0; x < n; ++x)
        for (int y = 0; y < m; ++y)
          V[y + (size_t)m * (x + (size_t)n * z)] =
              Volume[pmod(y - spin, m) + (size_t)m * (pmod(x - spin, n) + (size_t)n * pmod(z - spin, K))];
    wavelet_ht(V, m, n, K, levels, tau, bxy, bz);
    // circshift back and accumulate over spins
#pragma omp parallel for collapse(2)
    for (int z = 0; z < K; ++z)
      for (int x = 0; x < n; ++x)
        for (int y = 0; y < m; ++y) {
          size_t o = y + (size_t)m * (x + (size_t)n * z);
          T v = V[pmod(y + spin, m) + (size_t)m * (pmod(x + spin, n) + (size_t)n * pmod(z + spin, K))];
          sum[o] = spin == 0 ? v : sum[o] + v;
        }
  }
  // Vavg = max(mean(Vrec,4),0)
  const T cs = (T)cycleSpin;
#pragma omp parallel for
  for (size_t o = 0; o < vol; ++o) {
    T v = sum[o] / cs;
    sum[o] = v > T(0) ? v : T(0);
  }
  ht_aggregate<T>(sum, M, N, d, d2, K, stride, S, cnt, U, W);
}

// medfilt3(Volume,[3 3 3]) (denoiseAndAggregateGPU.m:49-52), 'symmetric'
// padding (for a one-voxel border: the edge voxel repeated).
template <class T>
void median3(const T* V, int m, int n, int K, std::vector<T>& out) {
  out.assign((size_t)m * n * K, T(0));
#pragma omp parallel for collapse(2)
  for (int z = 0; z < K; ++z)
    for (int x = 0; x < n; ++x)
      for (int y = 0; y < m; ++y) {
        T v[27];
        int q = 0;
        for (int dz = -1; dz <= 1; ++dz)
          for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy) {
              int yy = std::min(std::max(y + dy, 0), m - 1), xx = std::min(std::max(x + dx, 0), n - 1),
                  zz = std::min(std::max(z + dz, 0), K - 1);
              v[q++] = V[yy + (size_t)m * (xx + (size_t)n * zz)];
            }
        std::nth_element(v, v + 13, v + 27);
        out[y + (size_t)m * (x + (size_t)n * z)] = v[13];
      }
}

template <class T>
void denoise_median(const T* Volume, int M, int N, int d, int d2, int K, const uint32_t* S, const int32_t* cnt,
                    double* U, double* W, int stride) {
  std::vector<T> vavg;
  median3<T>(Volume, M * d, N * d, K, vavg);
  ht_aggregate<T>(vavg, M, N, d, d2, K, stride, S, cnt, U, W);
}

// Aggregation of denoiseAndAggregateGPU.m:58-92 from the filtered volume.
template <class T>
void ht_aggregate(std::vector<T>& sum, int M, int N, int d, int d2, int K, int stride, const uint32_t* S,
                  const int32_t* cnt, double* U, double* W) {
  const int m = M * d, n = N * d;
  const int G = M * N;
  std::vector<T> wg(G);
#pragma omp parallel for
  for (int g = 0; g < G; ++g) {
    int y = g % M, x = g / M;
    int nm = cnt ? cnt[g] : K;
    wg[g] = ht_weight<T>(&sum[(size_t)y * d + (size_t)x * d * m], 1, m, (size_t)m * n, d, nm);
  }
  std::vector<double> mk(d * d);
  sine_window(d, 0.1, 0.9, mk.data());
  std::vector<T> mask(d * d);
  for (int e = 0; e < d * d; ++e) mask[e] = (T)mk[e];
  auto value = [&](int g, int i, int r, int c) {
    int y = g % M, x = g / M;
    T b = sum[(size_t)(y * d + r) + (size_t)m * ((size_t)(x * d + c) + (size_t)n * i)];
    return (wg[g] * b) * mask[r + c * d];
  };
  auto wval = [&](int g, int r, int c) { return wg[g] * mask[r + c * d]; };
  aggregate<T>(M, N, d, d2, K, stride, S, cnt, value, wval, U, W);
}

// ---------------------------------------------------------------------------
// Step 2 — denoiseAndAggregateWieFast.m:23-100 (variant 0) and the legacy
// denoiseAndAggregateWie.m:16-90 (variant 1: idct inverse = T', clamp [0,1]).
// ---------------------------------------------------------------------------

// 1D Haar along the slot axis, circular — myWavDec1D.m:14-25 / myWavRec1D.m:10-25.
template <class T>
void haar_dec(T* v, int K, int levels, T cc) {
  std::vector<T> out(K), U(v, v + K);
  int cntp = 0, L = K;
  for (int lv = 0; lv < levels; ++lv) {
    std::vector<T> a(L / 2);
    for (int q = 0; q < L / 2; ++q) {
      T u0 = U[2 * q], u1 = U[pmod(2 * q - 1, L)];
      out[cntp + q] = fmaT(cc, u1, (-cc) * u0);  // Psi = [-Cc, Cc]
      a[q] = fmaT(cc, u1, cc * u0);               // Phi = [ Cc, Cc]
    }
    cntp += L / 2;
    U = a;
    L /= 2;
  }
  for (int q = 0; q < L; ++q) out[cntp + q] = U[q];
  std::copy(out.begin(), out.end(), v);
}

template <class T>
void haar_rec(T* v, int K, int levels, T cc) {
  std::vector<int> off(levels + 1);
  int c = 0;
  for (int lv = 0; lv < levels; ++lv) { off[lv] = c; c += K >> (lv + 1); }
  off[levels] = c;
  int L = K >> levels;  // approx length
  std::vector<T> R(v + off[levels], v + off[levels] + L);
  for (int lv = levels - 1; lv >= 0; --lv) {
    int Lo = 2 * L;
    std::vector<T> out(Lo);
    const T* dd = v + off[lv];
    for (int q = 0; q < L; ++q) {
      // even output 2q: detail tap k=0 (-Cc), approx tap k=0 (Cc)
      out[2 * q] = ((-cc) * dd[q]) + (cc * R[q]);
      // odd output 2q-1: detail tap k=1 (Cc), approx tap k=1 (Cc)
      out[pmod(2 * q - 1, Lo)] = (cc * dd[q]) + (cc * R[q]);
    }
    R.swap(out);
    L = Lo;
  }
  std::copy(R.begin(), R.end(), v);
}

template <class T>
void denoise_wiener(const T* V1, const T* V2, int M, int N, int d, int d2, int K,
                    const uint32_t* S, const double* sigma, int sigma_is_matrix, int variant,
                    double* U, double* W, int stride) {
  const int levels = K < 16 ? 2 : 3;
  const int dd = d * d, G = M * N;
  std::vector<double> Tm(dd), Ti(dd);
  dct_matrices(d, Tm.data(), Ti.data());
  std::vector<T> Tt(dd), Tinv(dd);
  for (int e = 0; e < dd; ++e) Tt[e] = (T)Tm[e];
  if (variant == 0) for (int e = 0; e < dd; ++e) Tinv[e] = (T)Ti[e];
  else for (int r = 0; r < d; ++r) for (int c = 0; c < d; ++c) Tinv[r + c * d] = (T)Tm[c + r * d];
  std::vector<T> s2(dd);
  for (int e = 0; e < dd; ++e) {
    double s = sigma_is_matrix ? sigma[e] : sigma[0];
    s2[e] = (T)(s * s);
  }
  const T cc = (T)(std::sqrt(2.0) / 2.0);
  std::vector<double> wk(dd);
  sine_window(d, 0.2, 0.8, wk.data());
  std::vector<T> wf(dd);
  for (int e = 0; e < dd; ++e) wf[e] = (T)wk[e];
  const size_t gsz = (size_t)dd * K;
  std::vector<T> out((size_t)G * gsz), n2(G);
#pragma omp parallel
  {
    std::vector<T> A(gsz), B(gsz), P(gsz), filt(gsz);
    // Y = Tl * X * Tr' applied per slot page (pagemtimes), serial fma chains
    auto fwd = [&](const T* X, T* Y) {
      for (int k = 0; k < K; ++k) {
        const T* x = X + (size_t)k * dd;
        T* p = &P[(size_t)k * dd];
        for (int n = 0; n < d; ++n)
          for (int r = 0; r < d; ++r) {
            T acc = T(0);
            for (int j = 0; j < d; ++j) acc = fmaT(Tt[r + j * d], x[j + n * d], acc);
            p[r + n * d] = acc;
          }
        T* y = Y + (size_t)k * dd;
        for (int l = 0; l < d; ++l)
          for (int r = 0; r < d; ++r) {
            T acc = T(0);
            for (int n = 0; n < d; ++n) acc = fmaT(p[r + n * d], Tt[l + n * d], acc);
            y[r + l * d] = acc;
          }
      }
    };
#pragma omp for schedule(static)
    for (int g = 0; g < G; ++g) {
      fwd(V1 + (size_t)g * gsz, A.data());
      fwd(V2 + (size_t)g * gsz, B.data());
      std::vector<T> col(K);
      for (int e = 0; e < dd; ++e) {
        for (int k = 0; k < K; ++k) col[k] = A[e + (size_t)k * dd];
        haar_dec(col.data(), K, levels, cc);
        for (int k = 0; k < K; ++k) A[e + (size_t)k * dd] = col[k];
        for (int k = 0; k < K; ++k) col[k] = B[e + (size_t)k * dd];
        haar_dec(col.data(), K, levels, cc);
        for (int k = 0; k < K; ++k) B[e + (size_t)k * dd] = col[k];
      }
      // filt = |V1|^2 ./ (|V1|^2 + sigma^2); filt(1,1,15:end) = 1  (:49-50)
      for (int k = 0; k < K; ++k)
        for (int e = 0; e < dd; ++e) {
          size_t o = e + (size_t)k * dd;
          T p = A[o] * A[o];
          T f = p / (p + s2[e]);
          if (e == 0 && k >= 14) f = T(1);
          filt[o] = f;
          B[o] = B[o] * f;
        }
      for (int e = 0; e < dd; ++e) {
        for (int k = 0; k < K; ++k) col[k] = B[e + (size_t)k * dd];
        haar_rec(col.data(), K, levels, cc);
        for (int k = 0; k < K; ++k) B[e + (size_t)k * dd] = col[k];
      }
      // inverse: X = Tinv * (Y * Tinv')  (:60-63), clamp (:64)
      T* og = &out[(size_t)g * gsz];
      for (int k = 0; k < K; ++k) {
        const T* y = &B[(size_t)k * dd];
        T* p = &P[(size_t)k * dd];
        for (int l = 0; l < d; ++l)
          for (int r = 0; r < d; ++r) {
            T acc = T(0);
            for (int n = 0; n < d; ++n) acc = fmaT(y[r + n * d], Tinv[l + n * d], acc);
            p[r + l * d] = acc;
          }
        for (int l = 0; l < d; ++l)
          for (int r = 0; r < d; ++r) {
            T acc = T(0);
            for (int j = 0; j < d; ++j) acc = fmaT(Tinv[r + j * d], p[j + l * d], acc);
            T v = acc > T(0) ? acc : T(0);
            if (variant == 1 && v > T(1)) v = T(1);
            og[(size_t)k * dd + r + l * d] = v;
          }
      }
      // weight = w / norm(col(filt))^2   (:81)
      T s = red32<T>((int)gsz, [&](int e) { return filt[e] * filt[e]; });
      T nr = std::sqrt(s);
      n2[g] = nr * nr;
    }
  }
  auto value = [&](int g, int i, int r, int c) {
    T wgt = wf[r + c * d] / n2[g];
    return wgt * out[(size_t)g * gsz + (size_t)i * dd + r + c * d];
  };
  auto wval = [&](int g, int r, int c) { return wf[r + c * d] / n2[g]; };
  aggregate<T>(M, N, d, d2, K, stride, S, nullptr, value, wval, U, W);
}

// getTau.m:9-51
void get_tau(int levels, int mode, double* tau) {
  for (int j = 0; j < 7; ++j)
    for (int i = 0; i < levels; ++i) {
      double v = 0;
      double base = 3.3 - 0.3 * i;
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

// myMirrorPadImage.m:3-8
void mirror_pad(const double* I, int m, int n, double* O, int Mp, int Np) {
  for (int c = 0; c < Np; ++c)
    for (int r = 0; r < Mp; ++r) {
      int sr = r < m ? r : m - 1 - (r - m);
      int sc = c < n ? c : n - 1 - (c - n);
      O[r + (size_t)c * Mp] = I[sr + (size_t)sc * m];
    }
}

void circshift2(const double* I, int m, int n, int s, double* O) {
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < m; ++r) O[r + (size_t)c * m] = I[pmod(r - s, m) + (size_t)pmod(c - s, n) * m];
}

template <class T>
std::vector<T> to_T(const double* I, size_t n) {
  std::vector<T> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = (T)I[i];
  return v;
}

void bior_filters(orc_filters* f) {
  std::memset(f, 0, sizeof(*f));
  const double Ca = 0.016572815184060, Cb = 0.121533978016438, Cc = std::sqrt(2.0) / 2;
  const double lo[10] = {Ca, -Ca, -Cb, Cb, Cc, Cc, Cb, -Cb, -Ca, Ca};
  const double shi[10] = {-Ca, -Ca, Cb, Cb, -Cc, Cc, -Cb, -Cb, Ca, Ca};
  f->len_xy = 10;
  for (int k = 0; k < 10; ++k) {
    f->a_lo_xy[k] = lo[k];
    f->s_hi_xy[k] = shi[k];
  }
  f->a_hi_xy[4] = -Cc; f->a_hi_xy[5] = Cc;
  f->s_lo_xy[4] = Cc; f->s_lo_xy[5] = Cc;
  f->len_z = 2;
  f->a_lo_z[0] = Cc; f->a_lo_z[1] = Cc; f->a_hi_z[0] = -Cc; f->a_hi_z[1] = Cc;
  f->s_lo_z[0] = Cc; f->s_lo_z[1] = Cc; f->s_hi_z[0] = -Cc; f->s_hi_z[1] = Cc;
}

// 3D Haar bank: the two-tap Haar pair on the spatial axes as well as the slot axis.
void haar_filters(orc_filters* f) {
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

// GBM3D.m:15-83
// tau_in (levels x 7) and sigwie_in (dw x dw) replace sigma * getTau and the
// scalar Wiener sigma on the coloured-noise path (GBM3D.m:30-36); sigma is then
// mean(sqrt(sigmaPSD)) as the matchers use it (matchBlocksCPU.m:21).
template <class T>
void gbm3d(const double* I0, int m0, int n0, double sigma, const orc_opts* o, double* Uout, double* U1out,
           const double* tau_in, const double* sigwie_in);

template <class T>
void gbm3d(const double* I0, int m0, int n0, double sigma, const orc_opts* o, double* Uout, double* U1out) {
  gbm3d<T>(I0, m0, n0, sigma, o, Uout, U1out, nullptr, nullptr);
}

template <class T>
void gbm3d(const double* I0, int m0, int n0, double sigma, const orc_opts* o, double* Uout, double* U1out,
           const double* tau_in, const double* sigwie_in) {
  const int d = o->blockSize, dw = o->blockSizeWie, d2 = o->matchSize, K = o->numMax;
  const int st1 = o->refStride > 0 ? o->refStride : d, st2 = o->refStrideWie > 0 ? o->refStrideWie : dw;
  // GBM3D.m:21-25 pads to a multiple of blockSize; with other strides, to the
  // smallest size whose references of both steps end exactly at the border
  auto padded = [&](int L) {
    if (st1 == d && (!o->Wiener || (st2 == dw && d % dw == 0))) return (L + d - 1) / d * d;
    int p = std::max(L, std::max(d, dw));
    while ((p - d) % st1 != 0 || (o->Wiener && (p - dw) % st2 != 0)) ++p;
    return p;
  };
  const int Mp = padded(m0), Np = padded(n0);
  const size_t px = (size_t)Mp * Np;
  std::vector<double> I(px);
  mirror_pad(I0, m0, n0, I.data(), Mp, Np);
  std::vector<double> tau(o->levels * 7);
  get_tau(o->levels, o->tauMode, tau.data());
  for (auto& t : tau) t *= sigma;
  if (tau_in) std::copy(tau_in, tau_in + o->levels * 7, tau.begin());
  orc_filters f;
  if (o->wavelet == 1) haar_filters(&f);
  else bior_filters(&f);
  const int nS = o->nSpins, nW = o->nSpinsWie, nslice = std::max(nS, nW);
  std::vector<double> Us((size_t)nslice * px, 0.0), Ws((size_t)nslice * px, 0.0), U1s((size_t)nS * px, 0.0);
  std::vector<double> sh(px), u(px), w(px);
  const double tol = 0.005 * sigma * sigma * d * d;
  // step 1
  for (int ii = 0; ii < nS; ++ii) {
    int s = o->spins[ii];
    circshift2(I.data(), Mp, Np, s, sh.data());
    std::vector<T> It = to_T<T>(sh.data(), px);
    int M = (Mp - d) / st1 + 1, N = (Np - d) / st1 + 1;
    std::vector<uint32_t> S((size_t)M * N * K);
    std::vector<int32_t> cnt(M * N);
    std::vector<T> Vol(st1 == d ? px * K : (size_t)M * d * N * d * K);
    MatchOut<T> mo{S.data(), cnt.data(), Vol.data(), nullptr, nullptr};
    match_blocks<T>(It.data(), nullptr, Mp, Np, d, d2, K, o->numMin, tol, o->numMax != o->numMin, mo, st1);
    if (o->filtType == 1)
      denoise_median<T>(Vol.data(), M, N, d, d2, K, S.data(), cnt.data(), u.data(), w.data(), st1);
    else
      denoise_ht<T>(Vol.data(), M, N, d, d2, K, S.data(), cnt.data(), o->levels, o->cycleSpin,
                    tau.data(), &f, u.data(), w.data(), st1);
    circshift2(u.data(), Mp, Np, -s, &U1s[ii * px]);
    circshift2(w.data(), Mp, Np, -s, &Ws[ii * px]);
  }
  std::vector<double> U1(px);
  for (size_t p = 0; p < px; ++p) {
    double a = 0, b = 0;
    for (int ii = 0; ii < nS; ++ii) { a += U1s[ii * px + p]; b += Ws[ii * px + p]; }
    U1[p] = a / b;
  }
  if (U1out)
    for (int c = 0; c < n0; ++c)
      for (int r = 0; r < m0; ++r) U1out[r + (size_t)c * m0] = U1[r + (size_t)c * Mp];
  if (!o->Wiener) {
    for (int c = 0; c < n0; ++c)
      for (int r = 0; r < m0; ++r) Uout[r + (size_t)c * m0] = U1[r + (size_t)c * Mp];
    return;
  }
  if (!o->staleWeights)
    std::fill(Ws.begin(), Ws.end(), 0.0);
  // step 2
  std::vector<double> sh2(px);
  for (int ii = 0; ii < nW; ++ii) {
    int s = o->spinsWie[ii];
    circshift2(U1.data(), Mp, Np, s, sh.data());
    circshift2(I.data(), Mp, Np, s, sh2.data());
    std::vector<T> Ip = to_T<T>(sh.data(), px), In = to_T<T>(sh2.data(), px);
    int M = (Mp - dw) / st2 + 1, N = (Np - dw) / st2 + 1;
    std::vector<uint32_t> S((size_t)M * N * K);
    std::vector<T> V1((size_t)dw * dw * K * M * N), V2(V1.size());
    MatchOut<T> mo{S.data(), nullptr, nullptr, V1.data(), V2.data()};
    match_blocks<T>(Ip.data(), In.data(), Mp, Np, dw, d2, K, K, 0.0, false, mo, st2);
    double sg = sigma;
    denoise_wiener<T>(V1.data(), V2.data(), M, N, dw, d2, K, S.data(), sigwie_in ? sigwie_in : &sg,
                      sigwie_in ? 1 : 0, 0, u.data(), w.data(), st2);
    circshift2(u.data(), Mp, Np, -s, &Us[ii * px]);
    circshift2(w.data(), Mp, Np, -s, &Ws[ii * px]);
  }
  const int nU = std::max(nS, nW);
  for (int c = 0; c < n0; ++c)
    for (int r = 0; r < m0; ++r) {
      size_t p = r + (size_t)c * Mp;
      // slices nW..nS-1 of W still hold step-1 weights when staleWeights is
      // set; otherwise they were cleared above.  Slices of U past nW are zero.
      double a = 0, b = 0;
      for (int ii = 0; ii < nU; ++ii) {
        a += Us[ii * px + p];
        b += Ws[ii * px + p];
      }
      Uout[r + (size_t)c * m0] = a / b;
    }
}


// ---------------------------------------------------------------------------
// Video — VBM3D.m:20-63, matchBlocksV.m:21-116 (top-K branch),
// denoiseAndAggregateV.m:11-89
// ---------------------------------------------------------------------------

// Block matching over a window of F frames (F odd): references tile the
// centre frame at stride d; candidates are the d x d offsets of the 2d x 2d
// window of every frame (search image per frame built like matchBlocksCPU's
// with d2 = d).  Ranked by (exact SSD, index a + b d + c d^2) like mink;
// S(1) is forced to d^2 F/2 + d/2 + 1.  Volume: image-shaped m x n x K.
template <class T>
void match_video(const T* I, int m, int n, int F, int d, int K, uint32_t* S, T* Volume) {
  const int h = d / 2, M = m / d, N = n / d, ref = (F - 1) / 2;
  const size_t mn = (size_t)m * n;
  auto pix = [&](int R, int C, int f) { return I[pad_index(R, m, h) + (size_t)m * pad_index(C, n, h) + mn * f]; };
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) {
      const int g = i + M * j, nc = d * d * F;
      std::vector<T> x((size_t)d * d);
      for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) x[r * d + c] = pix(i * d + h + r, j * d + h + c, ref);
      std::vector<std::pair<T, uint32_t>> key(nc);
      for (int f = 0; f < F; ++f)
        for (int b = 0; b < d; ++b)
          for (int a = 0; a < d; ++a) {
            T acc = T(0);
            for (int r = 0; r < d; ++r)
              for (int c = 0; c < d; ++c) {
                const T t = x[r * d + c] - pix(i * d + a + r, j * d + b + c, f);
                acc = fmaT(t, t, acc);
              }
            const uint32_t idx = (uint32_t)(a + b * d + f * d * d);
            key[idx] = {acc, idx};
          }
      std::stable_sort(key.begin(), key.end(),
                       [](const std::pair<T, uint32_t>& u, const std::pair<T, uint32_t>& v) { return u.first < v.first; });
      for (int k = 0; k < K; ++k) S[(size_t)g * K + k] = key[k].second + 1;
      S[(size_t)g * K] = (uint32_t)(d * d * F / 2 + d / 2 + 1);  // matchBlocksV.m:103
      for (int k = 0; k < K; ++k) {
        const int e = (int)S[(size_t)g * K + k] - 1;
        const int a = e % d, b = (e / d) % d, f = e / (d * d);
        for (int c = 0; c < d; ++c)
          for (int r = 0; r < d; ++r)
            Volume[(size_t)(i * d + r) + (size_t)m * (j * d + c) + mn * k] = pix(i * d + a + r, j * d + b + c, f);
      }
    }
}

// denoiseAndAggregateV.m:24-89: cycle-spun 3D wavelet hard threshold of the
// volume, Vavg = min(max(mean, 0), 1), weight 1/TV(blocks) (the same
// getBM3DAggWeights(3,1) measure as step 1), and aggregation without a window:
// block k of reference (y, x) lands in frame c at rows a + y d - d/2, columns
// b + x d - d/2 (discarded when it starts before row or column 0); sums are
// double, each term fl(w * block).  U, Wt: m x n x F.
template <class T>
void denoise_video(const T* Volume, int M, int N, int d, int F, int K, const uint32_t* S, int levels, int cycleSpin,
                   const double* tau, const orc_filters* f, double* U, double* Wt) {
  const int m = M * d, n = N * d, h = d / 2;
  const size_t vol = (size_t)m * n * K;
  Bank1D<T> bxy = make_bank<T>(f->len_xy, f->a_lo_xy, f->a_hi_xy, f->s_lo_xy, f->s_hi_xy);
  Bank1D<T> bz = make_bank<T>(f->len_z, f->a_lo_z, f->a_hi_z, f->s_lo_z, f->s_hi_z);
  std::vector<T> sum(vol, T(0)), V(vol);
  for (int spin = 0; spin < cycleSpin; ++spin) {
#pragma omp parallel for collapse(2)
    for (int z = 0; z < K; ++z)
      for (int x = 0; x < n; ++x)
        for (int y = 0; y < m; ++y)
          V[y + (size_t)m * (x + (size_t)n * z)] =
              Volume[pmod(y - spin, m) + (size_t)m * (pmod(x - spin, n) + (size_t)n * pmod(z - spin, K))];
    wavelet_ht(V, m, n, K, levels, tau, bxy, bz);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < K; ++z)
      for (int x = 0; x < n; ++x)
        for (int y = 0; y < m; ++y) {
          size_t o = y + (size_t)m * (x + (size_t)n * z);
          T v = V[pmod(y + spin, m) + (size_t)m * (pmod(x + spin, n) + (size_t)n * pmod(z + spin, K))];
          sum[o] = spin == 0 ? v : sum[o] + v;
        }
  }
  const T cs = (T)cycleSpin;
#pragma omp parallel for
  for (size_t o = 0; o < vol; ++o) {
    T v = sum[o] / cs;
    v = v > T(0) ? v : T(0);
    sum[o] = v < T(1) ? v : T(1);
  }
  const size_t px = (size_t)m * n;
  std::vector<double> Up((size_t)(m + d) * (n + d) * F, 0.0), Wp(Up.size(), 0.0);
  const int P = m + d, Q = n + d;
  for (int y = 0; y < M; ++y)
    for (int x = 0; x < N; ++x) {
      const int g = y + M * x;
      const T w = ht_weight<T>(&sum[(size_t)y * d + (size_t)x * d * m], 1, m, px, d, K);
      for (int k = 0; k < K; ++k) {
        const int e = (int)S[(size_t)g * K + k] - 1;
        const int a = e % d, b = (e / d) % d, fr = e / (d * d);
        const int R0 = a + y * d - h, C0 = b + x * d - h;
        if (R0 < 0 || C0 < 0) continue;
        for (int c = 0; c < d; ++c)
          for (int r = 0; r < d; ++r) {
            const T blk = sum[(size_t)(y * d + r) + (size_t)m * (x * d + c) + px * k];
            const size_t o = (size_t)(R0 + r) + (size_t)P * ((C0 + c) + (size_t)Q * fr);
            Up[o] += (double)(w * blk);
            Wp[o] += (double)w;
          }
      }
    }
  for (int fr = 0; fr < F; ++fr)
    for (int c = 0; c < n; ++c)
      for (int r = 0; r < m; ++r) {
        U[r + (size_t)m * (c + (size_t)n * fr)] = Up[r + (size_t)P * (c + (size_t)Q * fr)];
        Wt[r + (size_t)m * (c + (size_t)n * fr)] = Wp[r + (size_t)P * (c + (size_t)Q * fr)];
      }
}

// VBM3D.m:20-63: frames mirror-padded to multiples of d; for every match spin
// and every centre frame jj with a full window of nF frames, the circshifted
// window is matched and denoised, and U / weights are added (in single, as
// the reference's single Y and nn) into the window's frames; Y / nn is shifted
// back, and the output is the mean over spins of frames (nF-1)/2 ..
// Kf-1-(nF-1)/2, cropped.  out: m0 x n0 x (Kf - nF + 1).
template <class T>
void vbm3d(const double* I0, int m0, int n0, int Kf, double sigma, int d, int K, int levels, int cycleSpin,
           int tauMode, const int* spins, int nS, int nF, const orc_filters* f, double* out) {
  const int Mp = (m0 + d - 1) / d * d, Np = (n0 + d - 1) / d * d, M = Mp / d, N = Np / d;
  const size_t px = (size_t)Mp * Np, px0 = (size_t)m0 * n0;
  std::vector<double> I2(px * Kf);
  for (int k = 0; k < Kf; ++k) mirror_pad(I0 + px0 * k, m0, n0, &I2[px * k], Mp, Np);
  std::vector<double> tau(levels * 7);
  get_tau(levels, tauMode, tau.data());
  for (auto& t : tau) t *= sigma;
  const int hw = (nF - 1) / 2, nOut = Kf - nF + 1;
  std::vector<double> acc((size_t)px0 * nOut, 0.0);
  std::vector<float> Y(px * Kf), nn(px * Kf);
  std::vector<double> sh(px), U(px * nF), Wt(px * nF);
  for (int ii = 0; ii < nS; ++ii) {
    const int s = spins[ii];
    std::fill(Y.begin(), Y.end(), 0.f);
    std::fill(nn.begin(), nn.end(), 0.f);
    for (int jj = hw; jj < Kf - hw; ++jj) {
      std::vector<T> I3(px * nF);
      for (int q = 0; q < nF; ++q) {
        circshift2(&I2[px * (jj - hw + q)], Mp, Np, s, sh.data());
        for (size_t p = 0; p < px; ++p) I3[px * q + p] = (T)sh[p];
      }
      std::vector<uint32_t> S((size_t)M * N * K);
      std::vector<T> Vol(px * K);
      match_video<T>(I3.data(), Mp, Np, nF, d, K, S.data(), Vol.data());
      denoise_video<T>(Vol.data(), M, N, d, nF, K, S.data(), levels, cycleSpin, tau.data(), f, U.data(), Wt.data());
      for (int q = 0; q < nF; ++q)
        for (size_t p = 0; p < px; ++p) {
          const size_t o = px * (jj - hw + q) + p;
          Y[o] = (float)((double)Y[o] + U[px * q + p]);
          nn[o] = (float)((double)nn[o] + Wt[px * q + p]);
        }
    }
    for (int k = hw; k < Kf - hw; ++k)
      for (int c = 0; c < n0; ++c)
        for (int r = 0; r < m0; ++r) {
          // circshift(Y ./ nn, [-s, -s, 0]): output (r, c) reads (r + s, c + s)
          const size_t o = px * k + pmod(r + s, Mp) + (size_t)Mp * pmod(c + s, Np);
          acc[px0 * (k - hw) + r + (size_t)m0 * c] += (double)(Y[o] / nn[o]);
        }
  }
  for (size_t o = 0; o < acc.size(); ++o) out[o] = (double)(float)(acc[o] / nS);
}

// ---------------------------------------------------------------------------
// Global matcher — matchBlocksGPU.m:19-91 (A12)
// ---------------------------------------------------------------------------

// Symlet-4 decomposition filters (published values; Lo_d / Hi_d of the sym4
// bank that getWaveFilters2D('sym',4) loads, matchBlocksGPU.m:36).
const double kSym4Lo[8] = {-0.07576571478927333, -0.02963552764599851, 0.49761866763201545, 0.8037387518059161,
                           0.29785779560527736, -0.09921954357684722, -0.012603967262037833, 0.0322231006040427};
const double kSym4Hi[8] = {-0.0322231006040427, -0.012603967262037833, 0.09921954357684722, 0.29785779560527736,
                           -0.8037387518059161, 0.49761866763201545, 0.02963552764599851, -0.07576571478927333};

// One 2D hard-threshold denoise: myWavDec2DFFT (x-pass then y-pass per level),
// threshold |C| > tau on the three detail bands, myWavRec2DGPUfast (y-pass
// then x-pass per level; synthesis with the same filters, by correlation).
template <class T>
void wavelet2d_ht(std::vector<T>& U, int Ly, int Lx, int levels, T tau) {
  Bank1D<T> b = make_bank<T>(8, kSym4Lo, kSym4Hi, kSym4Lo, kSym4Hi);
  std::vector<std::vector<T>> C(levels * 4);
  std::vector<int> dims(levels * 2);
  std::vector<T> A = U, tx[2];
  int y = Ly, x = Lx;
  for (int lv = 0; lv < levels; ++lv) {
    dims[lv * 2] = y; dims[lv * 2 + 1] = x;
    for (int fx = 0; fx < 2; ++fx) {
      analysis_axis(A, y, x, 1, 1, b.a[fx], tx[fx]);
      for (int fy = 0; fy < 2; ++fy) {
        int code = fy + 2 * fx;
        auto& out = C[lv * 4 + code];
        analysis_axis(tx[fx], y, x / 2, 1, 0, b.a[fy], out);
        if (code)
          for (auto& v : out) v = v * (T)(std::fabs(v) > tau ? 1 : 0);
      }
    }
    A = C[lv * 4];
    y /= 2; x /= 2;
  }
  std::vector<T> R = C[(levels - 1) * 4];
  for (int lv = levels - 1; lv >= 0; --lv) {
    int oy = dims[lv * 2], ox = dims[lv * 2 + 1], iy = oy / 2, ix = ox / 2;
    auto band = [&](int code) -> const std::vector<T>& { return code ? C[lv * 4 + code] : R; };
    std::vector<T> Y[2], out;
    for (int fx = 0; fx < 2; ++fx) synthesis_axis(band(0 + 2 * fx), band(1 + 2 * fx), iy, ix, 1, 0, b, Y[fx]);
    synthesis_axis(Y[0], Y[1], oy, ix, 1, 1, b, out);
    R.swap(out);
  }
  U.swap(R);
}

// matchBlocksGPU.m:34-50: average of 5 shifted hard-threshold denoises.
template <class T>
void sym4_prefilter(std::vector<T>& I, int m, int n, double sigma) {
  const T tau = (T)(2 * sigma);
  std::vector<T> avg(I.size(), T(0)), sh(I.size());
  const T five = (T)5;
  for (int k = 0; k < 5; ++k) {
    for (int c = 0; c < n; ++c)
      for (int r = 0; r < m; ++r) sh[r + (size_t)c * m] = I[pmod(r - k, m) + (size_t)pmod(c - k, n) * m];
    wavelet2d_ht(sh, m, n, 3, tau);
    for (int c = 0; c < n; ++c)
      for (int r = 0; r < m; ++r) {
        size_t o = r + (size_t)c * m;
        avg[o] = avg[o] + sh[pmod(r + k, m) + (size_t)pmod(c + k, n) * m] / five;
      }
  }
  I.swap(avg);
}

// Search over every circular block position of the image: distances are exact
// SSDs (row-major, fma(t,t,acc)) ranked with mink's stable order; indices are
// 1-based linear positions in the m x n image; no slot-1 override.
template <class T>
void match_global(const std::vector<T>& I, int m, int n, int d, int K, int numMin, double tol, bool tol_branch,
                  uint32_t* S, int32_t* cnt) {
  const int M = m / d, N = n / d;
  const size_t P = (size_t)m * n;
#pragma omp parallel
  {
    std::vector<T> ssd(P);
    std::vector<std::pair<T, int>> keys(P);
#pragma omp for schedule(dynamic) collapse(2)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < M; ++i) {
        std::fill(ssd.begin(), ssd.end(), T(0));
        for (int r = 0; r < d; ++r)
          for (int c = 0; c < d; ++c) {
            const T xv = I[(i * d + r) + (size_t)(j * d + c) * m];
            for (int pc = 0; pc < n; ++pc) {
              const T* col = &I[(size_t)((pc + c) % n) * m];
              T* acc = &ssd[(size_t)pc * m];
              for (int pr = 0; pr < m; ++pr) {
                T t = xv - col[(pr + r) % m];
                acc[pr] = fmaT(t, t, acc[pr]);
              }
            }
          }
        for (size_t e = 0; e < P; ++e) keys[e] = {ssd[e], (int)e};
        auto less = [](const std::pair<T, int>& x, const std::pair<T, int>& y) {
          return x.first < y.first || (x.first == y.first && x.second < y.second);
        };
        std::vector<int> sel;
        if (!tol_branch) {
          std::partial_sort(keys.begin(), keys.begin() + K, keys.end(), less);
          for (int k = 0; k < K; ++k) sel.push_back(keys[k].second);
        } else {
          T nR = T(0);
          for (int c = 0; c < d; ++c)
            for (int r = 0; r < d; ++r) {
              const T xv = I[(i * d + r) + (size_t)(j * d + c) * m];
              nR = fmaT(xv, xv, nR);
            }
          for (size_t e = 0; e < P; ++e)
            if (ssd[e] / nR < (T)tol) sel.push_back((int)e);
          int want = -1;
          if ((int)sel.size() > K) want = K;
          else if ((int)sel.size() < numMin) want = numMin;
          if (want > 0) {
            std::partial_sort(keys.begin(), keys.begin() + want, keys.end(), less);
            sel.clear();
            for (int k = 0; k < want; ++k) sel.push_back(keys[k].second);
          }
        }
        const int g = i + M * j;
        for (int k = 0; k < K; ++k) S[(size_t)g * K + k] = k < (int)sel.size() ? (uint32_t)(sel[k] + 1) : 0u;
        if (cnt) cnt[g] = (int)sel.size();
      }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// C entry points for oracle/oracle.py (prec: 32 = FP32 GPU order, 64 = FP64)
// ---------------------------------------------------------------------------
extern "C" {

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

void orc_bior_filters(orc_filters* f) { bior_filters(f); }
void orc_get_tau(int levels, int mode, double* tau) { get_tau(levels, mode, tau); }
void orc_dct_matrices(int d, double* T, double* Tinv) { dct_matrices(d, T, Tinv); }
void orc_sine_window(int d, double lo, double hi, double* w) { sine_window(d, lo, hi, w); }
void orc_mirror_pad(const double* I, int m, int n, double* O, int M, int N) { mirror_pad(I, m, n, O, M, N); }

// [S,Volume] = matchBlocksCPU(I,sigma,opts); Volume is float (prec 32) or double.
int orc_match_blocks(int prec, const double* I, int m, int n, double sigma, int d, int d2,
                     int numMax, int numMin, uint32_t* S, int32_t* cnt, void* Volume, int stride) {
  const double tol = 0.005 * sigma * sigma * d * d;
  const size_t px = (size_t)m * n;
  if (prec == 32) {
    auto It = to_T<float>(I, px);
    MatchOut<float> o{S, cnt, (float*)Volume, nullptr, nullptr};
    match_blocks<float>(It.data(), nullptr, m, n, d, d2, numMax, numMin, tol, numMax != numMin, o, stride);
  } else {
    MatchOut<double> o{S, cnt, (double*)Volume, nullptr, nullptr};
    match_blocks<double>(I, nullptr, m, n, d, d2, numMax, numMin, tol, numMax != numMin, o, stride);
  }
  return 0;
}

// [S,V1,V2] = matchBlocksWie(I,In,sigma,opts)
int orc_match_blocks_wie(int prec, const double* I, const double* In, int m, int n, int d, int d2,
                         int K, uint32_t* S, void* V1, void* V2, int stride) {
  const size_t px = (size_t)m * n;
  if (prec == 32) {
    auto It = to_T<float>(I, px), Int = to_T<float>(In, px);
    MatchOut<float> o{S, nullptr, nullptr, (float*)V1, (float*)V2};
    match_blocks<float>(It.data(), Int.data(), m, n, d, d2, K, K, 0.0, false, o, stride);
  } else {
    MatchOut<double> o{S, nullptr, nullptr, (double*)V1, (double*)V2};
    match_blocks<double>(I, In, m, n, d, d2, K, K, 0.0, false, o, stride);
  }
  return 0;
}

// [U,W] = denoiseAndAggregateGPU(Volume,S,tau,Psi,Psi2,opts)
int orc_denoise_ht(int prec, const void* Volume, int M, int N, int d, int d2, int K,
                   const uint32_t* S, const int32_t* cnt, int levels, int cycleSpin,
                   const double* tau, const orc_filters* f, double* U, double* W, int stride) {
  if (prec == 32)
    denoise_ht<float>((const float*)Volume, M, N, d, d2, K, S, cnt, levels, cycleSpin, tau, f, U, W, stride);
  else
    denoise_ht<double>((const double*)Volume, M, N, d, d2, K, S, cnt, levels, cycleSpin, tau, f, U, W, stride);
  return 0;
}

// [U,W] = denoiseAndAggregateWieFast(V1,V2,S,sigma,opts) (variant 0) or
// denoiseAndAggregateWie (variant 1)
int orc_denoise_wiener(int prec, const void* V1, const void* V2, int M, int N, int d, int d2, int K,
                       const uint32_t* S, const double* sigma, int sigma_is_matrix, int variant,
                       double* U, double* W, int stride) {
  if (prec == 32)
    denoise_wiener<float>((const float*)V1, (const float*)V2, M, N, d, d2, K, S, sigma,
                          sigma_is_matrix, variant, U, W, stride);
  else
    denoise_wiener<double>((const double*)V1, (const double*)V2, M, N, d, d2, K, S, sigma,
                           sigma_is_matrix, variant, U, W, stride);
  return 0;
}

// [U,W] = denoiseAndAggregateGPU(Volume,S,tau,Psi,Psi2,opts) with filtType 'median'
int orc_denoise_median(int prec, const void* Volume, int M, int N, int d, int d2, int K, const uint32_t* S,
                       const int32_t* cnt, double* U, double* W, int stride) {
  if (prec == 32) denoise_median<float>((const float*)Volume, M, N, d, d2, K, S, cnt, U, W, stride);
  else denoise_median<double>((const double*)Volume, M, N, d, d2, K, S, cnt, U, W, stride);
  return 0;
}

// medfilt3(V,[3 3 3]) alone, for unit tests.
int orc_medfilt3(int prec, const void* V, int m, int n, int K, void* out) {
  const size_t N = (size_t)m * n * K;
  if (prec == 32) {
    std::vector<float> o;
    median3<float>((const float*)V, m, n, K, o);
    std::memcpy(out, o.data(), N * sizeof(float));
  } else {
    std::vector<double> o;
    median3<double>((const double*)V, m, n, K, o);
    std::memcpy(out, o.data(), N * sizeof(double));
  }
  return 0;
}

// One level of the 3D analysis + hard threshold, exposed for unit tests:
// returns the 8 bands (code order fy + 2fx + 4fz) concatenated.
int orc_wavelet_roundtrip(int prec, const void* V, int Ly, int Lx, int Lz, int levels,
                          const double* tau, const orc_filters* f, void* out) {
  size_t nv = (size_t)Ly * Lx * Lz;
  if (prec == 32) {
    auto bxy = make_bank<float>(f->len_xy, f->a_lo_xy, f->a_hi_xy, f->s_lo_xy, f->s_hi_xy);
    auto bz = make_bank<float>(f->len_z, f->a_lo_z, f->a_hi_z, f->s_lo_z, f->s_hi_z);
    std::vector<float> v((const float*)V, (const float*)V + nv);
    wavelet_ht(v, Ly, Lx, Lz, levels, tau, bxy, bz);
    std::memcpy(out, v.data(), nv * sizeof(float));
  } else {
    auto bxy = make_bank<double>(f->len_xy, f->a_lo_xy, f->a_hi_xy, f->s_lo_xy, f->s_hi_xy);
    auto bz = make_bank<double>(f->len_z, f->a_lo_z, f->a_hi_z, f->s_lo_z, f->s_hi_z);
    std::vector<double> v((const double*)V, (const double*)V + nv);
    wavelet_ht(v, Ly, Lx, Lz, levels, tau, bxy, bz);
    std::memcpy(out, v.data(), nv * sizeof(double));
  }
  return 0;
}

// S = matchBlocksGPU(I,sigma,opts); prefiltered (may be null) receives the
// image the search ran on.
int orc_match_blocks_global(int prec, const double* I, int m, int n, double sigma, int d, int numMax,
                            int numMin, uint32_t* S, int32_t* cnt, double* prefiltered) {
  const double tol = 0.005 * sigma * sigma * d * d;
  const size_t px = (size_t)m * n;
  if (prec == 32) {
    auto It = to_T<float>(I, px);
    if (sigma > 30.0 / 255.0) sym4_prefilter<float>(It, m, n, sigma);
    if (prefiltered) for (size_t i = 0; i < px; ++i) prefiltered[i] = It[i];
    match_global<float>(It, m, n, d, numMax, numMin, tol, numMax != numMin, S, cnt);
  } else {
    std::vector<double> It(I, I + px);
    if (sigma > 30.0 / 255.0) sym4_prefilter<double>(It, m, n, sigma);
    if (prefiltered) for (size_t i = 0; i < px; ++i) prefiltered[i] = It[i];
    match_global<double>(It, m, n, d, numMax, numMin, tol, numMax != numMin, S, cnt);
  }
  return 0;
}

// U = GBM3D(I,sigma,opts); U1out (may be null) receives out.U1.
int orc_gbm3d(int prec, const double* I, int m, int n, double sigma, const orc_opts* o,
              double* U, double* U1) {
  const int st1 = o->refStride > 0 ? o->refStride : o->blockSize;
  const int st2 = o->refStrideWie > 0 ? o->refStrideWie : o->blockSizeWie;
  // no padded size lets both reference grids end at the border
  if (o->Wiener && (o->blockSize - o->blockSizeWie) % std::gcd(st1, st2) != 0) return 1;
  if (prec == 32) gbm3d<float>(I, m, n, sigma, o, U, U1);
  else gbm3d<double>(I, m, n, sigma, o, U, U1);
  return 0;
}

int orc_match_video(int prec, const double* I, int m, int n, int F, int d, int K, uint32_t* S, void* Volume) {
  const size_t px = (size_t)m * n;
  if (prec == 32) {
    std::vector<float> t(px * F);
    for (size_t i = 0; i < t.size(); ++i) t[i] = (float)I[i];
    match_video<float>(t.data(), m, n, F, d, K, S, (float*)Volume);
  } else {
    match_video<double>(I, m, n, F, d, K, S, (double*)Volume);
  }
  return 0;
}

int orc_denoise_video(int prec, const void* Volume, int M, int N, int d, int F, int K, const uint32_t* S, int levels,
                      int cycleSpin, const double* tau, const orc_filters* f, double* U, double* W) {
  if (prec == 32) denoise_video<float>((const float*)Volume, M, N, d, F, K, S, levels, cycleSpin, tau, f, U, W);
  else denoise_video<double>((const double*)Volume, M, N, d, F, K, S, levels, cycleSpin, tau, f, U, W);
  return 0;
}

int orc_vbm3d(int prec, const double* I, int m, int n, int Kf, double sigma, int d, int K, int levels, int cycleSpin,
              int tauMode, const int* spins, int nS, int nF, const orc_filters* f, double* out) {
  if (nF < 1 || nF % 2 == 0 || nF > Kf) return 1;
  if (prec == 32) vbm3d<float>(I, m, n, Kf, sigma, d, K, levels, cycleSpin, tauMode, spins, nS, nF, f, out);
  else vbm3d<double>(I, m, n, Kf, sigma, d, K, levels, cycleSpin, tauMode, spins, nS, nF, f, out);
  return 0;
}

int orc_gbm3d_colored(int prec, const double* I, int m, int n, double sigma_match, const double* tau,
                      const double* sigwie, const orc_opts* o, double* U, double* U1) {
  const int st1 = o->refStride > 0 ? o->refStride : o->blockSize;
  const int st2 = o->refStrideWie > 0 ? o->refStrideWie : o->blockSizeWie;
  if (o->Wiener && (o->blockSize - o->blockSizeWie) % std::gcd(st1, st2) != 0) return 1;
  if (prec == 32) gbm3d<float>(I, m, n, sigma_match, o, U, U1, tau, sigwie);
  else gbm3d<double>(I, m, n, sigma_match, o, U, U1, tau, sigwie);
  return 0;
}

}  // extern "C"
