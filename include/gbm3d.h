/*
 * gbm3d.h — C ABI of the B200 (sm_100a) GBM3D two-step denoising library.
 *
 * Drop-in boundary for the MATLAB reference toby-sanders/GBM3D.  Each entry
 * point below replaces one MATLAB function that source/GBM3D.m calls; a MEX
 * gateway per function (gbm3d_b200/mex/) binds them under the reference's own
 * names so GBM3D.m / GBM3D_distributed.m / setBM3Dopts.m run unchanged.
 *
 * Conventions
 *   - Arrays are MATLAB column-major: element (r,c) of an m x n image is at
 *     r + c*m.  Host pointers unless the name ends in _device.
 *   - S (the match sets) is a uint32 array of K x M x N: S[k + K*(i + M*j)]
 *     is entry k of cell S{i+1,j+1}, a 1-based column-major index into the
 *     d2 x d2 search window (matchBlocksCPU.m:88,100-103).  S_count (M x N,
 *     may be NULL) holds numel(S{i,j}) when numMin < numMax lets a cell hold
 *     fewer than K matches; unused entries are 0.
 *   - Every call returns GBM3D_OK or an error code; gbm3d_last_error() gives
 *     the message.  The library never exits or aborts the process.
 *   - A context is bound to one device and one stream and is not thread-safe;
 *     use one context per host thread (MATLAB parfor workers are separate
 *     processes, each with its own context).
 *   - There is no CPU fallback: without a usable CUDA device every compute
 *     call fails with GBM3D_ERR_CUDA.
 */
#ifndef GBM3D_H
#define GBM3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GBM3D_OK 0
#define GBM3D_ERR_ARG 1         /* invalid argument / unsupported size */
#define GBM3D_ERR_CUDA 2        /* CUDA runtime error (or no device) */
#define GBM3D_ERR_NOMEM 3       /* device allocation failed */
#define GBM3D_ERR_NONFINITE 4   /* input holds NaN or Inf */
#define GBM3D_ERR_UNSUPPORTED 5 /* option value the reference has but this library does not */
#define GBM3D_ERR_TOO_LARGE 6   /* image exceeds the fixed scratch of gbm3d_matchBlocks_noalloc */

/* Size of the fixed device scratch of gbm3d_matchBlocks_noalloc, in floats
 * (16 MiB, held by every GPU that loads the library until the process exits). */
#define GBM3D_NOALLOC_MAX_FLOATS (4u << 20)

typedef struct gbm3d_ctx gbm3d_ctx;

/* Option struct with the reference's field names (utilities/setBM3Dopts.m:17-86,
 * utilities/checkBM3Dopts.m:10-24).  filtType: 0 = 'ht', 1 = 'median'.
 * refStride / refStrideWie: reference-block spacing of step 1 / step 2; 0 means
 * blockSize / blockSizeWie (the reference's tiling).  Not in the reference; with
 * stride s the references sit at 0, s, 2s, ... and M = floor((m-d)/s)+1.
 * staleWeights: 1 mirrors GBM3D.m:26-27,82 (step 2 reuses the step-1 weight
 * slices it does not overwrite). */
typedef struct gbm3d_opts {
  int numMax, numMin;
  int blockSize, blockSizeWie, matchSize, refStride;
  int levels, cycleSpin, tauMode;
  int Wiener, filtType;
  int nMatchSpins, matchSpins[8];
  int nMatchSpinsWie, matchSpinsWie[8];
  int staleWeights;
  int refStrideWie;
  int wavelet; /* step-1 bank of gbm3d_denoise: 0 = bior1.5 x Haar (GBM3D.m:40), 1 = 3D Haar */
  /* 0 plain (the reference's arithmetic, FP32); 1 precision form: block
   * distances on the bf16 tensor cores bound the candidates (every position
   * within the rounding bound of the K-th best), which are re-ranked by the
   * exact FP32 distance, so the match sets are the plain path's; aggregation
   * with Kahan-compensated FP32 sums; 2 learned pilot: the step-1 estimate
   * comes from the pilot network (gbm3d_pilot_*); 3 tensor form: the
   * precision form's matching with the plain aggregation, so the output is
   * the plain path's.  Tensor-core matching needs blockSize 8, numMin =
   * numMax <= 16 and 3 refStride + matchSize <= 56.  Not in the reference. */
  int form;
  /* video (gbm3d_vbm3d_device, gbm3d_matchBlocksV): frames in the temporal
   * window, odd; 0 means VBM3D.m's default of 11.  opts.wavelet = 2 selects
   * the video path's sym4 x Haar bank (getWaveFilters3D('sym','db',4,1)). */
  int videoFrames;
} gbm3d_opts;

/* Separable 3D wavelet bank: 1D analysis (a_) and synthesis (s_) filters for the
 * two spatial axes (len_xy taps) and for the slot axis (len_z taps).  The
 * reference's Psi/Psi2 (waveTransforms3D/getWaveFilters3Dbior.m:39-58) are the
 * outer products of these factors. */
typedef struct gbm3d_filters {
  int len_xy;
  double a_lo_xy[16], a_hi_xy[16], s_lo_xy[16], s_hi_xy[16];
  int len_z;
  double a_lo_z[16], a_hi_z[16], s_lo_z[16], s_hi_z[16];
} gbm3d_filters;

/* ---- context -------------------------------------------------------------- */
int gbm3d_ctx_create(int device, gbm3d_ctx** out);
void gbm3d_ctx_destroy(gbm3d_ctx* ctx);
/* Run subsequent work on this cudaStream_t (NULL = the context's own stream). */
int gbm3d_ctx_set_stream(gbm3d_ctx* ctx, void* cuda_stream);
/* Wait until the context's stream has finished all queued work. */
int gbm3d_ctx_synchronize(gbm3d_ctx* ctx);
const char* gbm3d_last_error(const gbm3d_ctx* ctx);
int gbm3d_version(void);

/* ---- option helpers ----------------------------------------------------------
 * gbm3d_default_opts   <- setBM3Dopts(profile)       utilities/setBM3Dopts.m:12-86
 * gbm3d_get_tau        <- getTau(levels,mode)        utilities/getTau.m:9-51
 * gbm3d_bior_filters   <- getWaveFilters3Dbior       waveTransforms3D/getWaveFilters3Dbior.m:12-58
 */
void gbm3d_default_opts(const char* profile, gbm3d_opts* out);
void gbm3d_get_tau(int levels, int mode, double* tau /* levels x 7 */);
void gbm3d_bior_filters(gbm3d_filters* out);

/* Separable factors of a Psi/Psi2 pair (single, Ly x Lx x Lz x 8 column-major,
 * the arguments denoiseAndAggregateGPU.m receives).  Host-only, no device
 * needed.  Returns GBM3D_ERR_ARG for a bank that is not an outer product of
 * 1D filters (every bank of the reference is). */
int gbm3d_filters_from_bank(const float* Psi, const float* Psi2, int len_xy, int len_z, gbm3d_filters* out);

/* ---- the reference's hot-path functions -------------------------------------- */

/* [S,Volume] = matchBlocksCPU(I,sigma,opts)           source/matchBlocksCPU.m:1-116
 * I: m x n double.  S: K x M x N, M=floor((m-d)/s)+1, N=floor((n-d)/s)+1 with
 * s = refStride (M = floor(m/d) for s = d).  S_count: M x N or NULL.  Volume:
 * m x n x K single for s = d, (M*d) x (N*d) x K otherwise, or NULL to skip
 * the gather. */
int gbm3d_matchBlocksCPU(gbm3d_ctx* ctx, const double* I, int m, int n, double sigma,
                         const gbm3d_opts* opts, uint32_t* S, int32_t* S_count, float* Volume);

/* S = matchBlocksGPU(I,sigma,opts)                       source/matchBlocksGPU.m:1-91
 * Global circular search: every block position of the m x n image is a
 * candidate; S (K x M x N) holds 1-based positions in the image, with no
 * slot-1 override.  When sigma > 30/255 the image is first prefiltered by the
 * reference's 5-shift, 3-level sym4 wavelet hard threshold (tau = 2 sigma),
 * which needs m and n divisible by 8.  Work grows as (m n)^2: small images. */
int gbm3d_matchBlocksGPU(gbm3d_ctx* ctx, const double* I, int m, int n, double sigma,
                         const gbm3d_opts* opts, uint32_t* S, int32_t* S_count);

/* [U,W] = denoiseAndAggregateGPU(Volume,S,tau,Psi,Psi2,opts)   source/denoiseAndAggregateGPU.m:1-92
 * Volume: (M*d) x (N*d) x K single; S: K x M x N; S_count may be NULL;
 * tau: levels x 7 double; filters: the separable factors of Psi/Psi2.
 * U, W: ((M-1)*s+d) x ((N-1)*s+d) double, s = refStride (M*d x N*d for s = d). */
int gbm3d_denoiseAndAggregateGPU(gbm3d_ctx* ctx, const float* Volume, const uint32_t* S,
                                 const int32_t* S_count, int M, int N, const double* tau,
                                 const gbm3d_filters* filters, const gbm3d_opts* opts,
                                 double* U, double* W);

/* [S,V1,V2] = matchBlocksWie(I,In,sigma,opts)            source/matchBlocksWie.m:1-92
 * I (pilot) and In (noisy): m x n double.  V1, V2: d x d x K x M x N single
 * (either may be NULL), M=floor((m-d)/s)+1 with s = refStrideWie. */
int gbm3d_matchBlocksWie(gbm3d_ctx* ctx, const double* I, const double* In, int m, int n,
                         double sigma, const gbm3d_opts* opts, uint32_t* S, float* V1, float* V2);

/* [U,W] = denoiseAndAggregateWieFast(V1,V2,S,sigma,opts)  source/denoiseAndAggregateWieFast.m:1-100
 * sigma: one double, or d x d doubles when sigma_is_matrix (broadcast over slots).
 * U, W: ((M-1)*s+d) x ((N-1)*s+d) double, s = refStrideWie. */
int gbm3d_denoiseAndAggregateWieFast(gbm3d_ctx* ctx, const float* V1, const float* V2,
                                     const uint32_t* S, int M, int N, const double* sigma,
                                     int sigma_is_matrix, const gbm3d_opts* opts,
                                     double* U, double* W);

/* [U,W] = denoiseAndAggregateWie(V1,V2,S,sigma,opts)      source/denoiseAndAggregateWie.m:1-90
 * Legacy variant: inverse DCT by the transpose and output clamped to [0,1]. */
int gbm3d_denoiseAndAggregateWie(gbm3d_ctx* ctx, const float* V1, const float* V2,
                                 const uint32_t* S, int M, int N, double sigma,
                                 const gbm3d_opts* opts, double* U, double* W);

/* [U,out] = GBM3D(I,sigma,opts)                            source/GBM3D.m:1-84
 * Whole two-step pipeline on the device.  I, U: m x n double host arrays;
 * U1 (out.U1, the step-1 estimate) may be NULL. */
int gbm3d_denoise(gbm3d_ctx* ctx, const double* I, int m, int n, double sigma,
                  const gbm3d_opts* opts, double* U, double* U1);

/* [U,out] = GBM3D(I,sigmaPSD,opts) for coloured noise (GBM3D.m:33-35): the
 * caller passes tau = getColoredTau(levels, sigmaPSD) (levels x 7),
 * sigmaWie = getColoredWie(sigmaPSD, blockSizeWie) (blockSizeWie^2, column-
 * major) and sigma_match = mean(sqrt(sigmaPSD(:))), the scalar the matchers
 * use (matchBlocksCPU.m:21).  Host pointers, as gbm3d_denoise. */
int gbm3d_denoise_colored(gbm3d_ctx* ctx, const double* I, int m, int n, double sigma_match, const double* tau,
                          const double* sigmaWie, const gbm3d_opts* opts, double* U, double* U1);

/* ---- learned pilot (opts.form = 2) -------------------------------------------------
 * A residual CNN (8 layers of 3x3 convolutions, 48 channels, bf16 weights and
 * activations, fp32 accumulation on the tensor cores) that produces the step-1
 * estimate from the noisy image and sigma; step 2 (Wiener) then runs as usual.
 * Not in the reference.  Parameters: fp32 vector of gbm3d_pilot_param_count()
 * values, per layer W [9][out][in] (tap = 3*dy + dx) then the bias [out];
 * inputs 2 (noisy/255, sigma/255), outputs 48, 48, ..., 1.  Images for the
 * pilot calls are fp32 device arrays [image][row][column]; sigma one float per
 * image (device).  A column-major m x n image is the [n][m] image here. */
int gbm3d_pilot_param_count(void);
int gbm3d_pilot_set_params(gbm3d_ctx* ctx, const float* params /* host */);
int gbm3d_pilot_get_params(gbm3d_ctx* ctx, float* params /* host */);
int gbm3d_pilot_forward(gbm3d_ctx* ctx, const float* img, const float* sigma, int nimg, int H, int W, float* pilot);
/* One Adam step (lr > 0) on mean((pilot - target)^2); *loss (host) gets the loss. */
int gbm3d_pilot_train_step(gbm3d_ctx* ctx, const float* img, const float* target, const float* sigma, int nimg,
                           int H, int W, float lr, float* loss);
/* Loss gradients (host, gbm3d_pilot_param_count() floats) without an update. */
int gbm3d_pilot_gradients(gbm3d_ctx* ctx, const float* img, const float* target, const float* sigma, int nimg,
                          int H, int W, float* grad, float* loss);

/* Colour GBM3D (device planes R, G, B; float64 column-major m x n): the
 * opponent transform Y = (R+G+B)/3, U = (R-B)/2, V = (R-2G+B)/4 (chroma
 * carried with an offset of 128 through the clamps at 0), block
 * matching on Y only, every channel filtered and aggregated with Y's match
 * sets at its own noise level (sigma/sqrt(3), sigma/sqrt(2), sigma*sqrt(3/8)),
 * and the inverse transform.  Asynchronous on the context stream.  Not in the
 * reference. */
int gbm3d_denoise_rgb_device(gbm3d_ctx* ctx, const double* R, const double* G, const double* B, int m, int n,
                             double sigma, const gbm3d_opts* opts, double* UR, double* UG, double* UB);

/* ---- video (source/VBM3D.m, matchBlocksV.m, denoiseAndAggregateV.m) ------------
 * Frames are float64 column-major m x n x frames on the reference's [0,1]
 * scale (the video step clamps its estimate to [0,1]).
 * [S,Volume] = matchBlocksV(I,sigma,opts)      source/matchBlocksV.m:21-116 (top-K)
 *   I: m x n x F (F = the window, odd); S: K x M x N (M = floor(m/d)), 1-based
 *   index a + (b-1) d + (f-1) d^2 into the d x d x F window; Volume m x n x K. */
int gbm3d_matchBlocksV(gbm3d_ctx* ctx, const double* I, int m, int n, int frames, const gbm3d_opts* opts,
                       uint32_t* S, float* Volume);
/* [U,out] = denoiseAndAggregateV(Y,Volume,I,S,sigma,opts)   source/denoiseAndAggregateV.m:11-89
 *   Volume (M d) x (N d) x K single; tau levels x 7 (sigma * getTau(levels, tauMode));
 *   filters NULL = sym4 x Haar.  U and W (= out.K): (M d) x (N d) x frames double. */
int gbm3d_denoiseAndAggregateV(gbm3d_ctx* ctx, const float* Volume, const uint32_t* S, int M, int N, int frames,
                               const double* tau, const gbm3d_filters* filters, const gbm3d_opts* opts, double* U,
                               double* W);
/* Y = VBM3D(I,sigma,opts)                                  source/VBM3D.m:20-63
 * Device pointers; out: m x n x (frames - videoFrames + 1), the frames with a
 * full temporal window.  Asynchronous on the context stream. */
int gbm3d_vbm3d_device(gbm3d_ctx* ctx, const double* I, int m, int n, int frames, double sigma,
                       const gbm3d_opts* opts, double* out);

/* Batched form: nimg images of any sizes (device pointers, float64
 * column-major, sigma per image) denoised with one option set.  With
 * use_graph, the first call runs the batch and captures its whole launch
 * sequence into one CUDA graph; a later call with the same pointers, sizes,
 * sigmas and options replays it with a single graph launch.  Asynchronous on
 * the context stream.  Not in the reference. */
int gbm3d_denoise_batch(gbm3d_ctx* ctx, int nimg, const double* const* I, const int* m, const int* n,
                        const double* sigma, const gbm3d_opts* opts, double* const* U, int use_graph);

/* Mixed batch: grey images, colour images and one video in one submission
 * (device pointers, float64 column-major).  Grey images run the whole-image
 * pipeline of gbm3d_denoise_device with opts (or their own grey_opts entry) at
 * their own sigma, colour images the opponent-space pipeline of
 * gbm3d_denoise_rgb_device with opts (or their rgb_opts entry), and the
 * video the VBM3D pipeline of gbm3d_vbm3d_device with video_opts (frames on
 * the [0,1] scale).  Any part may be empty (count 0, video null).  With
 * use_graph the first call runs everything and captures the whole launch
 * sequence into one CUDA graph; a later call with the same pointers, sizes,
 * sigmas and options replays it with a single graph launch (this replaces the
 * graph of gbm3d_denoise_batch, and the reverse).  Every output equals the
 * single-image entry's.  Asynchronous on the context stream.  Not in the
 * reference. */
typedef struct gbm3d_mixed_batch {
  int n_grey;
  const double* const* grey;      /* n_grey images */
  const int* grey_m;
  const int* grey_n;
  const double* grey_sigma;
  double* const* grey_out;
  int n_rgb;
  const double* const* rgb;       /* 3 n_rgb planes: R, G, B of image 0, then of image 1, ... */
  const int* rgb_m;
  const int* rgb_n;
  const double* rgb_sigma;
  double* const* rgb_out;         /* 3 n_rgb output planes, in the same order */
  const double* video;            /* video_m x video_n x video_frames, or null */
  int video_m, video_n, video_frames;
  double video_sigma;
  double* video_out;              /* video_m x video_n x (video_frames - videoFrames + 1) */
  /* Per-image options: n_grey (n_rgb) structs, image k taking entry k, or
   * null for the call's opts on every image of that kind.  A batch of uneven
   * sizes and noise levels can so give each image the autotuner's set for its
   * own size and sigma class.  Leave both null (zero-initialise the struct)
   * when one option set serves the whole batch. */
  const gbm3d_opts* grey_opts;
  const gbm3d_opts* rgb_opts;
} gbm3d_mixed_batch;
int gbm3d_denoise_mixed(gbm3d_ctx* ctx, const gbm3d_mixed_batch* batch, const gbm3d_opts* opts,
                        const gbm3d_opts* video_opts, int use_graph);
/* Lanes of gbm3d_denoise_mixed (1..16, default 1).  The submission's items
 * (images, colour images, the video) go to `lanes` streams, the largest first
 * to the least-loaded lane.  Each lane has its own buffers, and the lanes run
 * at once, inside one graph when use_graph is set, so small images' launches
 * fill the GPU together.  Every output is the same as with one lane.  The
 * learned-pilot form always runs on one lane.  Not in the reference: its
 * parfor over work items (GBM3D_distributed.m:54,94) is the host-side
 * counterpart. */
int gbm3d_ctx_set_lanes(gbm3d_ctx* ctx, int lanes);

/* Asynchronous form of gbm3d_denoise for a stream of images (U1 is not
 * returned): the call enqueues the host-to-device copy of I, the whole
 * pipeline and the device-to-host copy into U, and returns.  Copies run on
 * their own streams and the device keeps two input and two output slots, so
 * the copies of one call overlap the compute of the previous one.  I and U
 * must stay valid, and I unchanged, until gbm3d_ctx_synchronize, which also
 * reports a non-finite input among the calls since the last synchronisation.
 * Pinned (page-locked) host buffers are needed for the copies to overlap.
 * Not in the reference. */
int gbm3d_denoise_async(gbm3d_ctx* ctx, const double* I, int m, int n, double sigma, const gbm3d_opts* opts,
                        double* U);

/* ---- U = GBM3D_distributed(I,sigma,opts) on the device ----------------------------
 * source/GBM3D_distributed.m:54-120: the image is cut into overlapping tiles
 * (items from getBM3D_distribution: n_items rows of r1, r2, r3, r4, spin with
 * 1-based inclusive bounds, int32), each item is denoised on its own and the
 * tiles are stitched with ramp windows.  Device pointers (float64 column-major
 * images), results as the reference computes them tile by tile.
 * gbm3d_tiles_device: step 1 (pilot NULL) runs matchBlocksCPU +
 * denoiseAndAggregateGPU on circshift(I(r1:r2,r3:r4),[s s]) with tau (host,
 * levels x 7) and the bior1.5 x Haar bank; step 2 (pilot = the step-1
 * estimate) runs matchBlocksWie on the pilot tile + denoiseAndAggregateWieFast
 * at sigma.  Item ii writes circshift(U,[-s -s]) then circshift(W,[-s -s])
 * (column-major ny x nx each) at out + 2 tile^2 ii; every tile side is at most
 * `tile` and a whole reference grid.  The item table is host memory.
 * gbm3d_tiles_stitch_device: out = (sum over items, in table order, of
 * U .* win) ./ (sum of win .* W) (GBM3D_distributed.m:62-72, :103-113),
 * win = makeInterpWindow(ny, nx, k) built from ramp = linspace(0.01, 1, k)
 * (host).  Not in the reference: the reference runs these loops as parfor
 * over MATLAB workers. */
int gbm3d_tiles_device(gbm3d_ctx* ctx, const double* I, const double* pilot, int m, int n, double sigma,
                       const double* tau, const gbm3d_opts* opts, const int* items, int n_items, int tile,
                       double* out);
int gbm3d_tiles_stitch_device(gbm3d_ctx* ctx, const double* tiles, const int* items, int n_items, int tile, int m,
                              int n, int k, const double* ramp, double* out);

/* Same as gbm3d_denoise with device pointers; no host copies.  Asynchronous on
 * the context stream (synchronise before reading U). */
int gbm3d_denoise_device(gbm3d_ctx* ctx, const double* I, int m, int n, double sigma,
                         const gbm3d_opts* opts, double* U, double* U1);

/* The strip form: output columns [col_lo, col_hi) of gbm3d_denoise_device's
 * result, bit-identical to those columns of the whole-image call, into U
 * (m x (col_hi - col_lo), column-major, device).  I is the whole m x n image on
 * the device.  Every stage runs on the columns its consumers read (the strip
 * plus the halo that spin shifts, the search windows and the wavelet filters
 * reach), so one GPU per strip splits a single image with no exchange before
 * the final gather.  Forms 0 (plain) and 2 (learned pilot); the tensor-core
 * forms return GBM3D_ERR_UNSUPPORTED.  Replaces nothing in the reference: its
 * GBM3D.m:22-83 runs the whole image on one GPU.  Asynchronous on the context
 * stream. */
int gbm3d_denoise_strip_device(gbm3d_ctx* ctx, const double* I, int m, int n, double sigma,
                               const gbm3d_opts* opts, int col_lo, int col_hi, double* U);
/* Host only (no GPU needed): the share of the whole image's references that the
 * strip [col_lo, col_hi) matches, averaged over the spins of each step:
 * frac[0] step 1, frac[1] step 2 (0 without a Wiener step). */
int gbm3d_strip_work(const gbm3d_opts* opts, int m, int n, int col_lo, int col_hi, double* frac);

/* Per-stage device times (ms) of the last pipeline call, by CUDA events:
 * [0] prepare, [1] step-1 matching, [2] step-1 wavelet, [3] step-1 aggregation,
 * [4] step-2 matching, [5] step-2 Wiener, [6] step-2 aggregation, [7] total.
 * Returns the number of entries written.  Timing is recorded only after
 * gbm3d_ctx_enable_timing(ctx, 1). */
int gbm3d_ctx_enable_timing(gbm3d_ctx* ctx, int on);
int gbm3d_stage_times(const gbm3d_ctx* ctx, float* ms, int n);

/* Tensor-core matcher (forms 1 and 3): the limit of each of its waits for a
 * TMA copy or its MMAs, in SM clocks (0, the default: about two seconds).  A
 * wait that runs out ends the kernel's work after its own copies and MMAs in
 * flight have landed, and the call reports GBM3D_ERR_CUDA ("... did not
 * complete within its wait limit").  A negative value is a probe of that
 * path: every CTA first waits, with the limit -cycles, on a barrier that
 * nothing completes, so the next matching call fails that way.  Not in the
 * reference. */
int gbm3d_ctx_set_tc_wait(gbm3d_ctx* ctx, long long cycles);

/* Tensor-core matcher statistics: with enable = 1 the following calls count,
 * per reference block, the candidates its bound leaves for the exact re-rank
 * (hist[b] = references with 8 b .. 8 b + 7 candidates, hist[32] = 256 or
 * more; references with more than 64 are finished by the exhaustive matcher).  With hist non-null the counts
 * so far are copied out (the context stream is synchronised) and reset.  Not
 * in the reference. */
int gbm3d_ctx_tc_stats(gbm3d_ctx* ctx, int enable, int32_t* hist);

/* Number of kernels the last pipeline call launched. */
int gbm3d_last_launch_count(const gbm3d_ctx* ctx);

/* With timing on: device time (ms) summed over the last call's launches of
 * the kernel family `name` ("match", "wav_analysis", "wav_synthesis",
 * "aggregate", "wiener", "ht_weights", "make_pad", "accum", "ratio", "prep",
 * ...), measured between CUDA events recorded after consecutive launches on
 * the context stream.  Returns the number of such launches, or -1. */
int gbm3d_kernel_time(const gbm3d_ctx* ctx, const char* name, float* total_ms);

/* Tensor-core self-check: C (128 x 256 fp32, row-major) = A B^T for A 128 x 64
 * and B 256 x 64 row-major bf16 (raw 16-bit patterns), computed by one
 * tcgen05 MMA sequence with the operand layouts the matcher and the pilot
 * network use.  Host pointers. */
int gbm3d_tc_selfcheck(gbm3d_ctx* ctx, const uint16_t* A, const uint16_t* B, float* C);
/* The same product with the operand layout selected: mn_major = 0 stages A and
 * B K-major (as gbm3d_tc_selfcheck); 1 stages both MN-major (8 K-rows x 8
 * consecutive M or N elements per core matrix), the layout the pilot's
 * weight gradient reads its activation tiles in, with the descriptor's leading
 * byte offset the K-adjacent core stride and its stride byte offset the
 * M-adjacent one; 2 the same with the two offsets exchanged. */
int gbm3d_tc_selfcheck_layout(gbm3d_ctx* ctx, int mn_major, const uint16_t* A, const uint16_t* B, float* C);

/* Step-1 block matching that allocates nothing.  No counterpart in the
 * reference: it exists for callers that may not allocate device memory while
 * they run (servers and video pipelines that reserve all GPU memory at
 * start-up so no call can run out of memory or stall in the device-wide
 * synchronisation of cudaFree, and host applications whose own allocator owns
 * every device buffer).  Same search and selection as gbm3d_matchBlocksCPU.
 *   I: single-precision m x n image on the device (the single(I) of
 *      matchBlocksCPU.m:31); S: K x M x N uint32 and S_count: M x N int32
 *      (may be NULL) on the device; stream: a cudaStream_t (NULL = default).
 * The work is queued on the stream and not waited for.  Scratch is a fixed
 * device array of GBM3D_NOALLOC_MAX_FLOATS floats shared by all calls: an
 * image whose search image needs more, ((m+matchSize+3)/4*4) * (n+matchSize)
 * floats (about 2000 x 2000 pixels at matchSize 32), returns
 * GBM3D_ERR_TOO_LARGE before any work, and calls that overlap on the GPU (other streams or
 * host threads) race on it.  The first call on each device looks the
 * scratch's address up with cudaGetSymbolAddress; make that first call
 * before any stream capture.  No context, no gbm3d_last_error: the return
 * code is the whole report.  Unlike the context entry points, this one does
 * not scan the image for NaN or Inf (that needs a status word and a wait):
 * the caller passes a finite image, or gets match sets ranked on NaN
 * distances with GBM3D_OK. */
int gbm3d_matchBlocks_noalloc(const float* I, int m, int n, double sigma, const gbm3d_opts* opts,
                              uint32_t* S, int32_t* S_count, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GBM3D_H */
