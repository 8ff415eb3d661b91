"""Reference-named entry points over the CUDA library.

Each function has the name, argument meaning and return values of the MATLAB
function of toby-sanders/GBM3D it replaces, and calls libgbm3d.so through its
C ABI.  Arrays follow MATLAB's column-major layout (numpy order='F'):

  U, out          = GBM3D(I, sigma, opts)                     source/GBM3D.m:1
  S, Volume       = matchBlocksCPU(I, sigma, opts)            source/matchBlocksCPU.m:1
  S               = matchBlocksGPU(I, sigma, opts)            source/matchBlocksGPU.m:1
  U, W            = denoiseAndAggregateGPU(Volume, S, tau, Psi, Psi2, opts)
                                                              source/denoiseAndAggregateGPU.m:1
  S, V1, V2       = matchBlocksWie(I, In, sigma, opts)        source/matchBlocksWie.m:1
  U, W            = denoiseAndAggregateWieFast(V1, V2, S, sigma, opts)
                                                              source/denoiseAndAggregateWieFast.m:1
  U, W            = denoiseAndAggregateWie(V1, V2, S, sigma, opts)
                                                              source/denoiseAndAggregateWie.m:1
  Y, out          = VBM3D(I, sigma, opts)                     source/VBM3D.m:1
  S, Volume       = matchBlocksV(I, sigma, opts)              source/matchBlocksV.m:1
  U, out          = denoiseAndAggregateV(Y, Volume, I, S, sigma, opts)
                                                              source/denoiseAndAggregateV.m:1

S is returned as a MatchSet: a uint32 array of shape (K, M, N) whose column
S[:, i, j] is the reference's cell S{i+1, j+1}, plus the per-cell counts.
Errors raise GBM3DError with the library's message, as the MATLAB code raises
error(); nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import options as _opt
from ._lib import Context, GBM3DError, context, gbm3d_filters, gbm3d_mixed_batch, gbm3d_opts, lib


class MatchSet(np.ndarray):
    """uint32 (K, M, N) match indices; ``.count`` is numel(S{i,j}) per cell."""

    count: np.ndarray | None = None

    def cell(self, i: int, j: int) -> np.ndarray:
        """The MATLAB cell S{i+1, j+1} (trailing unused entries removed)."""
        k = self.shape[0] if self.count is None else int(self.count[i, j])
        return np.asarray(self[:k, i, j])


def _as_set(S, count=None) -> MatchSet:
    out = np.asfortranarray(S, dtype=np.uint32).view(MatchSet)
    out.count = count
    return out


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


# opts['form']: plain (FP32, the reference's arithmetic); precision (bf16
# tensor-core distances bound the candidates, exact FP32 re-rank, Kahan
# aggregation); learned (the pilot network replaces step 1); tensor (the
# tensor-core matcher with plain aggregation: the plain path's output)
FORMS = {"plain": 0, "precision": 1, "learned": 2, "tensor": 3}


def c_opts(opts: dict) -> gbm3d_opts:
    o = _opt.checkBM3Dopts(opts)
    c = gbm3d_opts()
    c.numMax, c.numMin = int(o["numMax"]), int(o["numMin"])
    c.blockSize, c.blockSizeWie, c.matchSize = int(o["blockSize"]), int(o["blockSizeWie"]), int(o["matchSize"])
    s1, s2 = _opt.strides(o)
    c.refStride = 0 if s1 == int(o["blockSize"]) else s1
    c.refStrideWie = 0 if s2 == int(o["blockSizeWie"]) else s2
    c.levels, c.cycleSpin, c.tauMode = int(o["levels"]), int(o["cycleSpin"]), int(o["tauMode"])
    c.Wiener = 1 if o["Wiener"] else 0
    ft = o.get("filtType", "ht")
    if ft not in ("ht", "median"):
        raise GBM3DError(1, "unrecognized filtering")  # denoiseAndAggregateGPU.m:54
    c.filtType = 0 if ft == "ht" else 1
    ms, mw = list(o["matchSpins"]), list(o["matchSpinsWie"])
    if len(ms) > 8 or len(mw) > 8:
        raise GBM3DError(1, "at most 8 match spins per step")
    c.nMatchSpins = len(ms)
    for i, s in enumerate(ms):
        c.matchSpins[i] = int(s)
    c.nMatchSpinsWie = len(mw)
    for i, s in enumerate(mw):
        c.matchSpinsWie[i] = int(s)
    c.staleWeights = 1 if o.get("staleWeights", True) else 0
    wn = o.get("wname", "bior")
    if wn not in ("bior", "haar"):
        raise GBM3DError(5, f"wname '{wn}': the pipeline's banks are 'bior' (bior1.5 x Haar) and 'haar'")
    c.wavelet = 1 if wn == "haar" else 0
    form = o.get("form", "plain")
    if form not in FORMS:
        raise GBM3DError(5, f"form '{form}': one of {', '.join(FORMS)}")
    c.form = FORMS[form]
    return c


def c_filters(fac: dict) -> gbm3d_filters:
    f = gbm3d_filters()
    f.len_xy = len(fac["a_lo_xy"])
    f.len_z = len(fac["a_lo_z"])
    for k in ("a_lo_xy", "a_hi_xy", "s_lo_xy", "s_hi_xy", "a_lo_z", "a_hi_z", "s_lo_z", "s_hi_z"):
        v = np.asarray(fac[k], dtype=np.float64)
        if v.size > 16:
            raise GBM3DError(5, "filters longer than 16 taps are not supported")
        getattr(f, k)[: v.size] = list(v)
    return f


def _sigma_scalar(sigma) -> float:
    """matchBlocksCPU.m:21 — a coloured-noise sigma matrix becomes mean(sqrt(sigma))."""
    s = np.asarray(sigma, dtype=np.float64)
    if s.ndim >= 1 and s.shape[0] > 1:
        return float(np.mean(np.sqrt(s)))
    return float(s.reshape(-1)[0])


def matchBlocksCPU(I, sigma, opts: dict, ctx: Context | None = None, volume: bool = True):
    """[S, Volume] = matchBlocksCPU(I, sigma, opts).

    With refStride s != blockSize the Volume is tile-space, (M d) x (N d) x K.
    volume=False skips the gather and returns None for it (the C ABI's NULL
    Volume): large images at dense strides need only the match sets.
    """
    ctx = ctx or context()
    o = _opt.checkBM3Dopts(opts)
    I = np.asfortranarray(I, dtype=np.float64)
    m, n = I.shape
    d, K = int(o["blockSize"]), int(o["numMax"])
    s = _opt.strides(o)[0]
    M, N = _opt.grid_count(m, d, s), _opt.grid_count(n, d, s)
    S = np.zeros((K, M, N), dtype=np.uint32, order="F")
    cnt = np.zeros((M, N), dtype=np.int32, order="F")
    V = np.zeros((m, n, K) if s == d else (M * d, N * d, K), dtype=np.float32, order="F") if volume else None
    co = c_opts(o)
    ctx.check(lib().gbm3d_matchBlocksCPU(ctx.h, _p(I), m, n, _sigma_scalar(sigma), C.byref(co),
                                         _p(S), _p(cnt), _p(V) if volume else None))
    return _as_set(S, cnt), V


def matchBlocksGPU(I, sigma, opts: dict, ctx: Context | None = None):
    """S = matchBlocksGPU(I, sigma, opts): global circular search over the
    whole image (indices into the m x n image, no slot-1 override), after the
    sym4 prefilter when sigma > 30/255 (matchBlocksGPU.m:34)."""
    ctx = ctx or context()
    o = _opt.checkBM3Dopts(opts)
    I = np.asfortranarray(I, dtype=np.float64)
    m, n = I.shape
    d, K = int(o["blockSize"]), int(o["numMax"])
    M, N = m // d, n // d
    S = np.zeros((K, M, N), dtype=np.uint32, order="F")
    cnt = np.zeros((M, N), dtype=np.int32, order="F")
    co = c_opts(o)
    ctx.check(lib().gbm3d_matchBlocksGPU(ctx.h, _p(I), m, n, float(sigma), C.byref(co), _p(S), _p(cnt)))
    return _as_set(S, cnt)


def denoiseAndAggregateGPU(Volume, S, tau, Psi, Psi2, opts: dict, ctx: Context | None = None):
    """[U, W] = denoiseAndAggregateGPU(Volume, S, tau, Psi, Psi2, opts).

    Psi/Psi2 may be the reference's 4D banks (factorised into separable 1D
    filters) or None for the default bior1.5 x Haar bank.
    """
    ctx = ctx or context()
    o = _opt.checkBM3Dopts(opts)
    if o.get("filtType", "ht") not in ("ht", "median"):
        raise GBM3DError(1, "unrecognized filtering")
    fac = _opt.bior_factors() if Psi is None else _opt.factors_from_bank(Psi, Psi2)
    Volume = np.asfortranarray(Volume, dtype=np.float32)
    K, M, N = S.shape
    cnt = getattr(S, "count", None)
    Sa = np.asfortranarray(S, dtype=np.uint32)
    d = int(o["blockSize"])
    if Volume.shape != (M * d, N * d, K):
        raise GBM3DError(1, f"Volume shape {Volume.shape} does not match S ({M * d}, {N * d}, {K})")
    tau = np.asfortranarray(tau, dtype=np.float64)
    if tau.shape != (int(o["levels"]), 7):
        raise GBM3DError(1, "tau must be levels x 7")
    s = _opt.strides(o)[0]
    U = np.zeros(((M - 1) * s + d, (N - 1) * s + d), order="F")
    W = np.zeros_like(U)
    co, cf = c_opts(o), c_filters(fac)
    cp = None
    if cnt is not None:
        cnt = np.asfortranarray(cnt, dtype=np.int32)
        cp = _p(cnt)
    ctx.check(lib().gbm3d_denoiseAndAggregateGPU(ctx.h, _p(Volume), _p(Sa), cp, M, N, _p(tau), C.byref(cf),
                                                 C.byref(co), _p(U), _p(W)))
    return U, W


def matchBlocksWie(I, In, sigma, opts: dict, ctx: Context | None = None):
    """[S, V1, V2] = matchBlocksWie(I, In, sigma, opts)."""
    ctx = ctx or context()
    o = _opt.checkBM3Dopts(opts)
    I = np.asfortranarray(I, dtype=np.float64)
    In = np.asfortranarray(In, dtype=np.float64)
    if I.shape != In.shape:
        raise GBM3DError(1, "I and In must have the same size")
    m, n = I.shape
    d, K = int(o["blockSizeWie"]), int(o["numMax"])
    s = _opt.strides(o)[1]
    M, N = _opt.grid_count(m, d, s), _opt.grid_count(n, d, s)
    S = np.zeros((K, M, N), dtype=np.uint32, order="F")
    V1 = np.zeros((d, d, K, M, N), dtype=np.float32, order="F")
    V2 = np.zeros_like(V1)
    co = c_opts(o)
    ctx.check(lib().gbm3d_matchBlocksWie(ctx.h, _p(I), _p(In), m, n, _sigma_scalar(sigma), C.byref(co),
                                         _p(S), _p(V1), _p(V2)))
    return _as_set(S), V1, V2


def _wiener(V1, V2, S, sigma, opts, ctx, variant):
    ctx = ctx or context()
    o = _opt.checkBM3Dopts(opts)
    V1 = np.asfortranarray(V1, dtype=np.float32)
    V2 = np.asfortranarray(V2, dtype=np.float32)
    d, _, K, M, N = V1.shape
    if V2.shape != V1.shape or S.shape != (K, M, N):
        raise GBM3DError(1, "V1, V2 and S sizes disagree")
    s = _opt.strides(o)[1]
    o = dict(o, blockSizeWie=d, numMax=K, numMin=min(int(o["numMin"]), K), refStrideWie=s)
    Sa = np.asfortranarray(S, dtype=np.uint32)
    sg = np.asfortranarray(np.atleast_1d(np.asarray(sigma, dtype=np.float64)))
    U = np.zeros(((M - 1) * s + d, (N - 1) * s + d), order="F")
    W = np.zeros_like(U)
    co = c_opts(o)
    if variant == 0:
        is_mat = 1 if sg.size > 1 else 0
        if is_mat and sg.shape != (d, d):
            raise GBM3DError(1, "sigma must be a scalar or a d x d matrix")
        ctx.check(lib().gbm3d_denoiseAndAggregateWieFast(ctx.h, _p(V1), _p(V2), _p(Sa), M, N, _p(sg), is_mat,
                                                         C.byref(co), _p(U), _p(W)))
    else:
        if sg.size != 1:
            raise GBM3DError(5, "denoiseAndAggregateWie takes a scalar sigma")
        ctx.check(lib().gbm3d_denoiseAndAggregateWie(ctx.h, _p(V1), _p(V2), _p(Sa), M, N, float(sg[0]),
                                                     C.byref(co), _p(U), _p(W)))
    return U, W


def denoiseAndAggregateWieFast(V1, V2, S, sigma, opts: dict, ctx: Context | None = None):
    """[U, W] = denoiseAndAggregateWieFast(V1, V2, S, sigma, opts)."""
    return _wiener(V1, V2, S, sigma, opts, ctx, 0)


def denoiseAndAggregateWie(V1, V2, S, sigma, opts: dict, ctx: Context | None = None):
    """[U, W] = denoiseAndAggregateWie(V1, V2, S, sigma, opts) (legacy variant)."""
    return _wiener(V1, V2, S, sigma, opts, ctx, 1)


def GBM3D(I, sigma, opts: dict | None = None, ctx: Context | None = None):
    """[U, out] = GBM3D(I, sigma, opts); out['U1'] is the step-1 estimate.

    ``opts`` with a 'profile' field is replaced by that profile (GBM3D.m:16-19);
    the 'tuned' profile picks the calibrated option set for the image's size
    and sigma (options.tuned_opts).
    """
    ctx = ctx or context()
    I = np.asfortranarray(I, dtype=np.float64)
    m, n = I.shape
    o = _opt.resolve_opts(opts, shape=(m, n), sigma=sigma)
    U = np.zeros((m, n), order="F")
    U1 = np.zeros((m, n), order="F")
    co = c_opts(o)
    sg = np.asarray(sigma, dtype=np.float64)
    if sg.ndim >= 1 and sg.shape[0] > 1:
        # coloured noise, sigma = sigma^2 * PSD (GBM3D.m:33-35)
        tau = np.asfortranarray(_opt.getColoredTau(int(o["levels"]), sg))
        swie = np.asfortranarray(_opt.getColoredWie(sg, int(o["blockSizeWie"])))
        ctx.check(lib().gbm3d_denoise_colored(ctx.h, _p(I), m, n, _sigma_scalar(sg), _p(tau), _p(swie),
                                              C.byref(co), _p(U), _p(U1)))
        return U, {"U1": U1, "tau": tau, "sigmaWie": swie}
    ctx.check(lib().gbm3d_denoise(ctx.h, _p(I), m, n, float(sg.reshape(-1)[0]), C.byref(co), _p(U), _p(U1)))
    return U, {"U1": U1}


def GBM3D_device(I_ptr: int, m: int, n: int, sigma: float, U_ptr: int, opts: dict | None = None,
                 U1_ptr: int = 0, ctx: Context | None = None) -> None:
    """Whole pipeline on device buffers (float64, column-major), asynchronous on the context stream."""
    ctx = ctx or context()
    co = c_opts(_opt.resolve_opts(opts, shape=(m, n), sigma=sigma))
    ctx.check(lib().gbm3d_denoise_device(ctx.h, C.c_void_p(I_ptr), m, n, float(sigma), C.byref(co),
                                         C.c_void_p(U_ptr), C.c_void_p(U1_ptr or 0)))


def GBM3D_strip_device(I_ptr: int, m: int, n: int, sigma: float, col_lo: int, col_hi: int, U_ptr: int,
                       opts: dict | None = None, ctx: Context | None = None) -> None:
    """Strip form: columns [col_lo, col_hi) of GBM3D_device's result (bit-identical
    to them) into U_ptr (float64, column-major m x (col_hi - col_lo)) from the
    whole image I_ptr (m x n), asynchronous on the context stream.  The options
    resolve for the whole image's size, as the whole-image call does."""
    ctx = ctx or context()
    co = c_opts(_opt.resolve_opts(opts, shape=(m, n), sigma=sigma))
    ctx.check(lib().gbm3d_denoise_strip_device(ctx.h, C.c_void_p(I_ptr), m, n, float(sigma), C.byref(co),
                                               int(col_lo), int(col_hi), C.c_void_p(U_ptr)))


def strip_work(m: int, n: int, col_lo: int, col_hi: int, opts: dict | None = None,
               sigma: float | None = None) -> tuple[float, float]:
    """Share of the whole image's references that the strip [col_lo, col_hi)
    matches in step 1 and step 2 (host only, no GPU)."""
    co = c_opts(_opt.resolve_opts(opts, shape=(m, n), sigma=sigma))
    frac = (C.c_double * 2)()
    rc = lib().gbm3d_strip_work(C.byref(co), m, n, int(col_lo), int(col_hi), frac)
    if rc != 0:
        raise GBM3DError(rc, "gbm3d_strip_work: invalid arguments")
    return float(frac[0]), float(frac[1])


def GBM3D_async(I_ptr: int, m: int, n: int, sigma: float, U_ptr: int, opts: dict | None = None,
                ctx: Context | None = None) -> None:
    """Enqueue one whole denoise of a host image (I_ptr: pinned float64,
    column-major m x n) into a host output U_ptr and return at once
    (gbm3d_denoise_async).  Successive calls overlap their copies with the
    previous call's compute; ``ctx.synchronize()`` waits for them all."""
    ctx = ctx or context()
    co = c_opts(_opt.resolve_opts(opts, shape=(m, n), sigma=sigma))
    ctx.check(lib().gbm3d_denoise_async(ctx.h, C.c_void_p(I_ptr), m, n, float(sigma), C.byref(co),
                                        C.c_void_p(U_ptr)))


def GBM3D_batch(images, sigmas, opts: dict | None = None, use_graph: bool = True, ctx: Context | None = None,
                outputs=None):
    """Batched form: denoise a list of device images (torch float64 tensors of
    shape (n, m), i.e. column-major m x n arrays) with one option set in one
    call; with use_graph the launch sequence is captured once into a CUDA graph
    and replayed when the same batch is denoised again.  Returns the outputs
    (allocated like the inputs unless given) once the work has finished."""
    import torch
    ctx = ctx or context()
    o = _opt.resolve_opts(opts)
    k = len(images)
    outs = outputs if outputs is not None else [torch.empty_like(x) for x in images]
    Ip = (C.c_void_p * k)(*[x.data_ptr() for x in images])
    Up = (C.c_void_p * k)(*[u.data_ptr() for u in outs])
    ms = (C.c_int * k)(*[int(x.shape[1]) for x in images])
    ns = (C.c_int * k)(*[int(x.shape[0]) for x in images])
    sg = (C.c_double * k)(*[float(s) for s in sigmas])
    co = c_opts(o)
    torch.cuda.synchronize()
    ctx.check(lib().gbm3d_denoise_batch(ctx.h, k, Ip, ms, ns, sg, C.byref(co), Up, 1 if use_graph else 0))
    ctx.check(lib().gbm3d_ctx_synchronize(ctx.h))
    return outs


def GBM3D_rgb(I, sigma, opts: dict | None = None, ctx: Context | None = None):
    """Colour GBM3D of an m x n x 3 RGB image (host array): opponent colour
    space, luma-driven block matching, every channel filtered with luma's
    match sets (gbm3d_denoise_rgb_device)."""
    import torch
    ctx = ctx or context()
    I = np.asarray(I, dtype=np.float64)
    m, n, _ = I.shape
    o = _opt.resolve_opts(opts, shape=(m, n), sigma=sigma)
    planes = [torch.from_numpy(np.asfortranarray(I[:, :, k]).ravel(order="F").copy()).cuda() for k in range(3)]
    outs = [torch.empty_like(p) for p in planes]
    co = c_opts(o)
    torch.cuda.synchronize()
    ctx.check(lib().gbm3d_denoise_rgb_device(ctx.h, *[C.c_void_p(p.data_ptr()) for p in planes], m, n, float(sigma),
                                             C.byref(co), *[C.c_void_p(u.data_ptr()) for u in outs]))
    ctx.check(lib().gbm3d_ctx_synchronize(ctx.h))
    return np.stack([u.cpu().numpy().reshape(m, n, order="F") for u in outs], axis=2)


def mixed_option_sets(opts, grey_opts, rgb_opts, n_grey: int, n_rgb: int):
    """(call-level options, per-grey-image option list or None, per-colour-
    image option list or None) of a mixed submission.  The 'tuned' profile
    depends on each image's size and sigma, so ``opts`` of that profile
    becomes every image's own entry (resolved per image) unless per-image
    lists are given; the call-level set is then the dense configuration,
    which no image uses."""
    if isinstance(opts, dict) and opts.get("profile") == "tuned":
        grey_opts = [opts] * n_grey if grey_opts is None else grey_opts
        rgb_opts = [opts] * n_rgb if rgb_opts is None else rgb_opts
        opts = dict(_opt.setBM3Dopts("default"), **_opt.DENSE)
    return opts, grey_opts, rgb_opts


def GBM3D_mixed(grey=(), grey_sigma=(), rgb=(), rgb_sigma=(), video=None, video_sigma: float = 0.0,
                opts: dict | None = None, vopts: dict | None = None, use_graph: bool = True,
                ctx: Context | None = None, outputs=None, grey_opts=None, rgb_opts=None):
    """Batched form over a mixed submission (gbm3d_denoise_mixed): grey
    device images (torch float64 (n, m) tensors, i.e. column-major m x n),
    colour images as (R, G, B) triples of such tensors, and one video (a
    torch float64 (frames, n, m) tensor on the [0, 1] scale), denoised in one
    call; with use_graph the whole launch sequence is captured into one CUDA
    graph on the first call and replayed by later calls with the same
    geometry.  Grey and colour images use ``opts``, the video ``vopts``
    (VBM3D.m's defaults).  ``grey_opts`` / ``rgb_opts``, when given, hold one
    option dict per image instead, each resolved at that image's size and
    sigma (so {"profile": "tuned"} gives every image the autotuner's set for
    its own size and noise class; ``opts`` of the 'tuned' profile does the
    same for every image without a list of its own).  Returns (grey outputs,
    colour output triples, video output (frames - nF + 1, n, m) or None) once
    the work has finished."""
    import torch
    ctx = ctx or context()
    opts, grey_opts, rgb_opts = mixed_option_sets(opts, grey_opts, rgb_opts, len(grey), len(rgb))
    o = c_opts(_opt.resolve_opts(opts))
    cv = c_video_opts(vopts) if video is not None else None
    grey, rgb = list(grey), [tuple(t) for t in rgb]
    if outputs is None:
        outputs = ([torch.empty_like(x) for x in grey], [tuple(torch.empty_like(p) for p in t) for t in rgb],
                   None if video is None else torch.empty((video.shape[0] - cv.videoFrames + 1,) + tuple(video.shape[1:]),
                                                          dtype=torch.float64, device=video.device))
    g_out, c_out, v_out = outputs
    b = gbm3d_mixed_batch()
    keep = []

    def arr(ctype, vals):
        a = (ctype * max(len(vals), 1))(*vals)
        keep.append(a)
        return C.cast(a, C.c_void_p)

    b.n_grey = len(grey)
    b.grey = arr(C.c_void_p, [x.data_ptr() for x in grey])
    b.grey_m = arr(C.c_int, [int(x.shape[1]) for x in grey])
    b.grey_n = arr(C.c_int, [int(x.shape[0]) for x in grey])
    b.grey_sigma = arr(C.c_double, [float(v) for v in grey_sigma])
    b.grey_out = arr(C.c_void_p, [u.data_ptr() for u in g_out])
    b.n_rgb = len(rgb)
    b.rgb = arr(C.c_void_p, [p.data_ptr() for t in rgb for p in t])
    b.rgb_m = arr(C.c_int, [int(t[0].shape[1]) for t in rgb])
    b.rgb_n = arr(C.c_int, [int(t[0].shape[0]) for t in rgb])
    b.rgb_sigma = arr(C.c_double, [float(v) for v in rgb_sigma])
    b.rgb_out = arr(C.c_void_p, [p.data_ptr() for t in c_out for p in t])
    if video is not None:
        b.video = video.data_ptr()
        b.video_frames, b.video_n, b.video_m = (int(x) for x in video.shape)
        b.video_sigma = float(video_sigma)
        b.video_out = v_out.data_ptr()
    if len(grey_sigma) != len(grey) or len(rgb_sigma) != len(rgb):
        raise GBM3DError(1, "one sigma per image")

    def per_image(optlist, shapes, sigmas):
        if optlist is None:
            return None
        if len(optlist) != len(shapes):
            raise GBM3DError(1, "one option set per image")
        a = (gbm3d_opts * max(len(optlist), 1))()
        for k, (d, sh, sg) in enumerate(zip(optlist, shapes, sigmas)):
            a[k] = c_opts(_opt.resolve_opts(d, shape=sh, sigma=sg))
        keep.append(a)
        return C.cast(a, C.c_void_p)

    b.grey_opts = per_image(grey_opts, [(int(x.shape[1]), int(x.shape[0])) for x in grey], grey_sigma)
    b.rgb_opts = per_image(rgb_opts, [(int(t[0].shape[1]), int(t[0].shape[0])) for t in rgb], rgb_sigma)
    torch.cuda.synchronize()
    ctx.check(lib().gbm3d_denoise_mixed(ctx.h, C.byref(b), C.byref(o), C.byref(cv) if cv is not None else None,
                                        1 if use_graph else 0))
    ctx.check(lib().gbm3d_ctx_synchronize(ctx.h))
    return outputs


# ---- video ------------------------------------------------------------------------

def video_opts(opts: dict | None = None) -> dict:
    """The defaults of VBM3D.m:8-20 (blockSize 32, numMax = numMin = 16, the
    sym4 x Haar bank, levels 3, cycleSpin 2, matchSpins [0, d/2], tauMode 2,
    nF 11) for the fields opts does not set."""
    o = dict(opts or {})
    o.setdefault("blockSize", 32)
    o.setdefault("numMax", 16)
    o.setdefault("numMin", 16)
    o.setdefault("wname", "sym")
    o.setdefault("levels", 3)
    o.setdefault("cycleSpin", 2)
    o.setdefault("matchSpins", [0, int(o["blockSize"]) // 2])
    o.setdefault("tauMode", 2)
    o.setdefault("nF", 11)
    return o


def c_video_opts(opts: dict) -> gbm3d_opts:
    o = video_opts(opts)
    if o.get("wname") not in ("sym",) or o.get("wnamez", "db") != "db" or int(o.get("order", 4)) != 4 \
            or int(o.get("orderz", 1)) != 1:
        raise GBM3DError(5, "the video path's bank is getWaveFilters3D('sym','db',4,1)")
    if o.get("wiener", False):
        raise GBM3DError(5, "VBM3D has no Wiener step")
    c = gbm3d_opts()
    c.numMax, c.numMin = int(o["numMax"]), int(o["numMin"])
    c.blockSize = c.blockSizeWie = int(o["blockSize"])
    c.matchSize = 2 * int(o["blockSize"])
    c.levels, c.cycleSpin, c.tauMode = int(o["levels"]), int(o["cycleSpin"]), int(o["tauMode"])
    ms = list(o["matchSpins"])
    if len(ms) > 8:
        raise GBM3DError(1, "at most 8 match spins")
    c.nMatchSpins = c.nMatchSpinsWie = len(ms)
    for i, v in enumerate(ms):
        c.matchSpins[i] = c.matchSpinsWie[i] = int(v)
    c.staleWeights = 1
    c.wavelet = 2
    c.videoFrames = int(o["nF"])
    return c


def VBM3D(I, sigma, opts: dict | None = None, ctx: Context | None = None):
    """[Y, out] = VBM3D(I, sigma, opts): frames I (m x n x K, values in [0,1]);
    Y holds frames (nF+1)/2 .. K-(nF-1)/2 (1-based), the ones with a full
    temporal window (VBM3D.m:44-63)."""
    import torch
    ctx = ctx or context()
    co = c_video_opts(opts)
    I = np.asfortranarray(I, dtype=np.float64)
    if I.ndim != 3:
        raise GBM3DError(1, "VBM3D takes an m x n x frames array")
    m, n, Kf = I.shape
    nF = co.videoFrames
    if Kf < nF:
        raise GBM3DError(1, "fewer frames than the temporal window")
    dev = torch.device("cuda", ctx.device)
    dI = torch.from_numpy(I.ravel(order="F").copy()).to(dev)
    dY = torch.empty(m * n * (Kf - nF + 1), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    ctx.check(lib().gbm3d_vbm3d_device(ctx.h, C.c_void_p(dI.data_ptr()), m, n, Kf, float(sigma), C.byref(co),
                                       C.c_void_p(dY.data_ptr())))
    ctx.check(lib().gbm3d_ctx_synchronize(ctx.h))
    return dY.cpu().numpy().reshape(m, n, Kf - nF + 1, order="F"), {"frames": (nF + 1) // 2 - 1 + np.arange(Kf - nF + 1)}


def matchBlocksV(I, sigma, opts: dict | None = None, ctx: Context | None = None):
    """[S, Volume] = matchBlocksV(I, sigma, opts): I is m x n x F (F odd);
    S (K x M x N) indexes the d x d x F candidate window (1-based), Volume is
    m x n x K single."""
    ctx = ctx or context()
    co = c_video_opts(opts)
    I = np.asfortranarray(I, dtype=np.float64)
    m, n, F = I.shape
    if F % 2 != 1:
        raise GBM3DError(1, "input volume should have odd number of frames")  # matchBlocksV.m:24
    d, K = co.blockSize, co.numMax
    M, N = m // d, n // d
    S = np.zeros((K, M, N), dtype=np.uint32, order="F")
    V = np.zeros((m, n, K), dtype=np.float32, order="F")
    ctx.check(lib().gbm3d_matchBlocksV(ctx.h, _p(I), m, n, F, C.byref(co), _p(S), _p(V)))
    return _as_set(S), V


def denoiseAndAggregateV(Y, Volume, I, S, sigma, opts: dict | None = None, ctx: Context | None = None):
    """[U, out] = denoiseAndAggregateV(Y, Volume, I, S, sigma, opts): U and
    out['K'] are (M d) x (N d) x F double (F = frames of I); Y is unused, as in
    the reference."""
    ctx = ctx or context()
    o = video_opts(opts)
    co = c_video_opts(o)
    d = co.blockSize
    F = np.shape(I)[2]
    K, M, N = np.shape(S)
    Volume = np.asfortranarray(Volume, dtype=np.float32)
    if Volume.shape[2] != K or Volume.shape[0] < M * d or Volume.shape[1] < N * d:
        raise GBM3DError(1, "Volume does not match S")
    Volume = np.asfortranarray(Volume[: M * d, : N * d, :])
    Sa = np.asfortranarray(S, dtype=np.uint32)
    tau = np.asfortranarray(float(sigma) * _opt.getTau(int(o["levels"]), int(o["tauMode"])))
    U = np.zeros((M * d, N * d, F), order="F")
    W = np.zeros_like(U)
    ctx.check(lib().gbm3d_denoiseAndAggregateV(ctx.h, _p(Volume), _p(Sa), M, N, F, _p(tau), None, C.byref(co),
                                               _p(U), _p(W)))
    return U, {"K": W}
