"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the CPU-baseline legs of bench.py
import this module, to check results against or as the timed CPU baseline.  The product
(gbm3d_b200) never imports it.

The functions mirror the MATLAB reference's signatures (toby-sanders/GBM3D):

  matchBlocksCPU(I, sigma, opts)                -> S, Volume   source/matchBlocksCPU.m:1
  denoiseAndAggregateGPU(Volume, S, tau, opts)  -> U, W        source/denoiseAndAggregateGPU.m:1
  matchBlocksWie(I, In, sigma, opts)            -> S, V1, V2   source/matchBlocksWie.m:1
  denoiseAndAggregateWieFast(V1, V2, S, sigma, opts) -> U, W   source/denoiseAndAggregateWieFast.m:1
  GBM3D(I, sigma, opts)                         -> U, U1       source/GBM3D.m:1

``prec=32`` runs the FP32 mode whose operation order the CUDA kernels follow
(the parity target, bit-identical); ``prec=64`` runs the same code in FP64.

PARITY UNPINNED: the reference is MATLAB-only and ships no golden vectors;
see the header of oracle/gbm3d_oracle.cpp for how the restatement is checked.

Arrays use MATLAB's column-major layout (numpy order='F').  S is returned as a
uint32 array of shape (K, M, N): S[:, i, j] is the cell S{i+1, j+1}.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")


class orc_filters(C.Structure):
    _fields_ = [
        ("len_xy", C.c_int),
        ("a_lo_xy", C.c_double * 16), ("a_hi_xy", C.c_double * 16),
        ("s_lo_xy", C.c_double * 16), ("s_hi_xy", C.c_double * 16),
        ("len_z", C.c_int),
        ("a_lo_z", C.c_double * 16), ("a_hi_z", C.c_double * 16),
        ("s_lo_z", C.c_double * 16), ("s_hi_z", C.c_double * 16),
    ]


class orc_opts(C.Structure):
    _fields_ = [
        ("numMax", C.c_int), ("numMin", C.c_int), ("blockSize", C.c_int),
        ("blockSizeWie", C.c_int), ("matchSize", C.c_int),
        ("levels", C.c_int), ("cycleSpin", C.c_int), ("tauMode", C.c_int), ("Wiener", C.c_int),
        ("nSpins", C.c_int), ("spins", C.c_int * 8),
        ("nSpinsWie", C.c_int), ("spinsWie", C.c_int * 8),
        ("staleWeights", C.c_int), ("filtType", C.c_int),
        ("refStride", C.c_int), ("refStrideWie", C.c_int), ("wavelet", C.c_int),
    ]


def build() -> None:
    """Compile the oracle with its Makefile (g++ + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _cpu_has_fma() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = set(line.split())
                    return "fma" in fl and "avx2" in fl
    except OSError:
        pass
    return False


_lib = None


def lib():
    global _lib
    if _lib is None:
        names = (["liboracle_fma.so"] if _cpu_has_fma() else []) + ["liboracle.so"]
        paths = [os.path.join(_BUILD, n) for n in names]
        if not any(os.path.exists(p) for p in paths):
            build()
        for p in paths:
            if os.path.exists(p):
                _lib = C.CDLL(p)
                break
        _lib.orc_num_threads.restype = C.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def bior_filters() -> orc_filters:
    f = orc_filters()
    lib().orc_bior_filters(C.byref(f))
    return f


def haar_filters() -> orc_filters:
    """3D Haar bank (spatial and slot axes), the 'Haar' option of the configs."""
    f = orc_filters()
    cc = np.sqrt(2.0) / 2
    f.len_xy = 2
    f.len_z = 2
    for pre in ("xy", "z"):
        getattr(f, "a_lo_" + pre)[0:2] = [cc, cc]
        getattr(f, "a_hi_" + pre)[0:2] = [-cc, cc]
        getattr(f, "s_lo_" + pre)[0:2] = [cc, cc]
        getattr(f, "s_hi_" + pre)[0:2] = [-cc, cc]
    return f


def get_tau(levels: int, mode: int = 1) -> np.ndarray:
    t = np.zeros((levels, 7), order="F")
    lib().orc_get_tau(levels, mode, _p(t))
    return t


def dct_matrices(d: int):
    T = np.zeros((d, d), order="F")
    Ti = np.zeros((d, d), order="F")
    lib().orc_dct_matrices(d, _p(T), _p(Ti))
    return T, Ti


def sine_window(d: int, lo: float, hi: float) -> np.ndarray:
    w = np.zeros((d, d), order="F")
    lib().orc_sine_window(d, C.c_double(lo), C.c_double(hi), _p(w))
    return w


def _stride(opts, key, d):
    s = opts.get(key)
    return int(s) if s else int(d)


def matchBlocksCPU(I, sigma, opts, prec=32):
    """refStride s (default blockSize): references at i*s; Volume is m x n x K
    for s = blockSize (the reference) and tile-space (M*d, N*d, K) otherwise."""
    I = np.asfortranarray(I, dtype=np.float64)
    m, n = I.shape
    d, d2, K = opts["blockSize"], opts["matchSize"], opts["numMax"]
    st = _stride(opts, "refStride", d)
    M, N = (m - d) // st + 1, (n - d) // st + 1
    S = np.zeros((K, M, N), dtype=np.uint32, order="F")
    cnt = np.zeros((M, N), dtype=np.int32, order="F")
    vshape = (m, n, K) if st == d else (M * d, N * d, K)
    Vol = np.zeros(vshape, dtype=np.float32 if prec == 32 else np.float64, order="F")
    lib().orc_match_blocks(prec, _p(I), m, n, C.c_double(sigma), d, d2, K, opts["numMin"],
                           _p(S), _p(cnt), _p(Vol), st)
    return S, Vol, cnt


def matchBlocksWie(I, In, sigma, opts, prec=32):
    I = np.asfortranarray(I, dtype=np.float64)
    In = np.asfortranarray(In, dtype=np.float64)
    m, n = I.shape
    d, d2, K = opts["blockSizeWie"], opts["matchSize"], opts["numMax"]
    st = _stride(opts, "refStrideWie", d)
    M, N = (m - d) // st + 1, (n - d) // st + 1
    S = np.zeros((K, M, N), dtype=np.uint32, order="F")
    dt = np.float32 if prec == 32 else np.float64
    V1 = np.zeros((d, d, K, M, N), dtype=dt, order="F")
    V2 = np.zeros_like(V1)
    lib().orc_match_blocks_wie(prec, _p(I), _p(In), m, n, d, d2, K, _p(S), _p(V1), _p(V2), st)
    return S, V1, V2


def denoiseAndAggregateGPU(Volume, S, tau, opts, cnt=None, filters=None, prec=32):
    dt = np.float32 if prec == 32 else np.float64
    Volume = np.asfortranarray(Volume, dtype=dt)
    K, M, N = S.shape
    d = opts["blockSize"]
    S = np.asfortranarray(S, dtype=np.uint32)
    tau = np.asfortranarray(tau, dtype=np.float64)
    f = filters if filters is not None else bior_filters()
    st = _stride(opts, "refStride", d)
    U = np.zeros(((M - 1) * st + d, (N - 1) * st + d), order="F")
    W = np.zeros_like(U)
    cp = None
    if cnt is not None:
        cnt = np.asfortranarray(cnt, dtype=np.int32)
        cp = _p(cnt)
    lib().orc_denoise_ht(prec, _p(Volume), M, N, d, opts["matchSize"], K, _p(S), cp,
                         opts["levels"], opts["cycleSpin"], _p(tau), C.byref(f), _p(U), _p(W), st)
    return U, W


def denoiseAndAggregateWieFast(V1, V2, S, sigma, opts, prec=32, variant=0):
    dt = np.float32 if prec == 32 else np.float64
    V1 = np.asfortranarray(V1, dtype=dt)
    V2 = np.asfortranarray(V2, dtype=dt)
    d, _, K, M, N = V1.shape
    S = np.asfortranarray(S, dtype=np.uint32)
    sg = np.asfortranarray(np.atleast_1d(np.asarray(sigma, dtype=np.float64)))
    is_mat = 1 if sg.size > 1 else 0
    st = _stride(opts, "refStrideWie", d)
    U = np.zeros(((M - 1) * st + d, (N - 1) * st + d), order="F")
    W = np.zeros_like(U)
    lib().orc_denoise_wiener(prec, _p(V1), _p(V2), M, N, d, opts["matchSize"], K, _p(S), _p(sg),
                             is_mat, variant, _p(U), _p(W), st)
    return U, W


def denoiseAndAggregateWie(V1, V2, S, sigma, opts, prec=32):
    """Legacy step-2 variant (source/denoiseAndAggregateWie.m:1)."""
    return denoiseAndAggregateWieFast(V1, V2, S, sigma, opts, prec=prec, variant=1)


def wavelet_ht(V, levels, tau, filters=None, prec=32):
    dt = np.float32 if prec == 32 else np.float64
    V = np.asfortranarray(V, dtype=dt)
    Ly, Lx, Lz = V.shape
    out = np.zeros_like(V)
    f = filters if filters is not None else bior_filters()
    tau = np.asfortranarray(tau, dtype=np.float64)
    lib().orc_wavelet_roundtrip(prec, _p(V), Ly, Lx, Lz, levels, _p(tau), C.byref(f), _p(out))
    return out


def make_opts(o: dict) -> orc_opts:
    c = orc_opts()
    for k in ("numMax", "numMin", "blockSize", "blockSizeWie", "matchSize", "levels",
              "cycleSpin", "tauMode"):
        setattr(c, k, int(o[k]))
    c.Wiener = 1 if o["Wiener"] else 0
    c.nSpins = len(o["matchSpins"])
    c.spins[: c.nSpins] = [int(s) for s in o["matchSpins"]]
    c.nSpinsWie = len(o["matchSpinsWie"])
    c.spinsWie[: c.nSpinsWie] = [int(s) for s in o["matchSpinsWie"]]
    c.staleWeights = 1 if o.get("staleWeights", True) else 0
    c.filtType = 1 if o.get("filtType", "ht") == "median" else 0
    c.refStride = int(o.get("refStride") or 0)
    c.refStrideWie = int(o.get("refStrideWie") or 0)
    c.wavelet = 1 if o.get("wname", "bior") == "haar" else 0
    return c


def GBM3D(I, sigma, opts, prec=32):
    I = np.asfortranarray(I, dtype=np.float64)
    m, n = I.shape
    U = np.zeros((m, n), order="F")
    U1 = np.zeros((m, n), order="F")
    oc = make_opts(opts)
    if lib().orc_gbm3d(prec, _p(I), m, n, C.c_double(sigma), C.byref(oc), _p(U), _p(U1)) != 0:
        raise ValueError("no padded size lets both reference grids end at the border")
    return U, U1


def GBM3D_colored(I, sigma_match, tau, sigmaWie, opts, prec=32):
    """GBM3D.m:33-35 for coloured noise: tau (levels x 7) and sigmaWie
    (blockSizeWie^2) given, sigma_match = mean(sqrt(sigmaPSD(:)))."""
    I = np.asfortranarray(I, dtype=np.float64)
    m, n = I.shape
    U = np.zeros((m, n), order="F")
    U1 = np.zeros((m, n), order="F")
    oc = make_opts(opts)
    tau = np.asfortranarray(tau, dtype=np.float64)
    sw = np.asfortranarray(sigmaWie, dtype=np.float64)
    if lib().orc_gbm3d_colored(prec, _p(I), m, n, C.c_double(sigma_match), _p(tau), _p(sw), C.byref(oc),
                               _p(U), _p(U1)) != 0:
        raise ValueError("no padded size lets both reference grids end at the border")
    return U, U1


def matchBlocksGPU(I, sigma, opts, prec=32):
    """S = matchBlocksGPU(I, sigma, opts) (source/matchBlocksGPU.m:1): global
    circular search; S indexes the m x n image.  Returns S, counts and the
    (prefiltered) image the search ran on."""
    I = np.asfortranarray(I, dtype=np.float64)
    m, n = I.shape
    d, K = opts["blockSize"], opts["numMax"]
    M, N = m // d, n // d
    S = np.zeros((K, M, N), dtype=np.uint32, order="F")
    cnt = np.zeros((M, N), dtype=np.int32, order="F")
    pre = np.zeros((m, n), order="F")
    lib().orc_match_blocks_global(prec, _p(I), m, n, C.c_double(sigma), d, K, opts["numMin"], _p(S), _p(cnt), _p(pre))
    return S, cnt, pre


def denoiseAndAggregateMedian(Volume, S, opts, cnt=None, prec=32):
    """denoiseAndAggregateGPU with opts.filtType = 'median' (medfilt3 instead of the wavelet)."""
    dt = np.float32 if prec == 32 else np.float64
    Volume = np.asfortranarray(Volume, dtype=dt)
    K, M, N = S.shape
    d = opts["blockSize"]
    S = np.asfortranarray(S, dtype=np.uint32)
    st = _stride(opts, "refStride", d)
    U = np.zeros(((M - 1) * st + d, (N - 1) * st + d), order="F")
    W = np.zeros_like(U)
    cp = None
    if cnt is not None:
        cnt = np.asfortranarray(cnt, dtype=np.int32)
        cp = _p(cnt)
    lib().orc_denoise_median(prec, _p(Volume), M, N, d, opts["matchSize"], K, _p(S), cp, _p(U), _p(W), st)
    return U, W


def medfilt3(V, prec=64):
    dt = np.float32 if prec == 32 else np.float64
    V = np.asfortranarray(V, dtype=dt)
    out = np.zeros_like(V)
    m, n, K = V.shape
    lib().orc_medfilt3(prec, _p(V), m, n, K, _p(out))
    return out


def sym4_haar_filters() -> orc_filters:
    """getWaveFilters3D('sym','db',4,1) (waveTransforms3D/getWaveFilters3D.m:6-33):
    sym4 decomposition filters on the spatial axes, db1 (Haar) on the slot
    axis; the video path synthesises with the same filters (Psi2 = Psi)."""
    from .fft_route import SYM4_HI, SYM4_LO
    f = orc_filters()
    cc = np.sqrt(2.0) / 2
    f.len_xy = 8
    f.len_z = 2
    for pre in ("a", "s"):
        getattr(f, pre + "_lo_xy")[0:8] = list(SYM4_LO)
        getattr(f, pre + "_hi_xy")[0:8] = list(SYM4_HI)
        getattr(f, pre + "_lo_z")[0:2] = [cc, cc]
        getattr(f, pre + "_hi_z")[0:2] = [-cc, cc]
    return f


def matchBlocksV(I, d, K, prec=32):
    """[S, Volume] = matchBlocksV(I, sigma, opts) (source/matchBlocksV.m), top-K branch."""
    I = np.asfortranarray(I, dtype=np.float64)
    m, n, F = I.shape
    M, N = m // d, n // d
    S = np.zeros((K, M, N), dtype=np.uint32, order="F")
    Vol = np.zeros((m, n, K), dtype=np.float32 if prec == 32 else np.float64, order="F")
    lib().orc_match_video(prec, _p(I), m, n, F, d, K, _p(S), _p(Vol))
    return S, Vol


def denoiseAndAggregateV(Volume, S, d, F, tau, levels, cycleSpin, filters=None, prec=32):
    """[U, out.K] of denoiseAndAggregateV.m (U, W: m x n x F, float64)."""
    f = filters if filters is not None else sym4_haar_filters()
    K, M, N = S.shape
    Volume = np.asfortranarray(Volume, dtype=np.float32 if prec == 32 else np.float64)
    S = np.asfortranarray(S, dtype=np.uint32)
    tau = np.asfortranarray(tau, dtype=np.float64)
    U = np.zeros((M * d, N * d, F), order="F")
    W = np.zeros_like(U)
    lib().orc_denoise_video(prec, _p(Volume), M, N, d, F, K, _p(S), levels, cycleSpin, _p(tau), C.byref(f), _p(U),
                            _p(W))
    return U, W


def VBM3D(I, sigma, d=8, K=16, levels=3, cycleSpin=2, tauMode=2, spins=(0, 4), nF=3, filters=None, prec=32):
    """Y = VBM3D(I, sigma, opts) (source/VBM3D.m): frames I m x n x Kf on the
    reference's [0,1] scale; returns frames (nF-1)/2 .. Kf-1-(nF-1)/2."""
    f = filters if filters is not None else sym4_haar_filters()
    I = np.asfortranarray(I, dtype=np.float64)
    m, n, Kf = I.shape
    out = np.zeros((m, n, Kf - nF + 1), order="F")
    sp = np.ascontiguousarray(spins, dtype=np.int32)
    if lib().orc_vbm3d(prec, _p(I), m, n, Kf, C.c_double(sigma), d, K, levels, cycleSpin, tauMode, _p(sp), len(sp),
                       nF, C.byref(f), _p(out)) != 0:
        raise ValueError("nF must be odd and at most the number of frames")
    return out
