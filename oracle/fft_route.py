"""Second restatement of the reference, along its FFT route — TEST INFRASTRUCTURE ONLY.

Where oracle/gbm3d_oracle.cpp computes every circular convolution and block
distance directly, this module follows the MATLAB code of toby-sanders/GBM3D
operation by operation: distances through fft2 cross-correlation and block-norm
maps, wavelets through fftn products with zero-padded 3D filters, the 1D Haar
through fft along the slot axis, aggregation through the same nested loops.
It runs in float64 on small images and generates the committed golden vectors
under tests/golden/ (script: tests/golden/make_golden.py).  Two restatements
that reach the same numbers by different arithmetic pin each other; neither is
the reference itself, which needs MATLAB.
"""
from __future__ import annotations

import numpy as np


def _circshift(a, shifts):
    return np.roll(a, shifts, axis=tuple(range(len(shifts))))


def _pad_to(h, shape):
    """fftn(h, shape): zero-pad (or truncate) each axis to shape."""
    out = np.zeros(shape)
    sl = tuple(slice(0, min(a, b)) for a, b in zip(h.shape, shape))
    out[sl] = h[sl]
    return out


def _search_pad(I, d2):
    """Ipad: 2x2 tiling cropped to (m+d2) x (n+d2), circshift by d2/2 (matchBlocksCPU.m:57-61)."""
    m, n = I.shape
    T = np.zeros((2 * m, 2 * n))
    T[:m, :n] = I
    T[:m, n:] = I
    T[m:, :n] = I
    T[m:, n:] = I
    return _circshift(T[: m + d2, : n + d2], (d2 // 2, d2 // 2))


def _block_norms(X, d, shape):
    """real(ifft2(conj(fft2(ones(d), shape)) .* fft2(X.^2)))."""
    g = _pad_to(np.ones((d, d)), shape)
    return np.real(np.fft.ifft2(np.conj(np.fft.fft2(g)) * np.fft.fft2(X ** 2)))


def match_blocks(I, d, d2, K, In=None, st=None):
    """matchBlocksCPU.m:21-116 (top-K branch) / matchBlocksWie.m:21-92.

    Returns S (K, M, N) uint32, Volume (m, n, K) and, with In, V1/V2 (d,d,K,M,N).
    st: reference stride (default d, the reference's tiling); with st != d the
    references sit at i*st, M = (m-d)//st + 1 and Volume is (M d, N d, K).
    """
    I = np.asarray(I, dtype=np.float64)
    m, n = I.shape
    st = st or d
    M, N = (m - d) // st + 1, (n - d) // st + 1
    h = d2 // 2
    Ipad = _search_pad(I, d2)
    Ipad2 = _search_pad(np.asarray(In, dtype=np.float64), d2) if In is not None else None
    bn = _block_norms(I, d, (m, n))
    bnp = _block_norms(Ipad, d, (m + d2, n + d2))
    S = np.zeros((K, M, N), dtype=np.uint32)
    Vol = np.zeros((m, n, K) if st == d else (M * d, N * d, K))
    V1 = np.zeros((d, d, K, M, N)) if In is not None else None
    V2 = np.zeros_like(V1) if In is not None else None
    for i in range(M):
        for j in range(N):
            y0, x0 = i * st, j * st
            xR = I[y0:y0 + d, x0:x0 + d]
            It = Ipad[y0:y0 + d + d2, x0:x0 + d + d2]
            cc = np.real(np.fft.ifft2(np.conj(np.fft.fft2(_pad_to(xR, (d + d2, d + d2)))) * np.fft.fft2(It)))
            nr = bn[y0, x0]
            D = (nr + bnp[y0:y0 + d2, x0:x0 + d2] - 2 * cc[:d2, :d2]) / nr
            idx = np.argsort(D.ravel(order="F"), kind="stable")[:K]  # mink
            s = (idx + 1).astype(np.uint32)
            s[0] = d2 * d2 // 2 + h + 1
            S[:, i, j] = s
            for k in range(K):
                a, b = (int(s[k]) - 1) % d2, (int(s[k]) - 1) // d2
                Vol[i * d:(i + 1) * d, j * d:(j + 1) * d, k] = It[a:a + d, b:b + d]
                if In is not None:
                    V1[:, :, k, i, j] = It[a:a + d, b:b + d]
                    V2[:, :, k, i, j] = Ipad2[y0:y0 + d + d2, x0:x0 + d + d2][a:a + d, b:b + d]
    return S, Vol, V1, V2


def wav_dec3(Psi, levels, U):
    """myWavDec3DFFT.m:10-23."""
    C = {}
    for i in range(levels):
        FU = np.fft.fftn(U)
        for j in range(7):
            c = np.fft.ifftn(FU * np.fft.fftn(_pad_to(Psi[..., j + 1], U.shape)))
            C[i, j] = np.real(c[::2, ::2, ::2])
        U = np.real(np.fft.ifftn(FU * np.fft.fftn(_pad_to(Psi[..., 0], U.shape))))[::2, ::2, ::2]
    C[levels, 0] = U
    return C


def wav_rec3(Psi2, levels, C):
    """myWavRec3DGPUfast.m:10-40."""
    Cup = {}
    for i in range(levels):
        sh = tuple(2 * s for s in C[i, 0].shape)
        acc = np.zeros(sh)
        for j in range(7):
            tmp = np.zeros(sh)
            tmp[::2, ::2, ::2] = C[i, j]
            acc += np.real(np.fft.ifftn(np.fft.fftn(tmp) * np.conj(np.fft.fftn(_pad_to(Psi2[..., j + 1], sh)))))
        Cup[i] = acc
    Cup[levels] = C[levels, 0]
    for i in range(levels, 0, -1):
        sh = Cup[i - 1].shape
        tmp = np.zeros(sh)
        tmp[::2, ::2, ::2] = Cup[i]
        Cup[i - 1] = Cup[i - 1] + np.real(np.fft.ifftn(np.fft.fftn(tmp) * np.conj(np.fft.fftn(_pad_to(Psi2[..., 0], sh)))))
    return Cup[0]


def agg_weight(B):
    """getBM3DAggWeights(3,1) (getBM3DAggWeights.m:11-19)."""
    w = np.sum(np.abs(np.diff(B, 3, axis=1))) * 2.0 ** -2
    w += np.sum(np.abs(np.diff(B, 3, axis=0))) * 2.0 ** -2
    w += np.sum(np.abs(np.diff(B, 1, axis=2))) * 1.0
    return w


def sine_window(d, lo, hi):
    v = np.sin(np.pi * np.linspace(lo, hi, d))
    return np.outer(v, v)


def denoise_ht(Volume, S, tau, Psi, Psi2, d, d2, levels, cycle_spin, st=None):
    """denoiseAndAggregateGPU.m:11-92 (filtType 'ht'); st: reference stride
    (Volume is (M d, N d, K); output ((M-1) st + d, (N-1) st + d))."""
    K, M, N = S.shape
    st = st or d
    m, n = M * d, N * d
    Vrec = np.zeros((m, n, K, cycle_spin))
    for spin in range(cycle_spin):
        V = _circshift(Volume, (spin, spin, spin))
        C = wav_dec3(Psi, levels, V)
        for i in range(levels):
            for j in range(7):
                C[i, j] = C[i, j] * (np.abs(C[i, j]) > tau[i, j])
        Vrec[..., spin] = _circshift(wav_rec3(Psi2, levels, C), (-spin, -spin, -spin))
    Vavg = np.maximum(Vrec.mean(axis=3), 0)
    mo, no = (M - 1) * st + d, (N - 1) * st + d
    U = np.zeros((mo + d2, no + d2))
    W = np.zeros_like(U)
    mask = sine_window(d, 0.1, 0.9)
    for y in range(M):
        for x in range(N):
            blocks = Vavg[y * d:(y + 1) * d, x * d:(x + 1) * d, :K]
            wt = 1.0 / (agg_weight(blocks) + np.finfo(float).eps)
            for i in range(K):
                a, b = (int(S[i, y, x]) - 1) % d2 + y * st, (int(S[i, y, x]) - 1) // d2 + x * st
                U[a:a + d, b:b + d] += wt * blocks[:, :, i] * mask
                W[a:a + d, b:b + d] += wt * mask
    h = d2 // 2
    return U[h:mo + h, h:no + h], W[h:mo + h, h:no + h]


def _dec1d(Psi, Phi, levels, U):
    """myWavDec1D.m:10-26 along axis 2 (slots)."""
    r = U.shape[2]
    C = np.zeros_like(U)
    cnt = 0
    for _ in range(levels):
        L = U.shape[2]
        FU = np.fft.fft(U, axis=2)
        shp = [1, 1, L] + [1] * (U.ndim - 3)
        hp = np.zeros(L); hp[:2] = Psi
        lp = np.zeros(L); lp[:2] = Phi
        dd = np.real(np.fft.ifft(FU * np.fft.fft(hp).reshape(shp), axis=2))
        C[:, :, cnt:cnt + L // 2] = dd[:, :, ::2]
        cnt += L // 2
        U = np.real(np.fft.ifft(FU * np.fft.fft(lp).reshape(shp), axis=2))[:, :, ::2]
    C[:, :, cnt:r] = U
    return C


def _rec1d(Psi, Phi, levels, C):
    """myWavRec1D.m:6-26 along axis 2."""
    r = C.shape[2]
    Cup = {}
    cnt = 0
    for i in range(levels):
        L = r // 2 ** i
        up = np.zeros(C.shape[:2] + (L,) + C.shape[3:])
        up[:, :, ::2] = C[:, :, cnt:cnt + r // 2 ** (i + 1)]
        cnt += r // 2 ** (i + 1)
        hp = np.zeros(L); hp[:2] = Psi
        shp = [1, 1, L] + [1] * (C.ndim - 3)
        Cup[i] = np.real(np.fft.ifft(np.fft.fft(up, axis=2) * np.conj(np.fft.fft(hp)).reshape(shp), axis=2))
    Cup[levels] = C[:, :, cnt:]
    for i in range(levels, 0, -1):
        L = Cup[i - 1].shape[2]
        up = np.zeros(Cup[i - 1].shape)
        up[:, :, ::2] = Cup[i]
        lp = np.zeros(L); lp[:2] = Phi
        shp = [1, 1, L] + [1] * (C.ndim - 3)
        Cup[i - 1] = Cup[i - 1] + np.real(np.fft.ifft(np.fft.fft(up, axis=2) * np.conj(np.fft.fft(lp)).reshape(shp), axis=2))
    return Cup[0]


def dct_matrix(d):
    k = np.arange(d)[:, None]
    nn = np.arange(d)[None, :]
    T = np.sqrt(2.0 / d) * np.cos(np.pi * (2 * nn + 1) * k / (2 * d))
    T[0, :] = np.sqrt(1.0 / d)
    return T


def denoise_wiener(V1, V2, S, sigma, d2, variant=0, st=None):
    """denoiseAndAggregateWieFast.m:23-100 (variant 0) / denoiseAndAggregateWie.m (variant 1)."""
    d, _, K, M, N = V1.shape
    st = st or d
    m, n = (M - 1) * st + d, (N - 1) * st + d
    levels = 2 if K < 16 else 3
    cc = np.sqrt(2.0) / 2
    Psi, Phi = np.array([-cc, cc]), np.array([cc, cc])
    T = dct_matrix(d)
    Ti = np.linalg.inv(T) if variant == 0 else T.T
    A = np.einsum("ij,jlkmn,ql->iqkmn", T, V1, T)
    A = _dec1d(Psi, Phi, levels, A)
    s2 = np.asarray(sigma, dtype=np.float64) ** 2
    if s2.ndim == 2:
        s2 = s2[:, :, None, None, None]
    filt = np.abs(A) ** 2 / (np.abs(A) ** 2 + s2)
    filt[0, 0, 14:] = 1
    B = np.einsum("ij,jlkmn,ql->iqkmn", T, V2, T)
    B = _dec1d(Psi, Phi, levels, B) * filt
    B = _rec1d(Psi, Phi, levels, B)
    B = np.einsum("ij,jlkmn,ql->iqkmn", Ti, B, Ti)
    B = np.maximum(B, 0)
    if variant == 1:
        B = np.minimum(B, 1)
    U = np.zeros((m + d2, n + d2))
    W = np.zeros_like(U)
    w = sine_window(d, 0.2, 0.8)
    for y in range(M):
        for x in range(N):
            wt = w / np.linalg.norm(filt[:, :, :, y, x].ravel()) ** 2
            for i in range(K):
                a, b = (int(S[i, y, x]) - 1) % d2 + y * st, (int(S[i, y, x]) - 1) // d2 + x * st
                U[a:a + d, b:b + d] += wt * B[:, :, i, y, x]
                W[a:a + d, b:b + d] += wt
    h = d2 // 2
    return U[h:m + h, h:n + h], W[h:m + h, h:n + h]


def padded_size(L, opts):
    """GBM3D.m:21-25 pads to a multiple of blockSize; with other strides, to the
    smallest size at which both steps' references end exactly at the border."""
    import math
    d, dw = opts["blockSize"], opts["blockSizeWie"]
    st1, st2 = opts.get("refStride") or d, opts.get("refStrideWie") or dw
    if st1 == d and (not opts["Wiener"] or (st2 == dw and d % dw == 0)):
        return -(-L // d) * d
    if opts["Wiener"] and (d - dw) % math.gcd(st1, st2):
        raise ValueError("no padded size lets both reference grids end at the border")
    p = max(L, d, dw)
    while (p - d) % st1 or (opts["Wiener"] and (p - dw) % st2):
        p += 1
    return p


def gbm3d(I, sigma, opts, Psi, Psi2, tau_unit):
    """GBM3D.m:15-83 for a scalar sigma; opts as gbm3d_b200.options dicts."""
    I = np.asarray(I, dtype=np.float64)
    m, n = I.shape
    d, dw, d2, K = opts["blockSize"], opts["blockSizeWie"], opts["matchSize"], opts["numMax"]
    st1, st2 = opts.get("refStride") or d, opts.get("refStrideWie") or dw
    Mp, Np = padded_size(m, opts), padded_size(n, opts)
    Ip = np.zeros((Mp, Np))
    Ip[:m, :n] = I
    Ip[m:, :n] = np.flipud(I[m - (Mp - m):m, :n])
    Ip[:m, n:] = np.fliplr(I[:m, n - (Np - n):n])
    Ip[m:, n:] = np.fliplr(np.flipud(I[m - (Mp - m):m, n - (Np - n):n]))
    tau = sigma * tau_unit
    nS, nW = len(opts["matchSpins"]), len(opts["matchSpinsWie"])
    U1s = np.zeros((Mp, Np, nS))
    Ws = np.zeros((Mp, Np, max(nS, nW)))
    for ii, s in enumerate(opts["matchSpins"]):
        S, Vol, _, _ = match_blocks(_circshift(Ip, (s, s)), d, d2, K, st=st1)
        u, w = denoise_ht(Vol, S, tau, Psi, Psi2, d, d2, opts["levels"], opts["cycleSpin"], st=st1)
        U1s[..., ii] = _circshift(u, (-s, -s))
        Ws[..., ii] = _circshift(w, (-s, -s))
    U1 = U1s.sum(axis=2) / Ws[..., :nS].sum(axis=2)
    if not opts["Wiener"]:
        return U1[:m, :n], U1[:m, :n]
    Us = np.zeros((Mp, Np, max(nS, nW)))
    for ii, s in enumerate(opts["matchSpinsWie"]):
        S, _, V1, V2 = match_blocks(_circshift(U1, (s, s)), dw, d2, K, In=_circshift(Ip, (s, s)), st=st2)
        u, w = denoise_wiener(V1, V2, S, sigma, d2, st=st2)
        Us[..., ii] = _circshift(u, (-s, -s))
        Ws[..., ii] = _circshift(w, (-s, -s))
    U = Us.sum(axis=2) / Ws.sum(axis=2)
    return U[:m, :n], U1[:m, :n]


SYM4_LO = np.array([-0.07576571478927333, -0.02963552764599851, 0.49761866763201545, 0.8037387518059161,
                    0.29785779560527736, -0.09921954357684722, -0.012603967262037833, 0.0322231006040427])
SYM4_HI = np.array([-0.0322231006040427, -0.012603967262037833, 0.09921954357684722, 0.29785779560527736,
                    -0.8037387518059161, 0.49761866763201545, 0.02963552764599851, -0.07576571478927333])


def sym4_bank():
    """getWaveFilters2D('sym',4): Psi(:,:,1..4) = Lo'Lo, Hi'Lo, Lo'Hi, Hi'Hi."""
    lo, hi = SYM4_LO, SYM4_HI
    return np.stack([np.outer(lo, lo), np.outer(hi, lo), np.outer(lo, hi), np.outer(hi, hi)], -1)


def wav_dec2(Psi, levels, U):
    """myWavDec2DFFT.m:10-23."""
    C = {}
    for i in range(levels):
        FU = np.fft.fft2(U)
        for j in range(3):
            C[i, j] = np.real(np.fft.ifft2(FU * np.fft.fft2(_pad_to(Psi[..., j + 1], U.shape))))[::2, ::2]
        U = np.real(np.fft.ifft2(FU * np.fft.fft2(_pad_to(Psi[..., 0], U.shape))))[::2, ::2]
    C[levels, 0] = U
    return C


def wav_rec2(Psi, levels, C):
    """myWavRec2DGPUfast.m:10-34."""
    Cup = {}
    for i in range(levels):
        sh = tuple(2 * s for s in C[i, 0].shape)
        acc = np.zeros(sh)
        for j in range(3):
            tmp = np.zeros(sh)
            tmp[::2, ::2] = C[i, j]
            acc += np.real(np.fft.ifft2(np.fft.fft2(tmp) * np.conj(np.fft.fft2(_pad_to(Psi[..., j + 1], sh)))))
        Cup[i] = acc
    Cup[levels] = C[levels, 0]
    for i in range(levels, 0, -1):
        sh = Cup[i - 1].shape
        tmp = np.zeros(sh)
        tmp[::2, ::2] = Cup[i]
        Cup[i - 1] = Cup[i - 1] + np.real(np.fft.ifft2(np.fft.fft2(tmp) * np.conj(np.fft.fft2(_pad_to(Psi[..., 0], sh)))))
    return Cup[0]


def match_blocks_global(I, sigma, d, K):
    """matchBlocksGPU.m:19-91 (top-K branch); returns S (K, M, N) and the searched image."""
    I = np.asarray(I, dtype=np.float64)
    m, n = I.shape
    M, N = m // d, n // d
    if sigma > 30 / 255:
        Psi = sym4_bank()
        avg = np.zeros_like(I)
        for k in range(1, 6):
            C = wav_dec2(Psi, 3, _circshift(I, (k - 1, k - 1)))
            for i in range(3):
                for j in range(3):
                    C[i, j] = C[i, j] * (np.abs(C[i, j]) > 2 * sigma)
            avg = avg + _circshift(wav_rec2(Psi, 3, C), (1 - k, 1 - k)) / 5
        I = avg
    g = _pad_to(np.ones((d, d)), (m, n))
    bn = np.real(_circshift(np.fft.ifft2(np.fft.fft2(g) * np.fft.fft2(I ** 2)), (-d + 1, -d + 1)))
    FI = np.fft.fft2(I)
    S = np.zeros((K, M, N), dtype=np.uint32)
    for i in range(M):
        for j in range(N):
            xR = I[i * d:(i + 1) * d, j * d:(j + 1) * d]
            cc = np.real(np.fft.ifft2(np.conj(np.fft.fft2(_pad_to(xR, (m, n)))) * FI))
            nr = bn[i * d, j * d]
            D = (nr + bn - 2 * cc) / nr
            S[:, i, j] = np.argsort(D.ravel(order="F"), kind="stable")[:K] + 1
    return S, I


def match_blocks_video(I, d, K):
    """matchBlocksV.m:21-116 (top-K branch): I is m x n x F (F odd); FFT route
    for the distances of every d x d offset in every frame of the 2d x 2d
    window.  Returns S (K, M, N) and Volume (m, n, K)."""
    I = np.asarray(I, dtype=np.float64)
    m, n, F = I.shape
    ref = (F - 1) // 2
    M, N = m // d, n // d
    T = np.zeros((2 * m, 2 * n, F))
    T[:m, :n], T[:m, n:], T[m:, :n], T[m:, n:] = I, I, I, I
    Ipad = np.roll(T[: m + d, : n + d], (d // 2, d // 2), axis=(0, 1))
    g = np.zeros((m, n))
    g[:d, :d] = 1
    bn = np.real(np.fft.ifft2(np.conj(np.fft.fft2(g))[..., None] * np.fft.fft2(I ** 2, axes=(0, 1)), axes=(0, 1)))
    gp = np.zeros((m + d, n + d))
    gp[:d, :d] = 1
    bnp = np.real(np.fft.ifft2(np.conj(np.fft.fft2(gp))[..., None] * np.fft.fft2(Ipad ** 2, axes=(0, 1)),
                               axes=(0, 1)))
    S = np.zeros((K, M, N), dtype=np.uint32)
    Vol = np.zeros((m, n, K))
    for i in range(M):
        for j in range(N):
            xR = I[i * d:(i + 1) * d, j * d:(j + 1) * d, ref]
            It = Ipad[i * d:(i + 2) * d, j * d:(j + 2) * d, :]
            xz = np.zeros((2 * d, 2 * d))
            xz[:d, :d] = xR
            cc = np.real(np.fft.ifft2(np.conj(np.fft.fft2(xz))[..., None] * np.fft.fft2(It, axes=(0, 1)), axes=(0, 1)))
            nr = bn[i * d, j * d, ref]
            D = (nr + bnp[i * d:(i + 1) * d, j * d:(j + 1) * d, :] - 2 * cc[:d, :d, :]) / nr
            idx = np.argsort(D.ravel(order="F"), kind="stable")[:K]
            s = (idx + 1).astype(np.uint32)
            s[0] = d * d * F // 2 + d // 2 + 1
            S[:, i, j] = s
            for k in range(K):
                e = int(s[k]) - 1
                a, b, c = e % d, (e // d) % d, e // (d * d)
                Vol[i * d:(i + 1) * d, j * d:(j + 1) * d, k] = It[a:a + d, b:b + d, c]
    return S, Vol


def denoise_video(Volume, S, tau, Psi, Psi2, d, F, levels, cycle_spin):
    """denoiseAndAggregateV.m:11-89."""
    K, M, N = S.shape
    m, n = M * d, N * d
    Vrec = np.zeros((m, n, K, cycle_spin))
    for spin in range(cycle_spin):
        V = _circshift(Volume, (spin, spin, spin))
        C = wav_dec3(Psi, levels, V)
        for i in range(levels):
            for j in range(7):
                C[i, j] = C[i, j] * (np.abs(C[i, j]) > tau[i, j])
        Vrec[..., spin] = _circshift(wav_rec3(Psi2, levels, C), (-spin, -spin, -spin))
    Vavg = np.minimum(np.maximum(Vrec.mean(axis=3), 0), 1)
    U = np.zeros((m + d, n + d, F))
    W = np.zeros_like(U)
    for y in range(M):
        for x in range(N):
            blocks = Vavg[y * d:(y + 1) * d, x * d:(x + 1) * d, :K]
            wt = 1.0 / agg_weight(blocks)
            for i in range(K):
                e = int(S[i, y, x]) - 1
                a, b, c = e % d + y * d - d // 2, (e // d) % d + x * d - d // 2, e // (d * d)
                if a >= 0 and b >= 0:
                    U[a:a + d, b:b + d, c] += wt * blocks[:, :, i]
                    W[a:a + d, b:b + d, c] += wt
    return U[:m, :n], W[:m, :n]


def vbm3d(I, sigma, d, K, levels, cycle_spin, tau_unit, spins, nF, Psi, Psi2):
    """VBM3D.m:20-63 (frames already in the reference's [0,1] scale)."""
    I = np.asarray(I, dtype=np.float64)
    m, n, Kf = I.shape
    Mp, Np = -(-m // d) * d, -(-n // d) * d
    I2 = np.zeros((Mp, Np, Kf))
    I2[:m, :n] = I
    I2[m:, :n] = np.flipud(I[m - (Mp - m):m, :n])
    I2[:m, n:] = np.fliplr(I[:m, n - (Np - n):n])
    I2[m:, n:] = np.fliplr(np.flipud(I[m - (Mp - m):m, n - (Np - n):n]))
    hw = (nF - 1) // 2
    Y = np.zeros((Mp, Np, Kf, len(spins)))
    for ii, s in enumerate(spins):
        nn = np.zeros((Mp, Np, Kf))
        for jj in range(hw, Kf - hw):
            ind = slice(jj - hw, jj + hw + 1)
            I3 = np.roll(I2[:, :, ind], (s, s), axis=(0, 1))
            S, Vol = match_blocks_video(I3, d, K)
            U, W = denoise_video(Vol, S, sigma * tau_unit, Psi, Psi2, d, nF, levels, cycle_spin)
            Y[:, :, ind, ii] += U
            nn[:, :, ind] += W
        Y[:, :, :, ii] = np.roll(Y[:, :, :, ii] / nn, (-s, -s), axis=(0, 1))
    return Y[:m, :n, hw:Kf - hw].mean(axis=3)
