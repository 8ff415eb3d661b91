"""Option profiles, thresholds, filter banks and small image utilities.

Host-side mirror of the reference's utility layer (toby-sanders/GBM3D):

  setBM3Dopts(profile)   utilities/setBM3Dopts.m:1-86
  checkBM3Dopts(opts)    utilities/checkBM3Dopts.m:10-24
  getTau(levels, mode)   utilities/getTau.m:9-51
  getWaveFilters3Dbior() waveTransforms3D/getWaveFilters3Dbior.m:12-58
  myMirrorPadImage       utilities/myMirrorPadImage.m:3-8
  myPSNR                 utilities/myPSNR.m:7-12

Options are plain dicts with the reference's field names.  Two fields exist
only here: ``refStride`` / ``refStrideWie`` (reference-block stride of step 1
/ step 2; absent or None means the block size, which is the reference's
tiling) and ``staleWeights`` (mirror GBM3D.m's reuse of step-1 weight slices
when step 2 has fewer spins; default True).  ``wname`` exists in the
reference but GBM3D.m ignores it (it always uses bior1.5 x Haar); here
``wname='haar'`` selects a 3D Haar bank for step 1.
"""
from __future__ import annotations

import json
import os

import numpy as np

PROFILES = ("default", "fast", "superFast", "accuracy")


def setBM3Dopts(profile: str = "default") -> dict:
    """Parameter profile; unknown names fall back to 'default' (setBM3Dopts.m:12-14)."""
    if profile not in PROFILES:
        profile = "default"
    o = dict(numMax=16, numMin=16, wname="bior", wnamez="db", order=15, orderz=1,
             levels=3, cycleSpin=2, tauMode=1, blockSize=16, blockSizeWie=8,
             matchSize=32, Wiener=True, filtType="ht")
    if profile == "default":
        o.update(matchSpins=[0, 4], matchSpinsWie=[0, 4])
    elif profile == "fast":
        o.update(matchSpins=[0, 4, 6], matchSpinsWie=[0])
    elif profile == "superFast":
        o.update(matchSpins=[0, 4, 6], matchSpinsWie=[0], blockSize=32, Wiener=False)
    else:  # accuracy
        o.update(matchSpins=[0, 4, 6], matchSpinsWie=[0, 4, 6])
    return o


def checkBM3Dopts(opts: dict | None) -> dict:
    """Fill missing fields with the reference defaults (checkBM3Dopts.m:10-24)."""
    o = dict(opts or {})
    o.setdefault("numMax", 16)
    o.setdefault("numMin", 16)
    o.setdefault("wname", "bior")
    o.setdefault("wnamez", "db")
    o.setdefault("order", 15)
    o.setdefault("orderz", 1)
    o.setdefault("levels", 3)
    o.setdefault("tauMode", 1)
    o.setdefault("filtType", "ht")
    o.setdefault("blockSize", 16)
    o.setdefault("blockSizeWie", 8)
    o.setdefault("matchSize", max(32, o["blockSize"]))
    o.setdefault("cycleSpin", 2)
    o.setdefault("matchSpins", [0, min(o["blockSize"], o["blockSizeWie"]) // 2])
    o.setdefault("Wiener", True)
    # present in every profile; checkBM3Dopts does not default it
    o.setdefault("matchSpinsWie", list(o["matchSpins"]))
    o.setdefault("staleWeights", True)
    return o


TUNED_SETS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_sets.json")
# the dense configuration the tuned sets are measured against (and the set for
# images below the smallest calibrated size)
DENSE = dict(blockSize=8, blockSizeWie=8, matchSize=32, numMax=16, numMin=16, refStride=3, refStrideWie=3,
             matchSpins=[0, 4], matchSpinsWie=[0, 4], cycleSpin=2, form="plain")


def tuned_opts(m: int, n: int, sigma: float, table: dict | None = None, sigma_below: bool = False) -> dict:
    """Options of the 'tuned' profile for an m x n image at noise level sigma:
    the autotuner's set for the largest calibrated size class not above
    min(m, n) and the calibrated sigma nearest in log scale (with
    ``sigma_below``, the largest calibrated sigma not above sigma, the
    smallest one below them all: lower noise classes hold denser sets)
    (gbm3d_b200/tuned_sets.json, written by ``python -m gbm3d_b200.autotune
    --classes``).  Each set stayed within 0.05 dB (less a 0.02 dB margin) of
    the dense configuration on its calibration images; below the smallest
    class the dense configuration itself is returned.  Not in the reference."""
    if table is None:
        with open(TUNED_SETS) as f:
            table = json.load(f)
    side = min(int(m), int(n))
    sizes = sorted({c["size"] for c in table["classes"]})
    fit = [z for z in sizes if z <= side]
    o = setBM3Dopts("default")
    o.update(DENSE)
    if not fit:
        return o
    size = fit[-1]
    rows = [c for c in table["classes"] if c["size"] == size]
    sg = max(float(sigma), 1e-6)
    if sigma_below:
        below = [c for c in rows if c["sigma"] <= sg]
        row = max(below, key=lambda c: c["sigma"]) if below else min(rows, key=lambda c: c["sigma"])
    else:
        row = min(rows, key=lambda c: (abs(np.log(c["sigma"] / sg)), c["sigma"]))
    o.update(row["opts"])
    return o


def resolve_opts(opts: dict | None, shape=None, sigma=None) -> dict:
    """GBM3D.m:15-19: a 'profile' field replaces every other field.  The
    'tuned' profile (not in the reference) depends on the image: it needs
    ``shape`` (m, n) and ``sigma`` and reads tuned_opts()."""
    if opts is None:
        opts = {"profile": "default"}
    if "profile" in opts:
        extra = {k: opts[k] for k in ("refStride", "refStrideWie", "staleWeights") if k in opts}
        if opts["profile"] == "tuned":
            if shape is None or sigma is None:
                raise ValueError("the 'tuned' profile needs the image size and sigma")
            o = tuned_opts(shape[0], shape[1], float(np.mean(np.sqrt(np.asarray(sigma, float))))
                           if np.ndim(sigma) >= 1 and np.size(sigma) > 1 else float(np.ravel(sigma)[0]))
            if "form" in opts:
                o["form"] = opts["form"]
        else:
            o = setBM3Dopts(opts["profile"])
        o.update(extra)
        opts = o
    return checkBM3Dopts(opts)


def strides(opts: dict) -> tuple[int, int]:
    """(step-1, step-2) reference strides; None or absent means the block size."""
    s1, s2 = opts.get("refStride"), opts.get("refStrideWie")
    return (int(s1) if s1 else int(opts["blockSize"]), int(s2) if s2 else int(opts["blockSizeWie"]))


def grid_count(L: int, d: int, s: int) -> int:
    """References along an axis of L pixels at stride s: floor((L-d)/s)+1."""
    return (L - d) // s + 1


def _bior_xy():
    Ca, Cb, Cc = 0.016572815184060, 0.121533978016438, np.sqrt(2.0) / 2
    lo = np.array([Ca, -Ca, -Cb, Cb, Cc, Cc, Cb, -Cb, -Ca, Ca])
    hi = np.zeros(10)
    hi[4], hi[5] = -Cc, Cc
    return lo, hi


def _fft2_sized(h, d1, d2):
    """fft2(h, d1, d2): zero-pad (or crop) h to d1 x d2 first."""
    z = np.zeros((d1, d2))
    a, b = min(h.shape[0], d1), min(h.shape[1], d2)
    z[:a, :b] = h[:a, :b]
    return np.fft.fft2(z)


def getColoredTau(levels: int, sigmaPSD, tau0: float = 6.0) -> np.ndarray:
    """levels x 7 thresholds for coloured noise, sigmaPSD = sigma^2 * |F(filter)|^2
    (utilities/getColoredTau.m:10-57): the 2D bior1.5 filters of the 7 detail
    bands (the 3D band order with the slot axis dropped), replicated 2^(i-1)
    times per axis at level i, and tau(i,j) = tau0 * sqrt(<PSD, |Psi_hat|^2> /
    sum |Psi_hat|^2)."""
    P = np.asarray(sigmaPSD, dtype=np.float64)
    d1, d2 = P.shape
    lo, hi = _bior_xy()
    f = [np.outer(lo, lo), np.outer(hi, lo), np.outer(lo, hi), np.outer(lo, lo),
         np.outer(hi, hi), np.outer(hi, lo), np.outer(lo, hi), np.outer(hi, hi)]
    f = [x.astype(np.float32).astype(np.float64) for x in f]  # Psi is single in the reference
    tau = np.zeros((levels, 7))
    for i in range(levels):
        k = 2 ** i
        for j in range(7):
            ph = np.kron(f[j + 1], np.ones((k, k)))  # imresize(.., 2^(i-1), 'nearest')
            F = np.abs(_fft2_sized(ph, d1, d2)) ** 2
            tau[i, j] = np.sqrt(np.sum(P * F) / np.sum(F))
    return tau * tau0


def gaussian_psf_hat(shape, omega: float) -> np.ndarray:
    """Transfer function of a unit-sum circular Gaussian of standard deviation
    omega centred on pixel (1,1) (the role of makeGausPSF(shape, omega) in
    getColoredWie.m:6; that helper is not part of the reference repository,
    so this form is an assumption)."""
    m, n = shape
    y = np.minimum(np.arange(m), m - np.arange(m))
    x = np.minimum(np.arange(n), n - np.arange(n))
    h = np.exp(-(y[:, None] ** 2 + x[None, :] ** 2) / (2.0 * omega ** 2))
    return np.fft.fft2(h / h.sum())


def _resize_bilinear_aa(a, out_len, axis):
    """One axis of imresize(.., 'bilinear') with antialiasing when shrinking:
    triangle kernel stretched by 1/scale, weights normalised, symmetric border."""
    L = a.shape[axis]
    scale = out_len / L
    width = 2.0 / scale if scale < 1 else 2.0
    u = np.arange(1, out_len + 1)
    x = u / scale + 0.5 * (1 - 1 / scale)
    left = np.floor(x - width / 2).astype(int)
    P = int(np.ceil(width)) + 2
    idx = left[:, None] + np.arange(P)[None, :]
    dist = x[:, None] - idx
    if scale < 1:
        w = scale * np.maximum(0.0, 1 - np.abs(scale * dist))
    else:
        w = np.maximum(0.0, 1 - np.abs(dist))
    w = w / w.sum(axis=1, keepdims=True)
    aux = np.concatenate([np.arange(1, L + 1), np.arange(L, 0, -1)])
    idx = aux[np.mod(idx - 1, 2 * L)] - 1
    a = np.moveaxis(a, axis, 0)
    out = np.einsum("up,up...->u...", w, a[idx])
    return np.moveaxis(out, 0, axis)


def getColoredWie(sigmaPSD, d: int) -> np.ndarray:
    """d x d Wiener sigmas for coloured noise (utilities/getColoredWie.m:6-18):
    the PSD smoothed by a Gaussian of width 3, resized to d x d (bilinear,
    antialiased), then sigmaWie(j,i) = sqrt(sum(PSD .* |fft2(idct2(e_ji))|^2)) / d."""
    P = np.asarray(sigmaPSD, dtype=np.float64)
    P = np.real(np.fft.ifft2(gaussian_psf_hat(P.shape, 3.0) * np.fft.fft2(P)))
    P = _resize_bilinear_aa(_resize_bilinear_aa(P, d, 0), d, 1)
    T = np.sqrt(2.0 / d) * np.cos(np.pi * (2 * np.arange(d)[None, :] + 1) * np.arange(d)[:, None] / (2 * d))
    T[0, :] = np.sqrt(1.0 / d)
    out = np.zeros((d, d))
    for i in range(d):
        for j in range(d):
            y = np.outer(T[j], T[i])  # idct2 of the impulse at (j, i)
            out[j, i] = np.sqrt(np.sum(P * np.abs(np.fft.fft2(y)) ** 2)) / d
    return out


def getTau(levels: int, mode: int = 1) -> np.ndarray:
    """levels x 7 threshold multipliers (getTau.m:9-51)."""
    tau = np.zeros((levels, 7), order="F")
    for j in range(7):
        for i in range(levels):
            base = 3.3 - 0.3 * i
            if mode == 1:
                v = base
            elif mode == 2:
                v = base if j < 3 else (base + 0.5 if j < 6 else base + 1.0)
            elif mode == 3:
                v = base if j < 3 else (base + 0.25 if j < 6 else base + 1.5)
            elif mode == 4:
                v = 2.9 if j < 3 else (2.9 + 0.5 if j < 6 else 2.9 + 1.0)
            else:
                v = 0.0
            tau[i, j] = v
    return tau


_CA = 0.016572815184060
_CB = 0.121533978016438
_CC = np.sqrt(2.0) / 2


def bior_factors() -> dict:
    """1D factors of the bior1.5 x Haar bank (getWaveFilters3Dbior.m:16-27,49-50)."""
    lo = np.array([_CA, -_CA, -_CB, _CB, _CC, _CC, _CB, -_CB, -_CA, _CA])
    hi = np.zeros(10)
    hi[4], hi[5] = -_CC, _CC
    shi = np.array([-_CA, -_CA, _CB, _CB, -_CC, _CC, -_CB, -_CB, _CA, _CA])
    return dict(a_lo_xy=lo, a_hi_xy=hi, s_lo_xy=np.abs(hi), s_hi_xy=shi,
                a_lo_z=np.array([_CC, _CC]), a_hi_z=np.array([-_CC, _CC]),
                s_lo_z=np.array([_CC, _CC]), s_hi_z=np.array([-_CC, _CC]))


def haar_factors() -> dict:
    """3D Haar bank: Haar on the spatial axes as well as the slot axis."""
    lo, hi = np.array([_CC, _CC]), np.array([-_CC, _CC])
    return dict(a_lo_xy=lo, a_hi_xy=hi, s_lo_xy=lo.copy(), s_hi_xy=hi.copy(),
                a_lo_z=lo.copy(), a_hi_z=hi.copy(), s_lo_z=lo.copy(), s_hi_z=hi.copy())


def _outer3(fy, fx, fz):
    return fy[:, None, None] * fx[None, :, None] * fz[None, None, :]


def bank_from_factors(fac: dict):
    """Psi, Psi2 (Ly x Lx x Lz x 8, single) built the way getWaveFilters3Dbior.m:39-58 does."""
    a = [(fac["a_lo_xy"], fac["a_hi_xy"]), (fac["a_lo_z"], fac["a_hi_z"])]
    s = [(fac["s_lo_xy"], fac["s_hi_xy"]), (fac["s_lo_z"], fac["s_hi_z"])]
    # reference band order: LLL, HLL, LHL, LLH, HHL, HLH, LHH, HHH in (y, x, z)
    order = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    Lxy, Lz = len(fac["a_lo_xy"]), len(fac["a_lo_z"])
    Psi = np.zeros((Lxy, Lxy, Lz, 8), dtype=np.float32, order="F")
    Psi2 = np.zeros_like(Psi)
    for f, (fy, fx, fz) in enumerate(order):
        Psi[:, :, :, f] = _outer3(a[0][fy], a[0][fx], a[1][fz])
        Psi2[:, :, :, f] = _outer3(s[0][fy], s[0][fx], s[1][fz])
    return Psi, Psi2


def getWaveFilters3Dbior():
    """[Psi, Psi2] of the reference (getWaveFilters3Dbior.m:1)."""
    return bank_from_factors(bior_factors())


def factors_from_bank(Psi, Psi2, tol: float = 1e-5) -> dict:
    """Recover separable 1D factors from a Psi/Psi2 pair.

    The kernels filter separably, so a bank passed through the drop-in
    denoiseAndAggregateGPU entry must be an outer product of 1D factors, as
    every bank of the reference is.  Known banks (bior1.5 x Haar, 3D Haar) are
    recognised exactly; any other rank-1 bank is factorised numerically.
    Raises ValueError for a bank that is not separable.
    """
    Psi = np.asarray(Psi, dtype=np.float64)
    Psi2 = np.asarray(Psi2, dtype=np.float64)
    for fac in (bior_factors(), haar_factors()):
        P, P2 = bank_from_factors(fac)
        if P.shape == Psi.shape and np.allclose(P, Psi, atol=tol) and np.allclose(P2, Psi2, atol=tol):
            return fac

    def split(B):
        # B[..., f] = u_fy (x) u_fx (x) v_fz.  With (a, c) the position of the
        # largest |LLL| entry: lo = LLL[:, a, c] / LLL[a, a, c] (lo[a] = 1),
        # vlo = LLL[a, a, :], hi = HLL[:, a, c] / vlo[c], vhi = LLH[a, a, :].
        t = B[..., 0]
        a, _, c = np.unravel_index(np.argmax(np.abs(t)), t.shape)
        if t[a, a, c] == 0:
            raise ValueError("filter bank is not separable")
        lo = t[:, a, c] / t[a, a, c]
        vlo = t[a, a, :].copy()
        hi = B[:, a, c, 1] / vlo[c]
        vhi = B[a, a, :, 3].copy()
        return lo, hi, vlo, vhi

    out = {}
    for tag, B in (("a", Psi), ("s", Psi2)):
        lo, hi, vlo, vhi = split(B)
        out[f"{tag}_lo_xy"], out[f"{tag}_hi_xy"] = lo, hi
        out[f"{tag}_lo_z"], out[f"{tag}_hi_z"] = vlo, vhi
    P, P2 = bank_from_factors(out)
    if not (np.allclose(P, Psi, atol=tol * 10) and np.allclose(P2, Psi2, atol=tol * 10)):
        raise ValueError("filter bank is not separable")
    return out


def myMirrorPadImage(I, M: int, N: int) -> np.ndarray:
    """Pad by flipping the last (M-m) rows / (N-n) cols (myMirrorPadImage.m:3-8)."""
    I = np.asarray(I, dtype=np.float64)
    m, n = I.shape
    O = np.zeros((M, N), order="F")
    O[:m, :n] = I
    O[m:M, :n] = np.flipud(I[m - (M - m):m, :n])
    O[:m, n:N] = np.fliplr(I[:m, n - (N - n):n])
    O[m:M, n:N] = np.fliplr(np.flipud(I[m - (M - m):m, n - (N - n):n]))
    return O


def myPSNR(Iref, Irec, maxI=None) -> float:
    """PSNR in dB; maxI defaults to max(Iref) as in myPSNR.m:7-12."""
    Iref = np.asarray(Iref, dtype=np.float64)
    Irec = np.asarray(Irec, dtype=np.float64)
    if maxI is None:
        maxI = Iref.max()
    mse = np.sum((Iref - Irec) ** 2) / Iref.size
    return float(10 * np.log10(maxI ** 2 / mse))
