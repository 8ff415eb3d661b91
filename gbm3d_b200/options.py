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


def resolve_opts(opts: dict | None) -> dict:
    """GBM3D.m:15-19: a 'profile' field replaces every other field."""
    if opts is None:
        opts = {"profile": "default"}
    if "profile" in opts:
        extra = {k: opts[k] for k in ("refStride", "refStrideWie", "staleWeights") if k in opts}
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
