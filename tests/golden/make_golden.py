"""Generate the golden vectors in tests/golden/*.npz.

    python tests/golden/make_golden.py [--reference DIR] [case ...]

DIR is the reference checkout (default: $GBM3D_REFERENCE_ROOT, else
/root/reference); only the demo-photo cases and the sym4 check read it.

The vectors come from oracle/fft_route.py, the restatement that follows the
MATLAB reference's FFT route operation by operation in float64 (the reference
itself needs MATLAB, which cannot run here).  Inputs are seeded synthetic
images (gbm3d_b200.synth), so every case is reproducible, and one crop of the
reference's demo photo (read from the reference checkout at generation time;
the fixture stores the crop itself).  Each file holds the
inputs and, per stage, the outputs of the reference function with that name.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gbm3d_b200 import options, synth  # noqa: E402
from oracle import fft_route as F  # noqa: E402


def banks(fac):
    Psi, Psi2 = options.bank_from_factors(fac)
    # float64 banks built from the same factors (the FFT route runs in float64)
    order = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    A = [(fac["a_lo_xy"], fac["a_hi_xy"]), (fac["a_lo_z"], fac["a_hi_z"])]
    S = [(fac["s_lo_xy"], fac["s_hi_xy"]), (fac["s_lo_z"], fac["s_hi_z"])]
    o3 = lambda a, b, c: a[:, None, None] * b[None, :, None] * c[None, None, :]  # noqa: E731
    P = np.stack([o3(A[0][a], A[0][b], A[1][c]) for a, b, c in order], -1)
    P2 = np.stack([o3(S[0][a], S[0][b], S[1][c]) for a, b, c in order], -1)
    return P, P2


# patch 8, reference stride 3, group 16, search +-12 (matchSize 24)
STRIDE3 = dict(blockSize=8, blockSizeWie=8, matchSize=24, refStride=3, refStrideWie=3)

# the option set the autotuner picks for 4096^2 at sigma 25: patch 8, step-1
# stride 8, step-2 stride 7, one match spin per step, one cycle spin
TUNED8X7 = dict(blockSize=8, blockSizeWie=8, matchSize=32, refStride=8, refStrideWie=7, matchSpins=[0],
                matchSpinsWie=[0], cycleSpin=1, staleWeights=False)

CASES = [
    # name, m, n, sigma, seed, profile, wavelet, option overrides
    ("default_64x96_s25", 64, 96, 25.0, 3, "default", "bior", {}),
    ("default_70x90_s10", 70, 90, 10.0, 5, "default", "bior", {}),
    ("fast_64x64_s50", 64, 64, 50.0, 7, "fast", "bior", {}),
    ("haar_64x64_s25", 64, 64, 25.0, 11, "default", "haar", {}),
    ("stride3_50x58_s25", 50, 58, 25.0, 31, "default", "bior", STRIDE3),
    ("stride3haar_40x48_s10", 40, 48, 10.0, 32, "default", "haar", STRIDE3),
]


REFERENCE = os.environ.get("GBM3D_REFERENCE_ROOT", "/root/reference")  # the reference checkout (--reference)


def fabio_path():
    """The reference's demo photo (demoDenoise.m:13), MIT licence."""
    return os.path.join(REFERENCE, "fabio.jpeg")


def fabio_crop(m, n, sigma, seed):
    """(clean, noisy): a central m x n crop of the reference's demo photo as
    demoDenoise.m reads it (imread, then rgb2gray on uint8: the luma weights
    0.298936021293775, 0.587043074451121, 0.114020904255103, rounded to uint8),
    on the 0-255 scale, plus N(0, sigma^2) noise from the project's generator."""
    from PIL import Image
    rgb = np.asarray(Image.open(fabio_path()).convert("RGB"), dtype=np.float64)
    w = np.array([0.298936021293775, 0.587043074451121, 0.114020904255103])
    grey = np.clip(np.floor(rgb @ w + 0.5), 0, 255)
    r0, c0 = (grey.shape[0] - m) // 2, (grey.shape[1] - n) // 2
    clean = np.asfortranarray(grey[r0:r0 + m, c0:c0 + n])
    rng = np.random.Generator(np.random.PCG64(seed + 1_000_003))
    return clean, np.asfortranarray(clean + sigma * rng.standard_normal((m, n)))


def make(name, m, n, sigma, seed, profile, wav, over, image=None):
    clean, noisy = image(m, n, sigma, seed) if image else synth.noisy_image(m, n, sigma, seed=seed)
    opts = options.resolve_opts({"profile": profile})
    opts.update(over)
    fac = options.bior_factors() if wav == "bior" else options.haar_factors()
    P, P2 = banks(fac)
    tau_unit = options.getTau(opts["levels"], opts["tauMode"])
    d, dw, d2, K = opts["blockSize"], opts["blockSizeWie"], opts["matchSize"], opts["numMax"]
    st1, st2 = opts.get("refStride") or d, opts.get("refStrideWie") or dw
    out = dict(clean=clean, noisy=noisy, sigma=sigma, profile=profile, wavelet=wav)
    if over:
        out["opts"] = json.dumps(over, sort_keys=True)
    # stage tests on the image padded as the pipeline pads it
    Mp, Np = F.padded_size(m, opts), F.padded_size(n, opts)
    Ip = options.myMirrorPadImage(noisy, Mp, Np)
    S1, Vol, _, _ = F.match_blocks(Ip, d, d2, K, st=st1)
    U1, W1 = F.denoise_ht(Vol, S1, sigma * tau_unit, P, P2, d, d2, opts["levels"], opts["cycleSpin"], st=st1)
    pilot = U1 / W1
    S2, _, V1, V2 = F.match_blocks(pilot, dw, d2, K, In=Ip, st=st2)
    U2, W2 = F.denoise_wiener(V1, V2, S2, sigma, d2, st=st2)
    out.update(padded=Ip, S1=S1, U1=U1, W1=W1, pilot=pilot, S2=S2, U2=U2, W2=W2)
    if wav == "bior":
        U, Ustep1 = F.gbm3d(noisy, sigma, opts, P, P2, tau_unit)
        out.update(U=U, Ustep1=Ustep1)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: getattr(v, "shape", v) for k, v in out.items() if k not in ("profile", "wavelet")})


def make_global(name, m, n, sigma, seed):
    """matchBlocksGPU (global search, sym4 prefilter when sigma > 30/255)."""
    _, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    S, pre = F.match_blocks_global(noisy, sigma, 16, 16)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), noisy=noisy, sigma=sigma, S=S, prefiltered=pre)
    print(name, S.shape)


def make_video(name, m, n, frames, sigma, seed, d=8):
    """VBM3D (nF = 3, patch d (8, or VBM3D.m's default 32), group 16, sym4 x
    Haar, tauMode 2, spins [0 d/2]) on frames scaled to [0,1], and the stages
    of its first window."""
    clean, noisy = synth.video(m, n, frames, sigma, seed=seed)
    I, s = noisy / 255.0, sigma / 255.0
    fac = dict(a_lo_xy=F.SYM4_LO, a_hi_xy=F.SYM4_HI, s_lo_xy=F.SYM4_LO, s_hi_xy=F.SYM4_HI,
               a_lo_z=options.haar_factors()["a_lo_z"], a_hi_z=options.haar_factors()["a_hi_z"],
               s_lo_z=options.haar_factors()["a_lo_z"], s_hi_z=options.haar_factors()["a_hi_z"])
    P, P2 = banks(fac)
    tau_unit = options.getTau(3, 2)
    Y = F.vbm3d(I, s, d, 16, 3, 2, tau_unit, [0, d // 2], 3, P, P2)
    S, Vol = F.match_blocks_video(I[:, :, :3], d, 16)
    U, W = F.denoise_video(Vol, S, s * tau_unit, P, P2, d, 3, 3, 2)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), clean=clean, noisy=noisy, sigma=sigma, Y=Y, S=S,
                        Vol=Vol, U=U, W=W)
    print(name, Y.shape)


def check_sym4_data():
    """The restated sym4 coefficients equal the reference's filter data file."""
    p = os.path.join(REFERENCE, "archive", "waveletFilters", "sym4Filters.mat")
    if os.path.exists(p):
        import scipy.io as sio
        d = sio.loadmat(p)
        assert np.array_equal(np.ravel(d["Lo_d"]), F.SYM4_LO) and np.array_equal(np.ravel(d["Hi_d"]), F.SYM4_HI)
        print("sym4 coefficients match", p)


if __name__ == "__main__":
    args = sys.argv[1:]
    if "--reference" in args:
        i = args.index("--reference")
        REFERENCE = args[i + 1]
        del args[i:i + 2]
    only = args  # optional case names; default: all
    for c in CASES:
        if not only or c[0] in only:
            make(*c)
    if not only or "default_fabio_96x80_s25" in only:
        make("default_fabio_96x80_s25", 96, 80, 25.0, 41, "default", "bior", {}, image=fabio_crop)
    if not only or "tuned8x7_fabio_96x80_s25" in only:
        make("tuned8x7_fabio_96x80_s25", 96, 80, 25.0, 41, "default", "bior", TUNED8X7, image=fabio_crop)
    if "video_32x40x4_s25" in only:
        make_video("video_32x40x4_s25", 32, 40, 4, 25.0, 23)
    if "video_64x96x4_d32_s25" in only:
        make_video("video_64x96x4_d32_s25", 64, 96, 4, 25.0, 24, d=32)
    if only:
        sys.exit(0)
    make_global("global_64x64_s25", 64, 64, 25.0, 21)
    make_global("global_48x64_s01", 48, 64, 0.1, 22)
    make_video("video_32x40x4_s25", 32, 40, 4, 25.0, 23)
    make_video("video_64x96x4_d32_s25", 64, 96, 4, 25.0, 24, d=32)
    check_sym4_data()
