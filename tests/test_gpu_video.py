"""Video path (VBM3D) on the GPU against the CPU oracle.

matchBlocksV (block matching across a window of frames), denoiseAndAggregateV
(sym4 x Haar wavelet hard threshold, [0,1] clamp, aggregation into the
frames) and the whole VBM3D driver follow the FP32 operation order of the
oracle's FP32 mode, so the contract is bit-identity: identical match sets and
identical floating-point outputs.  The error of the FP32 path against the
FP64 golden vectors (the FFT-route restatement) is stated per case.
"""
import os

import numpy as np
import pytest

from conftest import max_abs
from gbm3d_b200 import api, options, synth

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "video_32x40x4_s25.npz")


def _frames(m, n, F, sigma, seed):
    clean, noisy = synth.video(m, n, F, sigma, seed=seed)
    return clean / 255.0, noisy / 255.0, sigma / 255.0


CASES_MATCH = [
    # (m, n, frames, d, K, seed)
    (32, 40, 3, 8, 16, 1),
    (64, 48, 5, 8, 16, 2),
    (64, 64, 3, 16, 16, 3),
    (96, 64, 5, 32, 16, 4),
    (48, 56, 11, 8, 8, 5),
    (64, 96, 3, 32, 16, 6),  # patch 32, 3-frame window: the batched configuration's video shape
]


@pytest.mark.parametrize("m,n,F,d,K,seed", CASES_MATCH)
def test_matchBlocksV_bit_identical(gpu, oracle, m, n, F, d, K, seed):
    _, I, s = _frames(m, n, F, 25.0, seed)
    o = {"blockSize": d, "numMax": K, "numMin": K, "nF": F}
    S, V = api.matchBlocksV(I, s, o)
    S0, V0 = oracle.matchBlocksV(I, d, K, prec=32)
    assert np.array_equal(np.asarray(S), S0), f"{np.mean(np.asarray(S) != S0):.4f} of the indices differ"
    assert np.array_equal(V, V0)
    assert np.all(np.asarray(S)[0] == d * d * F // 2 + d // 2 + 1)  # slot 1 is the reference (matchBlocksV.m:103)


# the 320 x 288 case reaches the dense sym4 x Haar wavelet kernels at every level
@pytest.mark.parametrize("m,n,F,d,K,seed", CASES_MATCH[:4] + [(320, 288, 3, 8, 16, 7)])
def test_denoiseAndAggregateV_bit_identical(gpu, oracle, m, n, F, d, K, seed):
    """The stage alone, fed the oracle's match sets and volume."""
    _, I, s = _frames(m, n, F, 25.0, seed)
    S0, V0 = oracle.matchBlocksV(I, d, K, prec=32)
    o = {"blockSize": d, "numMax": K, "numMin": K, "nF": F, "levels": 3}
    U, out = api.denoiseAndAggregateV(None, V0, I, S0, s, o)
    U0, W0 = oracle.denoiseAndAggregateV(V0, S0, d, F, s * options.getTau(3, 2), 3, 2, prec=32)
    assert np.array_equal(U, U0), f"U max-abs {max_abs(U, U0):.3e}"
    assert np.array_equal(out["K"], W0), f"W max-abs {max_abs(out['K'], W0):.3e}"


CASES_VBM3D = [
    # (m, n, frames, nF, d, spins, seed)
    (32, 40, 4, 3, 8, (0, 4), 23),
    (30, 44, 5, 3, 8, (0, 4), 6),     # not a multiple of d: mirror padding
    (64, 64, 7, 5, 16, (0, 8), 7),
    (40, 48, 6, 5, 8, (0, 2, 5), 8),  # three spins: the mean divides by 3
    (80, 100, 4, 3, 32, (0, 16), 9),  # VBM3D's default patch 32 (register-tiled matcher), mirror padding
    (192, 256, 4, 3, 32, (0, 16), 10),  # levels 1-2 of the wavelet on the dense sym4 x Haar kernels
]


@pytest.mark.parametrize("m,n,Kf,nF,d,spins,seed", CASES_VBM3D)
def test_vbm3d_bit_identical(gpu, oracle, m, n, Kf, nF, d, spins, seed):
    clean, I, s = _frames(m, n, Kf, 25.0, seed)
    o = {"blockSize": d, "nF": nF, "matchSpins": list(spins)}
    Y, out = api.VBM3D(I, s, o)
    Y0 = oracle.VBM3D(I, s, d=d, K=16, spins=spins, nF=nF, prec=32)
    assert Y.shape == (m, n, Kf - nF + 1)
    assert np.array_equal(Y, Y0), f"max-abs {max_abs(Y, Y0):.3e} on [0,1]"
    hw = (nF - 1) // 2
    ps_noisy = options.myPSNR(clean[:, :, hw:Kf - hw], I[:, :, hw:Kf - hw], 1)
    ps = options.myPSNR(clean[:, :, hw:Kf - hw], Y, 1)
    print(f"VBM3D {m}x{n}x{Kf} nF={nF}: noisy {ps_noisy:.2f} dB -> {ps:.2f} dB")
    assert ps > ps_noisy + 1.5  # small frames: much of each frame is border


def test_vbm3d_golden(gpu):
    """Against the FP64 FFT-route golden vectors (nF = 3, patch 8, spins [0 4])."""
    g = np.load(GOLDEN)
    I, s = g["noisy"] / 255.0, float(g["sigma"]) / 255.0
    S, V = api.matchBlocksV(I[:, :, :3], s, {"blockSize": 8, "nF": 3})
    print(f"matchBlocksV: {np.mean(np.asarray(S) == g['S']):.4f} of the indices agree with FP64")
    Y, _ = api.VBM3D(I, s, {"blockSize": 8, "nF": 3})
    err = max_abs(Y, g["Y"])
    print(f"VBM3D: max-abs vs FP64 golden {err:.3e} on [0,1] ({err * 255:.3e} on 0-255)")
    assert err * 255 < 1.0


def test_video_option_errors(gpu):
    _, I, s = _frames(32, 32, 4, 25.0, 9)
    with pytest.raises(api.GBM3DError):
        api.matchBlocksV(I, s, {"blockSize": 8})  # an even number of frames
    with pytest.raises(api.GBM3DError):
        api.VBM3D(I[:, :, :3], s, {"blockSize": 8, "nF": 5})  # fewer frames than the window
    with pytest.raises(api.GBM3DError):
        api.VBM3D(I, s, {"blockSize": 8, "nF": 3, "numMin": 8})  # the tolerance branch
    with pytest.raises(api.GBM3DError):
        api.VBM3D(I, s, {"blockSize": 8, "nF": 3, "wname": "bior"})
