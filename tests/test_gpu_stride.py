"""Reference stride (refStride / refStrideWie) and the 3D Haar step-1 bank on
the CUDA path, against the CPU oracle.

The reference tiles its references at stride blockSize; the configurations
this library targets use patch 8 at stride 3 (BM3D's dense grid), group 16 and
a +-12 or +-16 search, and a 3D Haar bank for step 1.  The oracle generalises
the reference's loops to a stride (and was pinned against the FFT-route
restatement at stride 3, tests/golden/stride3_*.npz); here the kernels must
reproduce it bit for bit, as at the reference's own settings.
"""
import json
import os

import numpy as np
import pytest

from conftest import max_abs
from gbm3d_b200 import options, synth
from gbm3d_b200.api import _as_set

pytestmark = pytest.mark.gpu
TOL = 1e-4  # max-abs on the 0-255 scale


def _stride_opts(d=8, s=3, d2=24, sw=None, **kw):
    o = options.resolve_opts({"profile": "default"})
    o.update(blockSize=d, blockSizeWie=d, matchSize=d2, refStride=s, refStrideWie=sw or s)
    o.update(kw)
    return o


@pytest.mark.parametrize("m,n,d,s,d2,sigma,seed", [
    (64, 64, 8, 3, 24, 25.0, 1),
    (70, 59, 8, 3, 32, 10.0, 2),   # grid does not reach the last rows/cols
    (64, 80, 8, 3, 16, 50.0, 3),
    (64, 64, 16, 5, 32, 25.0, 4),
    (40, 40, 8, 1, 24, 25.0, 5),   # every pixel a reference
    (64, 64, 8, 8, 24, 25.0, 6),   # stride = blockSize: the reference's tiling
])
def test_matchBlocksCPU_stride(gpu, oracle, m, n, d, s, d2, sigma, seed):
    _, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _stride_opts(d, s, d2)
    S, V = gpu.matchBlocksCPU(noisy, sigma, o)
    So, Vo, co = oracle.matchBlocksCPU(noisy, sigma, o, prec=32)
    assert S.shape == So.shape == (16, (m - d) // s + 1, (n - d) // s + 1)
    assert np.array_equal(np.asarray(S), So), f"{int((np.asarray(S) != So).sum())} match entries differ"
    assert np.array_equal(S.count, co)
    assert V.shape == Vo.shape and np.array_equal(V, Vo)


def test_matchBlocksCPU_stride_tolerance_branch(gpu, oracle):
    _, noisy = synth.noisy_image(64, 64, 10.0, seed=7)
    o = _stride_opts(numMin=4)
    S, V = gpu.matchBlocksCPU(noisy, 10.0, o)
    So, Vo, co = oracle.matchBlocksCPU(noisy, 10.0, o, prec=32)
    assert np.array_equal(S.count, co) and np.array_equal(np.asarray(S), So) and np.array_equal(V, Vo)


@pytest.mark.parametrize("wav", ["bior", "haar"])
@pytest.mark.parametrize("m,n,sigma,seed", [(64, 64, 25.0, 11), (71, 56, 50.0, 12)])
def test_denoiseAndAggregateGPU_stride(gpu, oracle, m, n, sigma, seed, wav):
    _, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _stride_opts()
    So, Vo, co = oracle.matchBlocksCPU(noisy, sigma, o, prec=32)
    tau = sigma * options.getTau(3, 1)
    fac = options.bior_factors() if wav == "bior" else options.haar_factors()
    Psi, Psi2 = options.bank_from_factors(fac)
    U, W = gpu.denoiseAndAggregateGPU(Vo, _as_set(So, co), tau, Psi, Psi2, o)
    f = oracle.bior_filters() if wav == "bior" else oracle.haar_filters()
    Uo, Wo = oracle.denoiseAndAggregateGPU(Vo, So, tau, o, cnt=co, filters=f, prec=32)
    K, M, N = So.shape
    assert U.shape == ((M - 1) * 3 + 8, (N - 1) * 3 + 8)
    assert np.array_equal(U, Uo) and np.array_equal(W, Wo)


@pytest.mark.parametrize("m,n,sigma,seed,d2", [(64, 64, 25.0, 13, 24), (65, 59, 10.0, 14, 32)])
def test_wiener_stride(gpu, oracle, m, n, sigma, seed, d2):
    clean, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _stride_opts(d2=d2)
    pilot = clean + np.random.default_rng(seed).normal(0, 2.0, clean.shape)
    S, V1, V2 = gpu.matchBlocksWie(pilot, noisy, sigma, o)
    So, V1o, V2o = oracle.matchBlocksWie(pilot, noisy, sigma, o, prec=32)
    assert np.array_equal(np.asarray(S), So)
    assert np.array_equal(V1, V1o) and np.array_equal(V2, V2o)
    U, W = gpu.denoiseAndAggregateWieFast(V1o, V2o, _as_set(So), sigma, o)
    Uo, Wo = oracle.denoiseAndAggregateWieFast(V1o, V2o, So, sigma, o, prec=32)
    assert np.array_equal(U, Uo) and np.array_equal(W, Wo)


@pytest.mark.parametrize("m,n,sigma,seed,d2,wname", [
    (64, 64, 25.0, 21, 24, "haar"),    # patch 8, stride 3, group 16, +-12, 3D Haar
    (96, 80, 10.0, 22, 32, "bior"),    # patch 8, stride 3, group 16, +-16, bior
    (96, 96, 50.0, 23, 32, "bior"),
    (75, 61, 25.0, 24, 24, "haar"),    # generalised padding
    (256, 256, 25.0, 25, 24, "haar"),  # the CPU-runnable configuration's size
])
def test_GBM3D_pipeline_stride(gpu, oracle, m, n, sigma, seed, d2, wname):
    clean, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _stride_opts(d2=d2, wname=wname)
    U, out = gpu.GBM3D(noisy, sigma, o)
    Uo, U1o = oracle.GBM3D(noisy, sigma, o, prec=32)
    U64, _ = oracle.GBM3D(noisy, sigma, o, prec=64)
    print(f"stride-3 {wname} {m}x{n} sigma={sigma}: max-abs vs FP64 oracle = {max_abs(U, U64):.3e}")
    assert max_abs(U, Uo) <= TOL and max_abs(out["U1"], U1o) <= TOL
    assert np.array_equal(out["U1"], U1o), "step-1 estimate not bit-identical"
    assert np.array_equal(U, Uo), "final estimate not bit-identical"
    assert options.myPSNR(clean, U, 255) > options.myPSNR(clean, noisy, 255) + 3


def test_GBM3D_stride_golden(gpu):
    """Against the FFT-route golden vectors at stride 3: within the FP32-vs-FP64 gap."""
    path = os.path.join(os.path.dirname(__file__), "golden", "stride3_50x58_s25.npz")
    g = np.load(path)
    o = options.resolve_opts({"profile": str(g["profile"])})
    o.update(json.loads(str(g["opts"])))
    U, out = gpu.GBM3D(g["noisy"], float(g["sigma"]), o)
    assert max_abs(out["U1"], g["Ustep1"]) < 2e-3
    assert max_abs(U, g["U"]) < 2e-3


def test_GBM3D_tuned_options_golden(gpu, oracle):
    """The tuned form's option set (step-1 stride 8, step-2 stride 7, one
    spin per step, one cycle spin) on a crop of the reference's demo photo:
    bit-identical to the oracle's FP32 mode, and within the FP32-vs-FP64 gap
    of the FFT-route golden vectors."""
    path = os.path.join(os.path.dirname(__file__), "golden", "tuned8x7_fabio_96x80_s25.npz")
    g = np.load(path)
    o = options.resolve_opts({"profile": str(g["profile"])})
    o.update(json.loads(str(g["opts"])))
    U, out = gpu.GBM3D(g["noisy"], float(g["sigma"]), o)
    Uo, U1o = oracle.GBM3D(g["noisy"], float(g["sigma"]), o, prec=32)
    assert np.array_equal(out["U1"], U1o) and np.array_equal(U, Uo), "not bit-identical to the oracle"
    assert max_abs(out["U1"], g["Ustep1"]) < 1e-3  # 1.1e-4 measured
    assert max_abs(U, g["U"]) < 1e-3  # 1.0e-4 measured


def test_stride_errors(gpu):
    from gbm3d_b200 import GBM3DError
    _, noisy = synth.noisy_image(64, 64, 25.0, seed=1)
    with pytest.raises(GBM3DError):
        gpu.GBM3D(noisy, 25.0, _stride_opts(s=9))  # stride larger than the block leaves gaps
    with pytest.raises(GBM3DError):
        gpu.GBM3D(noisy, 25.0, _stride_opts(wname="sym"))
