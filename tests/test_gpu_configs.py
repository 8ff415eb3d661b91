"""The measured configurations against the oracle, at their own sizes.

Dense configuration (patch 8, reference stride 3, group 16, search +-16,
bior1.5 x Haar, 3 levels, 2 cycle spins, match spins [0 4] + [0 4]):
  * 1024 x 1024 at sigma 10, 25 and 50: the whole two-step pipeline through
    gbm3d_denoise is bit-identical to the oracle's FP32 mode (U and the step-1
    estimate U1), the match sets of both steps are identical (step 1 on the
    noisy image, step 2 on the pipeline's own pilot), and the error against
    the oracle's FP64 run is reported beside the 1e-4 bar;
  * the precision form at 4096 x 4096, sigma 25: the fraction of the step-1
    references whose tensor-core match set equals the plain matcher's (all
    1,857,769 of them), the PSNR of the whole pipeline against the plain
    path's, and on a 512 x 512 crop the max-abs against the FP64 oracle.
The oracle runs on all host threads; one 1024^2 image takes it tens of
seconds in FP32 and FP64 together.
"""
import time

import numpy as np
import pytest

from conftest import max_abs
from gbm3d_b200 import autotune, options, synth

pytestmark = pytest.mark.gpu
TOL = 1e-4  # max-abs on the 0-255 scale


def _dense(**kw):
    o = options.resolve_opts({"profile": "default"})
    o.update(autotune.BASELINE)
    o.update(kw)
    return o


@pytest.mark.parametrize("sigma", [10.0, 25.0, 50.0])
def test_dense_1024_against_oracle(gpu, oracle, sigma):
    clean, noisy = synth.noisy_image(1024, 1024, sigma, seed=2000 + int(sigma))
    o = _dense()
    U, out = gpu.GBM3D(noisy, sigma, o)
    U1 = out["U1"]
    t0 = time.perf_counter()
    Uo, U1o = oracle.GBM3D(noisy, sigma, o, prec=32)
    t32 = time.perf_counter() - t0
    t0 = time.perf_counter()
    U64, U164 = oracle.GBM3D(noisy, sigma, o, prec=64)
    t64 = time.perf_counter() - t0
    print(f"sigma {sigma:g}: oracle FP32 {t32:.1f} s, FP64 {t64:.1f} s on {oracle.num_threads()} threads; "
          f"max-abs vs FP64 oracle U {max_abs(U, U64):.3e}, U1 {max_abs(U1, U164):.3e}; PSNR GPU "
          f"{options.myPSNR(clean, U, 255):.4f} dB, FP64 oracle {options.myPSNR(clean, U64, 255):.4f} dB")
    assert max_abs(U1, U1o) <= TOL and max_abs(U, Uo) <= TOL
    assert np.array_equal(U1, U1o), "step-1 estimate differs from the FP32 oracle"
    assert np.array_equal(U, Uo), "final estimate differs from the FP32 oracle"
    # the match sets of both steps, the second on the pipeline's own pilot
    S1, _ = gpu.matchBlocksCPU(noisy, sigma, o)
    S1o, _, _ = oracle.matchBlocksCPU(noisy, sigma, o, prec=32)
    assert np.array_equal(np.asarray(S1), S1o), f"{int((np.asarray(S1) != S1o).sum())} step-1 entries differ"
    S2, _, _ = gpu.matchBlocksWie(U1, noisy, sigma, o)
    S2o, _, _ = oracle.matchBlocksWie(U1, noisy, sigma, o, prec=32)
    assert np.array_equal(np.asarray(S2), S2o), f"{int((np.asarray(S2) != S2o).sum())} step-2 entries differ"
    # the FP64 run of the same code is close in quality (its error is reported above, not bounded)
    assert abs(options.myPSNR(clean, U, 255) - options.myPSNR(clean, U64, 255)) < 0.02


def test_precision_4096(gpu, oracle):
    sigma = 25.0
    clean, noisy = synth.noisy_image(4096, 4096, sigma, seed=3000)
    o = _dense()
    op = dict(o, form="precision")
    Sp, _ = gpu.matchBlocksCPU(noisy, sigma, o, volume=False)
    Sq, _ = gpu.matchBlocksCPU(noisy, sigma, op, volume=False)
    Sp, Sq = np.asarray(Sp), np.asarray(Sq)
    agree = float(np.mean(np.all(Sp == Sq, axis=0)))
    del Sp, Sq
    U, _ = gpu.GBM3D(noisy, sigma, o)
    Uq, _ = gpu.GBM3D(noisy, sigma, op)
    p_plain, p_prec = options.myPSNR(clean, U, 255), options.myPSNR(clean, Uq, 255)
    # a 512 x 512 crop of the same image through the oracle's FP64 mode
    crop_c, crop = clean[1792:2304, 1792:2304], noisy[1792:2304, 1792:2304]
    Uc, _ = gpu.GBM3D(crop, sigma, op)
    U64, _ = oracle.GBM3D(crop, sigma, o, prec=64)
    err64 = max_abs(Uc, U64)
    print(f"precision form at 4096^2: step-1 match-set agreement {agree:.6f} over "
          f"{1363 * 1363} references; PSNR {p_prec:.4f} dB against plain {p_plain:.4f} dB; 512^2 crop: "
          f"max-abs vs FP64 oracle {err64:.3e}, PSNR {options.myPSNR(crop_c, Uc, 255):.4f} dB "
          f"(FP64 oracle {options.myPSNR(crop_c, U64, 255):.4f} dB)")
    assert agree == 1.0
    assert abs(p_prec - p_plain) < 0.01
    assert abs(options.myPSNR(crop_c, Uc, 255) - options.myPSNR(crop_c, U64, 255)) < 0.02
