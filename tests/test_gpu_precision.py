"""Precision form: bf16 tensor-core block distances with an exact FP32 re-rank
of the 32 best candidates, and Kahan-compensated aggregation.

The plain path is pinned to the oracle bit for bit; the precision form is held
to the plain path: the share of references whose match set is identical
(ranked by the exact distance and the window index in both), the validity of
every set, and the PSNR of the whole pipeline (within 0.05 dB of plain).
"""
import numpy as np
import pytest

from conftest import max_abs
from gbm3d_b200 import options, synth

pytestmark = pytest.mark.gpu


def _opts(form, d2=32, **kw):
    o = options.resolve_opts({"profile": "default"})
    o.update(blockSize=8, blockSizeWie=8, matchSize=d2, refStride=3, refStrideWie=3, form=form)
    o.update(kw)
    return o


def _ssd(I, i, j, e, s, d, d2):
    """Exact distance of candidate e (1-based window index) of reference (i, j), float64,
    on the reference's search image (rows/cols r < d2/2 hold r + d2/2, then periodic)."""
    h = d2 // 2
    m, n = I.shape
    rows = [r + h if r < h else (r - h) % m for r in range(m + d2)]
    cols = [c + h if c < h else (c - h) % n for c in range(n + d2)]
    P = I[np.ix_(rows, cols)]
    a, b = (e - 1) % d2, (e - 1) // d2
    ref = P[i * s + h:i * s + h + d, j * s + h:j * s + h + d]
    cand = P[i * s + a:i * s + a + d, j * s + b:j * s + b + d]
    return float(((ref - cand) ** 2).sum())


@pytest.mark.parametrize("sigma,d2,seed", [(25.0, 32, 1), (10.0, 32, 2), (50.0, 24, 3), (25.0, 16, 4)])
def test_precision_match_sets_agree(gpu, sigma, d2, seed):
    _, noisy = synth.noisy_image(256, 256, sigma, seed=seed)
    S0, V0 = gpu.matchBlocksCPU(noisy, sigma, _opts("plain", d2))
    S1, V1 = gpu.matchBlocksCPU(noisy, sigma, _opts("precision", d2))
    S0, S1 = np.asarray(S0), np.asarray(S1)
    K, M, N = S0.shape
    same = np.all(S0 == S1, axis=0)
    rate = same.mean()
    print(f"sigma={sigma} d2={d2}: match-set agreement {rate:.5f} over {M * N} references")
    assert rate >= 0.97
    # every precision set is a valid, duplicate-free window selection led by the reference
    h = d2 // 2
    assert np.all(S1[0] == h + h * d2 + 1)
    assert S1.min() >= 1 and S1.max() <= d2 * d2
    srt = np.sort(S1[1:], axis=0)
    assert np.all(srt[1:] != srt[:-1])
    # where the sets agree, the gathered blocks agree
    for i, j in list(zip(*np.nonzero(same)))[::97]:
        blk = np.s_[i * 8:(i + 1) * 8, j * 8:(j + 1) * 8, :]
        assert np.array_equal(V0[blk], V1[blk])
    # where they differ, the precision set is no better than the exact optimum
    I32 = noisy.astype(np.float32).astype(np.float64)
    for (i, j) in list(zip(*np.nonzero(~same)))[:20]:
        tot0 = sum(_ssd(I32, i, j, int(e), 3, 8, d2) for e in S0[1:, i, j])
        tot1 = sum(_ssd(I32, i, j, int(e), 3, 8, d2) for e in S1[1:, i, j])
        assert tot1 >= tot0 * (1 - 1e-6)


@pytest.mark.parametrize("sigma,seed", [(25.0, 11), (10.0, 12), (50.0, 13)])
def test_precision_pipeline_psnr(gpu, oracle, sigma, seed):
    clean, noisy = synth.noisy_image(256, 256, sigma, seed=seed)
    Up, _ = gpu.GBM3D(noisy, sigma, _opts("plain"))
    Uq, _ = gpu.GBM3D(noisy, sigma, _opts("precision"))
    U64, _ = oracle.GBM3D(noisy, sigma, _opts("plain"), prec=64)
    pp, pq = options.myPSNR(clean, Up, 255), options.myPSNR(clean, Uq, 255)
    print(f"sigma={sigma}: PSNR plain {pp:.3f} precision {pq:.3f} (delta {pq - pp:+.4f} dB); "
          f"max-abs precision vs FP64 oracle {max_abs(Uq, U64):.3e}, plain vs FP64 {max_abs(Up, U64):.3e}")
    assert pq >= pp - 0.05


def test_precision_form_rejects_unsupported(gpu):
    from gbm3d_b200 import GBM3DError
    _, noisy = synth.noisy_image(64, 64, 25.0, seed=1)
    with pytest.raises(GBM3DError):
        gpu.GBM3D(noisy, 25.0, _opts("precision", blockSize=16, refStride=4, refStrideWie=4))
    with pytest.raises(GBM3DError):
        gpu.GBM3D(noisy, 25.0, _opts("precision", numMin=4))
