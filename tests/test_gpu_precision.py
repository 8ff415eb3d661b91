"""Tensor-core matching (precision and tensor forms).

The 16-bit tensor-core distances (bf16 in the precision form, f16 in the
tensor form) only bound the candidates: every position
whose approximate distance lies within the rounding bound of the K-th best is
re-ranked by the exact FP32 distance in the exhaustive matcher's operation
order.  So the contract is identity: the match sets and the gathered volume
equal the plain path's (itself bit-identical to the oracle) at every stride
and search size, including images whose candidate lists overflow (a flat
image: every distance ties) and so take the exhaustive search.  The tensor
form (tensor-core matching, plain aggregation) therefore returns the plain
path's output bit for bit; the precision form adds Kahan-compensated
aggregation, held to the plain path's PSNR.
"""
import numpy as np
import pytest

from conftest import max_abs
from gbm3d_b200 import options, synth

pytestmark = pytest.mark.gpu


def _opts(form, d2=32, s=3, sw=None, **kw):
    o = options.resolve_opts({"profile": "default"})
    o.update(blockSize=8, blockSizeWie=8, matchSize=d2, refStride=s, refStrideWie=sw or s, form=form)
    o.update(kw)
    return o


@pytest.mark.parametrize("m,n,sigma,d2,s,seed", [
    (256, 256, 25.0, 32, 3, 1), (256, 256, 10.0, 32, 3, 2), (256, 256, 50.0, 24, 3, 3), (256, 256, 25.0, 16, 3, 4),
    (512, 512, 25.0, 32, 8, 5), (512, 512, 25.0, 32, 7, 6), (384, 320, 10.0, 32, 6, 7), (300, 260, 50.0, 32, 8, 8),
    (200, 232, 25.0, 24, 5, 9), (256, 256, 25.0, 32, 1, 10),
])
@pytest.mark.parametrize("form", ["precision", "tensor"])
def test_tensor_match_sets_identical(gpu, oracle, m, n, sigma, d2, s, seed, form):
    _, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    S0, V0 = gpu.matchBlocksCPU(noisy, sigma, _opts("plain", d2, s))
    S1, V1 = gpu.matchBlocksCPU(noisy, sigma, _opts(form, d2, s))
    S0, S1 = np.asarray(S0), np.asarray(S1)
    same = np.all(S0 == S1, axis=0)
    print(f"{form} {m}x{n} sigma={sigma} d2={d2} stride {s}: match-set agreement {same.mean():.6f} "
          f"over {same.size}")
    assert same.all(), f"{int((~same).sum())} of {same.size} match sets differ"
    assert np.array_equal(V0, V1)
    if m * n <= 256 * 256:
        So, _, _ = oracle.matchBlocksCPU(noisy, sigma, _opts("plain", d2, s), prec=32)
        assert np.array_equal(S1, So)


@pytest.mark.parametrize("form", ["precision", "tensor"])
def test_tensor_match_overflow_takes_exhaustive_search(gpu, form):
    """Flat image: every candidate ties, each list overflows, the exhaustive
    matcher finishes every reference (lowest window indices win)."""
    I = np.full((128, 136), 90.0)
    I[40:80, 30:70] = 140.0  # one step edge: a mix of tied and distinct distances
    for s in (8, 3):
        S0, V0 = gpu.matchBlocksCPU(I, 25.0, _opts("plain", 32, s))
        S1, V1 = gpu.matchBlocksCPU(I, 25.0, _opts(form, 32, s))
        assert np.array_equal(np.asarray(S0), np.asarray(S1))
        assert np.array_equal(V0, V1)


def test_tensor_candidate_statistics(gpu):
    """The bound leaves few candidates on a noisy image; the f16 operands of
    the tensor form leave no more than the bf16 ones of the precision form."""
    _, noisy = synth.noisy_image(512, 512, 25.0, seed=31)
    ctx = gpu.context()
    mean = {}
    for form in ("precision", "tensor"):
        ctx.tc_stats(True)
        gpu.matchBlocksCPU(noisy, 25.0, _opts(form, 32, 8))
        h = np.array(ctx.tc_stats(False))
        assert h.sum() == 64 * 64  # one count per reference block
        mean[form] = float((h * (np.arange(33) * 8 + 4)).sum() / h.sum())
        print(form, "candidates per reference (bucket midpoints):", round(mean[form], 1), "histogram", h.tolist())
    assert mean["tensor"] <= mean["precision"]
    assert mean["tensor"] < 64


def test_tensor_matcher_wait_limit_is_reported(gpu):
    """Every wait of the tensor-core matcher is bounded.  The probe makes each
    CTA wait on a barrier that nothing completes: the wait runs out after 2000
    clocks, the kernel lets its TMA copies in flight land, releases TMEM and
    reports it; the context stays usable."""
    from gbm3d_b200 import GBM3DError
    _, noisy = synth.noisy_image(256, 256, 25.0, seed=32)
    ctx = gpu.context()
    o = _opts("tensor", 32, 8, 7, matchSpins=[0], matchSpinsWie=[0], cycleSpin=1, staleWeights=False)
    ctx.set_tc_wait(-2000)
    try:
        with pytest.raises(GBM3DError, match="wait limit"):
            gpu.GBM3D(noisy, 25.0, o)
    finally:
        ctx.set_tc_wait(0)
    Ut, _ = gpu.GBM3D(noisy, 25.0, o)
    Up, _ = gpu.GBM3D(noisy, 25.0, dict(o, form="plain"))
    assert np.array_equal(Ut, Up)


@pytest.mark.parametrize("sigma,s,sw,seed", [(25.0, 8, 7, 21), (10.0, 3, 3, 22), (50.0, 8, 6, 23)])
def test_tensor_form_equals_plain(gpu, sigma, s, sw, seed):
    _, noisy = synth.noisy_image(320, 288, sigma, seed=seed)
    kw = dict(matchSpins=[0], matchSpinsWie=[0], cycleSpin=1, staleWeights=False) if s == 8 else {}
    Up, op = gpu.GBM3D(noisy, sigma, _opts("plain", 32, s, sw, **kw))
    Ut, ot = gpu.GBM3D(noisy, sigma, _opts("tensor", 32, s, sw, **kw))
    assert np.array_equal(op["U1"], ot["U1"])
    assert np.array_equal(Up, Ut)


@pytest.mark.parametrize("sigma,seed", [(25.0, 11), (10.0, 12), (50.0, 13)])
def test_precision_pipeline_psnr(gpu, oracle, sigma, seed):
    clean, noisy = synth.noisy_image(256, 256, sigma, seed=seed)
    Up, _ = gpu.GBM3D(noisy, sigma, _opts("plain"))
    Uq, _ = gpu.GBM3D(noisy, sigma, _opts("precision"))
    U64, _ = oracle.GBM3D(noisy, sigma, _opts("plain"), prec=64)
    pp, pq = options.myPSNR(clean, Up, 255), options.myPSNR(clean, Uq, 255)
    print(f"sigma={sigma}: PSNR plain {pp:.3f} precision {pq:.3f} (delta {pq - pp:+.4f} dB); "
          f"max-abs precision vs FP64 oracle {max_abs(Uq, U64):.3e}, plain vs FP64 {max_abs(Up, U64):.3e}")
    assert abs(pq - pp) < 0.01


def test_precision_form_rejects_unsupported(gpu):
    from gbm3d_b200 import GBM3DError
    _, noisy = synth.noisy_image(64, 64, 25.0, seed=1)
    with pytest.raises(GBM3DError):
        gpu.GBM3D(noisy, 25.0, _opts("precision", blockSize=16, refStride=4, refStrideWie=4))
    with pytest.raises(GBM3DError):
        gpu.GBM3D(noisy, 25.0, _opts("precision", numMin=4))
