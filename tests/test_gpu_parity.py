"""CUDA path (libgbm3d.so through its C ABI) against the CPU oracle.

The kernels follow the FP32 operation order of the oracle's FP32 mode, so the
contract checked here is bit-identity: identical match sets (ties broken by
the lowest column-major window index, as MATLAB's mink does) and identical
floating-point outputs.  The required tolerance, 1e-4 max-abs on a 0-255
scale, is asserted as well so a failure reports which bar was missed, and the
error against the FP64 run of the oracle is stated (not bounded) per case.
Stages are also tested in isolation by feeding them the oracle's upstream
outputs, so a difference does not cascade.
"""
import numpy as np
import pytest

from conftest import max_abs
from gbm3d_b200 import options, synth

pytestmark = pytest.mark.gpu
TOL = 1e-4  # max-abs on the 0-255 scale


def _report(name, got, ref64):
    print(f"{name}: max-abs vs FP64 oracle = {max_abs(got, ref64):.3e}")


def _opts(profile="default", **kw):
    o = options.resolve_opts({"profile": profile})
    o.update(kw)
    return o


CASES_MATCH = [
    # (m, n, d, d2, sigma, seed)
    (64, 96, 16, 32, 25.0, 1),
    (128, 128, 16, 32, 10.0, 2),
    (96, 64, 8, 32, 50.0, 3),
    (64, 64, 8, 24, 25.0, 4),
    (64, 64, 32, 32, 25.0, 5),
    (72, 88, 8, 16, 25.0, 6),
    (100, 76, 16, 24, 25.0, 7),  # not a multiple of d: trailing rows/cols hold no references
]


@pytest.mark.parametrize("m,n,d,d2,sigma,seed", CASES_MATCH)
def test_matchBlocksCPU(gpu, oracle, m, n, d, d2, sigma, seed):
    _, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _opts(blockSize=d, matchSize=d2)
    S, V = gpu.matchBlocksCPU(noisy, sigma, o)
    So, Vo, co = oracle.matchBlocksCPU(noisy, sigma, o, prec=32)
    assert np.array_equal(np.asarray(S), So), f"{int((np.asarray(S) != So).sum())} match entries differ"
    assert np.array_equal(S.count, co)
    assert np.array_equal(V, Vo)


def test_matchBlocksCPU_ties_flat_image(gpu, oracle):
    """All distances tie: lowest indices win and S(1) is overwritten by the reference."""
    I = np.full((64, 64), 77.0)
    o = _opts()
    S, _ = gpu.matchBlocksCPU(I, 25.0, o)
    So, _, _ = oracle.matchBlocksCPU(I, 25.0, o, prec=32)
    assert np.array_equal(np.asarray(S), So)


def test_matchBlocksCPU_tolerance_branch(gpu, oracle):
    _, noisy = synth.noisy_image(96, 96, 10.0, seed=8)
    o = _opts(numMin=4, numMax=16)
    S, V = gpu.matchBlocksCPU(noisy, 10.0, o)
    So, Vo, co = oracle.matchBlocksCPU(noisy, 10.0, o, prec=32)
    assert np.array_equal(S.count, co)
    assert np.array_equal(np.asarray(S), So)
    assert np.array_equal(V, Vo)


@pytest.mark.parametrize("m,n,sigma,seed,wav", [(64, 96, 25.0, 1, "bior"), (128, 128, 50.0, 2, "bior"),
                                                 (64, 64, 25.0, 3, "haar")])
def test_denoiseAndAggregateGPU(gpu, oracle, m, n, sigma, seed, wav):
    _, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _opts()
    So, Vo, co = oracle.matchBlocksCPU(noisy, sigma, o, prec=32)
    tau = sigma * options.getTau(3, 1)
    fac = options.bior_factors() if wav == "bior" else options.haar_factors()
    Psi, Psi2 = options.bank_from_factors(fac)
    from gbm3d_b200.api import _as_set
    U, W = gpu.denoiseAndAggregateGPU(Vo, _as_set(So, co), tau, Psi, Psi2, o)
    f = oracle.bior_filters() if wav == "bior" else oracle.haar_filters()
    Uo, Wo = oracle.denoiseAndAggregateGPU(Vo, So, tau, o, cnt=co, filters=f, prec=32)
    assert max_abs(U / W, Uo / Wo) <= TOL
    assert np.array_equal(U, Uo) and np.array_equal(W, Wo)


@pytest.mark.parametrize("m,n,sigma,seed,d2", [(64, 96, 25.0, 1, 32), (128, 128, 10.0, 2, 32), (64, 64, 50.0, 3, 24)])
def test_matchBlocksWie(gpu, oracle, m, n, sigma, seed, d2):
    clean, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _opts(matchSize=d2)
    pilot = clean + np.random.default_rng(seed).normal(0, 2.0, clean.shape)
    S, V1, V2 = gpu.matchBlocksWie(pilot, noisy, sigma, o)
    So, V1o, V2o = oracle.matchBlocksWie(pilot, noisy, sigma, o, prec=32)
    assert np.array_equal(np.asarray(S), So)
    assert np.array_equal(V1, V1o) and np.array_equal(V2, V2o)


@pytest.mark.parametrize("variant", ["fast", "legacy"])
@pytest.mark.parametrize("m,n,sigma,seed", [(64, 96, 25.0, 1), (128, 64, 10.0, 2)])
def test_denoiseAndAggregateWiener(gpu, oracle, m, n, sigma, seed, variant):
    clean, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _opts()
    pilot = clean + np.random.default_rng(seed).normal(0, 2.0, clean.shape)
    if variant == "legacy":  # denoiseAndAggregateWie expects a [0,1] scale
        pilot, noisy, sigma = pilot / 255, noisy / 255, sigma / 255
    So, V1o, V2o = oracle.matchBlocksWie(pilot, noisy, sigma, o, prec=32)
    from gbm3d_b200.api import _as_set
    fn = gpu.denoiseAndAggregateWieFast if variant == "fast" else gpu.denoiseAndAggregateWie
    U, W = fn(V1o, V2o, _as_set(So), sigma, o)
    Uo, Wo = oracle.denoiseAndAggregateWieFast(V1o, V2o, So, sigma, o, prec=32, variant=0 if variant == "fast" else 1)
    assert np.array_equal(U, Uo) and np.array_equal(W, Wo)


def test_wiener_sigma_matrix(gpu, oracle):
    clean, noisy = synth.noisy_image(64, 64, 25.0, seed=9)
    o = _opts()
    So, V1o, V2o = oracle.matchBlocksWie(clean, noisy, 25.0, o, prec=32)
    sig = np.asfortranarray(np.linspace(10, 40, 64).reshape(8, 8))
    from gbm3d_b200.api import _as_set
    U, W = gpu.denoiseAndAggregateWieFast(V1o, V2o, _as_set(So), sig, o)
    Uo, Wo = oracle.denoiseAndAggregateWieFast(V1o, V2o, So, sig, o, prec=32)
    assert np.array_equal(U, Uo) and np.array_equal(W, Wo)


PIPE = [
    # (m, n, sigma, seed, profile)
    (64, 96, 25.0, 1, "default"),
    (128, 128, 10.0, 2, "default"),
    (128, 128, 50.0, 3, "default"),
    (70, 90, 25.0, 4, "default"),     # mirror padding to a multiple of 16
    (96, 96, 25.0, 5, "fast"),        # stale step-1 weights in the final normalisation
    (96, 128, 25.0, 6, "accuracy"),
    (128, 128, 25.0, 7, "superFast"),  # blockSize 32, no Wiener step
    (256, 256, 25.0, 8, "default"),
]


@pytest.mark.parametrize("m,n,sigma,seed,profile", PIPE)
def test_GBM3D_pipeline(gpu, oracle, m, n, sigma, seed, profile):
    clean, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _opts(profile)
    U, out = gpu.GBM3D(noisy, sigma, {"profile": profile})
    Uo, U1o = oracle.GBM3D(noisy, sigma, o, prec=32)
    U64, _ = oracle.GBM3D(noisy, sigma, o, prec=64)
    _report(f"GBM3D {profile} {m}x{n} sigma={sigma}", U, U64)
    assert max_abs(U, Uo) <= TOL and max_abs(out["U1"], U1o) <= TOL
    assert np.array_equal(out["U1"], U1o), "step-1 estimate not bit-identical"
    assert np.array_equal(U, Uo), "final estimate not bit-identical"
    assert options.myPSNR(clean, U, 255) > options.myPSNR(clean, noisy, 255) + 5


def test_GBM3D_golden(gpu, oracle):
    """Against the committed FFT-route golden vectors: within the FP32-vs-FP64 gap."""
    import glob
    import os
    for p in sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "default_*.npz"))):
        g = np.load(p)
        U, out = gpu.GBM3D(g["noisy"], float(g["sigma"]), {"profile": "default"})
        assert max_abs(U, g["U"]) < 1e-2, p


def test_errors_are_reported(gpu):
    with pytest.raises(gpu.GBM3DError):
        gpu.GBM3D(np.full((64, 64), np.nan), 25.0)
    with pytest.raises(gpu.GBM3DError):
        gpu.matchBlocksCPU(np.zeros((16, 16)), 25.0, _opts())  # smaller than matchSize
    with pytest.raises(gpu.GBM3DError):
        gpu.GBM3D(np.zeros((64, 64)), 25.0, dict(_opts(), blockSize=12, matchSize=32))
    # the context stays usable after an error
    _, noisy = synth.noisy_image(64, 64, 25.0, seed=1)
    U, _ = gpu.GBM3D(noisy, 25.0)
    assert np.isfinite(U).all()


def test_deterministic(gpu):
    _, noisy = synth.noisy_image(128, 96, 25.0, seed=12)
    U1, _ = gpu.GBM3D(noisy, 25.0)
    U2, _ = gpu.GBM3D(noisy, 25.0)
    assert np.array_equal(U1, U2)


@pytest.mark.parametrize("m,n,sigma,seed,d", [(64, 64, 25.0, 21, 16), (48, 64, 0.1, 22, 16), (64, 96, 10.0, 23, 8)])
def test_matchBlocksGPU_global(gpu, oracle, m, n, sigma, seed, d):
    _, noisy = synth.noisy_image(m, n, sigma, seed=seed)
    o = _opts(blockSize=d)
    S = gpu.matchBlocksGPU(noisy, sigma, o)
    So, co, _ = oracle.matchBlocksGPU(noisy, sigma, o, prec=32)
    assert np.array_equal(np.asarray(S), So), f"{int((np.asarray(S) != So).sum())} entries differ"
    assert np.array_equal(S.count, co)


def test_matchBlocksGPU_tolerance_branch(gpu, oracle):
    _, noisy = synth.noisy_image(64, 64, 0.1, seed=24)
    o = _opts(numMin=2, numMax=16)
    S = gpu.matchBlocksGPU(noisy, 0.1, o)
    So, co, _ = oracle.matchBlocksGPU(noisy, 0.1, o, prec=32)
    assert np.array_equal(S.count, co)
    assert np.array_equal(np.asarray(S), So)


def test_denoiseAndAggregateGPU_median(gpu, oracle):
    """filtType 'median': medfilt3 of the volume replaces the wavelet (denoiseAndAggregateGPU.m:49-52)."""
    _, noisy = synth.noisy_image(64, 96, 25.0, seed=31)
    o = _opts(filtType="median")
    So, Vo, co = oracle.matchBlocksCPU(noisy, 25.0, o, prec=32)
    from gbm3d_b200.api import _as_set
    U, W = gpu.denoiseAndAggregateGPU(Vo, _as_set(So, co), 25.0 * options.getTau(3, 1), None, None, o)
    Uo, Wo = oracle.denoiseAndAggregateMedian(Vo, So, o, cnt=co, prec=32)
    assert np.array_equal(U, Uo) and np.array_equal(W, Wo)


@pytest.mark.parametrize("K,s", [(8, 8), (8, 5), (32, 8)])
def test_GBM3D_pipeline_group_sizes(gpu, oracle, K, s):
    """Groups of 8 and 32 slots (the aggregation's enumeration divides by K
    with a multiply-high; the wavelet and Wiener passes run 8 or 32 slots).
    NaN compares equal: with fewer than 15 slots an all-zero pilot group gets
    an infinite Wiener weight in the reference's arithmetic too."""
    clean, noisy = synth.noisy_image(120, 136, 25.0, seed=40 + K + s)
    o = _opts(blockSize=8, blockSizeWie=8, numMax=K, numMin=K, refStride=s, refStrideWie=s)
    U, out = gpu.GBM3D(noisy, 25.0, o)
    Uo, U1o = oracle.GBM3D(noisy, 25.0, o, prec=32)
    assert np.array_equal(out["U1"], U1o, equal_nan=True), "step-1 estimate not bit-identical"
    assert np.array_equal(U, Uo, equal_nan=True), "final estimate not bit-identical"


def test_GBM3D_pipeline_median(gpu, oracle):
    clean, noisy = synth.noisy_image(96, 96, 25.0, seed=32)
    o = dict(_opts(), filtType="median")
    U, out = gpu.GBM3D(noisy, 25.0, o)
    Uo, U1o = oracle.GBM3D(noisy, 25.0, o, prec=32)
    assert np.array_equal(out["U1"], U1o) and np.array_equal(U, Uo)


def test_GBM3D_distributed_cuda_matches_oracle_tiles(gpu):
    """Tiled GBM3D: the CUDA drop-ins per tile reproduce the oracle per tile bit for bit."""
    from gbm3d_b200 import distributed as D
    from test_distributed import oracle_backend
    clean, noisy = synth.noisy_image(300, 290, 25.0, seed=42)
    U, out = D.GBM3D_distributed(noisy, 25.0, {"profile": "default"})
    Uo, outo = D.GBM3D_distributed(noisy, 25.0, {"profile": "default"}, backend=oracle_backend())
    assert np.array_equal(out["U2"], outo["U2"]) and np.array_equal(U, Uo)
    assert options.myPSNR(clean, U, 255) > options.myPSNR(clean, noisy, 255) + 5


def test_GBM3D_distributed_device_matches_host_driver(gpu):
    """The device tile driver (one call per step, device-side stitching) equals
    the host driver over the CUDA drop-ins bit for bit, on an image whose edge
    tiles are pulled back (getBM3D_distribution.m:29-36)."""
    from gbm3d_b200 import distributed as D
    clean, noisy = synth.noisy_image(600, 540, 25.0, seed=43)
    U, out = D.GBM3D_distributed(noisy, 25.0, {"profile": "default"})
    Uh, outh = D.GBM3D_distributed(noisy, 25.0, {"profile": "default"}, backend=D.cuda_backend())
    assert np.array_equal(out["U2"], outh["U2"]) and np.array_equal(U, Uh)
    assert options.myPSNR(clean, U, 255) > options.myPSNR(clean, noisy, 255) + 5


@pytest.mark.parametrize("m,n,sigma,omega,seed", [(64, 64, 25.0, 1.0, 31), (96, 80, 40.0, 2.0, 32)])
def test_GBM3D_colored_noise(gpu, oracle, m, n, sigma, omega, seed):
    """GBM3D.m:33-35: matrix sigma (sigma^2 * PSD) -> getColoredTau / getColoredWie."""
    clean, noisy, psd = synth.colored_noisy_image(m, n, sigma, omega=omega, seed=seed)
    o = _opts()
    U, out = gpu.GBM3D(noisy, psd, o)
    Uo, U1o = oracle.GBM3D_colored(noisy, float(np.mean(np.sqrt(psd))), out["tau"], out["sigmaWie"], o, prec=32)
    assert np.array_equal(out["U1"], U1o) and np.array_equal(U, Uo)
    assert options.myPSNR(clean, U, 255) > options.myPSNR(clean, noisy, 255)
