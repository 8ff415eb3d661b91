"""The strip form: output columns of one image computed on their own.

gbm3d_denoise_strip_device runs every stage on the columns its consumers
read, so a strip must equal the same columns of the whole-image call bit for
bit (the whole-image call is itself bit-identical to the oracle, see
test_gpu_parity / test_gpu_stride).  Cases cover the reference's profiles
(patch 16 at stride 16 with two spins per step, the stale-weight 'fast'
profile), dense stride 3, the tuned option set, the 3D Haar bank with two cycle
spins, the median filter, no Wiener step, strips at both image edges (where
the spin shifts and the wavelet's circular filters wrap) and one-column strips.
"""
import numpy as np
import pytest

from gbm3d_b200 import options, synth
from gbm3d_b200 import distributed as D

pytestmark = pytest.mark.gpu


def _run(gpu, noisy, sigma, o, bounds):
    import torch
    from gbm3d_b200 import api
    ctx = api.context()
    m, n = noisy.shape
    dI = torch.from_numpy(np.asfortranarray(noisy).ravel(order="F").copy()).cuda()
    dU = torch.empty_like(dI)
    torch.cuda.synchronize()
    api.GBM3D_device(dI.data_ptr(), m, n, sigma, dU.data_ptr(), o, ctx=ctx)
    ctx.synchronize()
    full = dU.cpu().numpy().reshape((m, n), order="F")
    strips = []
    for lo, hi in bounds:
        t = torch.full(((hi - lo) * m,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        api.GBM3D_strip_device(dI.data_ptr(), m, n, sigma, lo, hi, t.data_ptr(), o, ctx=ctx)
        ctx.synchronize()
        strips.append(t.cpu().numpy().reshape((m, hi - lo), order="F"))
    return full, strips


def _opts(**kw):
    o = options.resolve_opts({"profile": kw.pop("profile", "default")})
    o.update(kw)
    return o


CASES = [
    ("default", 200, 260, 25.0, {}),
    ("fast_stale", 190, 230, 25.0, {"profile": "fast"}),
    ("dense3", 120, 150, 25.0, {"blockSize": 8, "blockSizeWie": 8, "refStride": 3, "refStrideWie": 3}),
    ("tuned8x7", 256, 300, 25.0, {"blockSize": 8, "blockSizeWie": 8, "refStride": 8, "refStrideWie": 7,
                                  "matchSpins": [0], "matchSpinsWie": [0], "cycleSpin": 1}),
    ("haar_cycles", 150, 170, 50.0, {"blockSize": 8, "blockSizeWie": 8, "refStride": 4, "refStrideWie": 4,
                                     "wname": "haar", "cycleSpin": 2, "matchSize": 24}),
    ("median", 140, 160, 25.0, {"blockSize": 8, "blockSizeWie": 8, "refStride": 4, "refStrideWie": 4,
                                "filtType": "median"}),
    ("no_wiener", 160, 180, 10.0, {"Wiener": False}),
]


@pytest.mark.parametrize("name,m,n,sigma,kw", CASES, ids=[c[0] for c in CASES])
def test_strips_equal_whole_image(gpu, name, m, n, sigma, kw):
    clean, noisy = synth.noisy_image(m, n, sigma, seed=len(name) + m)
    o = _opts(**kw)
    bounds = D.strip_bounds(n, 3) + [(0, 1), (n - 5, n), (n // 2 - 8, n // 2 + 9)]
    full, strips = _run(gpu, noisy, sigma, o, bounds)
    assert options.myPSNR(clean, full, 255) > options.myPSNR(clean, noisy, 255) + 3
    for (lo, hi), U in zip(bounds, strips):
        assert np.array_equal(U, full[:, lo:hi]), f"strip [{lo}, {hi}) differs from the whole-image call"


def test_strip_driver_assembles_whole_image(gpu):
    """GBM3D_strips on one process (three strips in turn) equals GBM3D."""
    clean, noisy = synth.noisy_image(180, 210, 25.0, seed=77)
    o = _opts(blockSize=8, blockSizeWie=8, refStride=3, refStrideWie=3)
    U, _ = gpu.GBM3D(noisy, 25.0, o)
    Us = D.GBM3D_strips(noisy, 25.0, o, strips=3)
    assert np.array_equal(Us, U)


def test_strip_errors(gpu):
    from gbm3d_b200 import api
    from gbm3d_b200._lib import GBM3DError
    import torch
    m, n = 64, 64
    dI = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    dU = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    o = _opts(blockSize=8, blockSizeWie=8, refStride=4, refStrideWie=4)
    with pytest.raises(GBM3DError) as e:
        api.GBM3D_strip_device(dI.data_ptr(), m, n, 25.0, 10, 10, dU.data_ptr(), o)
    assert "strip columns" in str(e.value)
    with pytest.raises(GBM3DError) as e:
        api.GBM3D_strip_device(dI.data_ptr(), m, n, 25.0, 0, n + 1, dU.data_ptr(), o)
    assert "strip columns" in str(e.value)
    o2 = dict(o, form="precision", numMin=16)
    with pytest.raises(GBM3DError) as e:
        api.GBM3D_strip_device(dI.data_ptr(), m, n, 25.0, 0, 32, dU.data_ptr(), o2)
    assert "strip form" in str(e.value)
