"""Size-independent properties at the configurations' full sizes, on the GPU.

The oracle needs minutes at these sizes, so instead of comparing with it the
tests check properties that any correct run must have:
  * scale equivariance: GBM3D(2 I, 2 sigma) = 2 GBM3D(I, sigma) bit for bit
    (a power-of-two scale changes no rounding, no tie between distances and
    no threshold decision; the oracle shows the same identity);
  * determinism: the same call twice gives the same bits;
  * a denoising gain, and for the tuned option set the bench's quality bound
    (at most 0.05 dB below the dense plain configuration on the same image).
Dense configuration: patch 8, stride 3, group 16, search +-16, bior1.5 x Haar.
"""
import numpy as np
import pytest

from gbm3d_b200 import autotune, options, synth

pytestmark = pytest.mark.gpu

TUNED = dict(refStride=8, refStrideWie=7, matchSpins=[0], matchSpinsWie=[0], cycleSpin=1, staleWeights=False)


def _dense(**kw):
    o = options.resolve_opts({"profile": "default"})
    o.update(autotune.BASELINE)
    o.update(kw)
    return o


class _Device:
    """One device-resident image and output through gbm3d_denoise_device."""

    def __init__(self, noisy):
        import torch
        from gbm3d_b200 import _lib
        self.torch = torch
        self.m, self.n = noisy.shape
        self.ctx = _lib.Context(0)
        self.dI = torch.from_numpy(np.asfortranarray(noisy).ravel(order="F").copy()).cuda()
        self.dU = torch.empty_like(self.dI)

    def run(self, o, sigma, scale=1.0):
        from gbm3d_b200 import api
        src = self.dI * scale if scale != 1.0 else self.dI
        self.torch.cuda.synchronize()  # the library runs on its own stream
        api.GBM3D_device(src.data_ptr(), self.m, self.n, sigma * scale, self.dU.data_ptr(), o, ctx=self.ctx)
        self.ctx.synchronize()
        return self.dU.cpu().numpy().reshape(self.m, self.n, order="F").copy()

    def close(self):
        self.ctx.close()


@pytest.mark.parametrize("sigma", [10.0, 25.0, 50.0])
def test_dense_1024_properties(gpu, sigma):
    clean, noisy = synth.noisy_image(1024, 1024, sigma, seed=1000 + int(sigma))
    dev = _Device(noisy)
    try:
        o = _dense()
        U = dev.run(o, sigma)
        assert np.array_equal(dev.run(o, sigma), U), "not deterministic"
        assert np.array_equal(dev.run(o, sigma, scale=2.0), 2.0 * U), "not scale-equivariant"
        gain = options.myPSNR(clean, U, 255) - options.myPSNR(clean, noisy, 255)
        assert gain > {10.0: 5.0, 25.0: 10.0, 50.0: 12.0}[sigma], gain
    finally:
        dev.close()


def test_tuned_4096_properties(gpu):
    clean, noisy = synth.noisy_image(4096, 4096, 25.0, seed=100)
    dev = _Device(noisy)
    try:
        o = _dense(**TUNED)
        U = dev.run(o, 25.0)
        assert np.array_equal(dev.run(o, 25.0, scale=2.0), 2.0 * U), "not scale-equivariant"
        Up = dev.run(_dense(), 25.0)
        p_tuned, p_plain = options.myPSNR(clean, U, 255), options.myPSNR(clean, Up, 255)
        assert p_tuned >= p_plain - 0.05, (p_tuned, p_plain)
        assert p_plain - options.myPSNR(clean, noisy, 255) > 15.0
    finally:
        dev.close()


def test_precision_form_2048_properties(gpu):
    """The precision form (bf16 tensor-core distances, exact FP32 re-rank,
    Kahan aggregation) at 2048^2: bf16 rounding also commutes with a
    power-of-two scale, so the identity holds bit for bit, and its PSNR stays
    within 0.01 dB of the plain path's on the same image."""
    clean, noisy = synth.noisy_image(2048, 2048, 25.0, seed=2025)
    dev = _Device(noisy)
    try:
        o = _dense(form="precision")
        U = dev.run(o, 25.0)
        assert np.array_equal(dev.run(o, 25.0, scale=2.0), 2.0 * U), "not scale-equivariant"
        Up = dev.run(_dense(), 25.0)
        assert abs(options.myPSNR(clean, U, 255) - options.myPSNR(clean, Up, 255)) < 0.01
    finally:
        dev.close()
