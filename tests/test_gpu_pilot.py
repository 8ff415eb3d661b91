"""Learned pilot on the GPU: tensor-core forward, backward and training
against the CPU reference (oracle/pilot_ref.py, itself pinned by finite
differences in test_pilot_ref.py).

The kernels round inputs, weights and activations to bf16 and accumulate in
fp32, as the reference models; the remaining differences are accumulation
order and the bf16 rounding of the backward activations, so the bars are
relative: forward within 1e-2 of the residual's range, gradients within 5e-2
of each layer's gradient norm with cosine similarity above 0.999.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from oracle import pilot_ref as R  # noqa: E402

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _params(seed, last_scale=10.0):
    p = R.init_params(seed)
    p[-(9 * 48 + 1):] *= last_scale  # a last layer large enough to be measured
    return p


@pytest.mark.parametrize("N,H,W", [(2, 20, 150), (1, 9, 128), (3, 5, 37)])
def test_pilot_forward_matches_reference(gpu, N, H, W):
    from gbm3d_b200 import pilot
    import torch
    rng = np.random.default_rng(N * 100 + H)
    img = rng.uniform(0, 255, (N, H, W))
    sig = rng.uniform(5, 50, N)
    p = _params(1)
    pilot.set_params(p)
    out = torch.empty((N, H, W), device="cuda")
    pilot.forward_device(_dev(img), _dev(sig), out)
    got = out.cpu().numpy().astype(np.float64)
    ref, _ = R.forward(p, img, sig)
    r_got, r_ref = (img - got) / 255, (img - ref) / 255
    err = np.abs(r_got - r_ref).max()
    print(f"forward {N}x{H}x{W}: max |r| {np.abs(r_ref).max():.4f}, max error {err:.2e}")
    assert err <= 1e-2 * np.abs(r_ref).max()


def test_pilot_gradients_match_reference(gpu):
    from gbm3d_b200 import pilot
    from gbm3d_b200._lib import context, lib
    rng = np.random.default_rng(5)
    N, H, W = 2, 12, 40
    img = rng.uniform(0, 255, (N, H, W))
    tgt = img + rng.normal(0, 8, img.shape)
    sig = rng.uniform(5, 50, N)
    p = _params(2)
    pilot.set_params(p)
    import torch
    ctx = context()
    g = np.zeros(pilot.param_count(), dtype=np.float32)
    loss = C.c_float(0)
    di, dt, ds = _dev(img), _dev(tgt), _dev(sig)
    torch.cuda.synchronize()  # the inputs are on the device before the library's stream reads them
    ctx.check(lib().gbm3d_pilot_gradients(ctx.h, C.c_void_p(di.data_ptr()), C.c_void_p(dt.data_ptr()),
                                          C.c_void_p(ds.data_ptr()), N, H, W, g.ctypes.data_as(C.c_void_p),
                                          C.byref(loss)))
    ref, lref = R.gradients(p, img, sig, tgt)
    assert abs(loss.value - lref) <= 1e-2 * lref
    off = np.cumsum([0] + [9 * co * ci + co for ci, co in R.LAYERS])
    for l in range(len(R.LAYERS)):
        a, b = g[off[l]:off[l + 1]].astype(np.float64), ref[off[l]:off[l + 1]]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        print(f"layer {l}: |g| {np.linalg.norm(b):.3e} relative error {rel:.2e} cosine {cos:.6f}")
        assert rel < 5e-2 and cos > 0.999


def test_pilot_training_reduces_loss(gpu):
    """A few hundred Adam steps of the library's own kernels on (noisy, step-1)
    pairs from the plain pipeline."""
    from gbm3d_b200 import pilot
    data = pilot.make_dataset(n_crops=64, crop=64, size=256, seed=3, log=None)
    _, losses = pilot.train(steps=300, batch=8, lr=2e-3, data=data, log=None)
    first, last = np.mean(losses[:20]), np.mean(losses[-20:])
    print(f"training loss {first:.2f} -> {last:.2f}")
    assert last < 0.5 * first


def test_pilot_deterministic(gpu):
    from gbm3d_b200 import pilot
    data = pilot.make_dataset(n_crops=16, crop=64, size=256, seed=4, log=None)
    a, _ = pilot.train(steps=5, batch=4, data=data, log=None)
    b, _ = pilot.train(steps=5, batch=4, data=data, log=None)
    assert np.array_equal(a, b)


def _wiener_on(pilot_img, noisy, sigma, o):
    """Step 2 alone (matchBlocksWie + denoiseAndAggregateWieFast, one spin)
    with the given image as its pilot: the method without a step-1 estimate
    when the pilot is the noisy image itself."""
    from gbm3d_b200 import api
    S, V1, V2 = api.matchBlocksWie(pilot_img, noisy, sigma, o)
    U, W = api.denoiseAndAggregateWieFast(V1, V2, S, sigma, o)
    return U / W


@pytest.mark.parametrize("sigma,seed", [(15.0, 61), (25.0, 62), (50.0, 63)])
def test_trained_pilot_gains(gpu, sigma, seed):
    """What the trained network adds, on a 512^2 image: the 2-step result with
    its pilot against (a) Wiener filtering with the noisy image as the pilot
    (no step-1 estimate at all) and (b) the same network untrained."""
    import time
    from gbm3d_b200 import api, options, pilot, synth
    if not os.path.exists(pilot.WEIGHTS):
        pytest.skip("no trained weights")
    clean, noisy = synth.noisy_image(512, 512, sigma, seed=seed)
    o = pilot.dense_opts(refStrideWie=8, matchSpinsWie=[0])
    pilot.load()
    t0 = time.perf_counter()
    Ul, outl = api.GBM3D(noisy, sigma, dict(o, form="learned"))
    t_learned = time.perf_counter() - t0
    t0 = time.perf_counter()
    Un = _wiener_on(noisy, noisy, sigma, dict(o, form="plain"))
    t_nopilot = time.perf_counter() - t0
    pilot.set_params(pilot.init_params(0))
    Uu, _ = api.GBM3D(noisy, sigma, dict(o, form="learned"))
    pilot.load()
    pl, pn, pu = (options.myPSNR(clean, U, 255) for U in (Ul, Un, Uu))
    p1 = options.myPSNR(clean, outl["U1"], 255)
    print(f"sigma {sigma:g}: learned pilot {pl:.3f} dB (its step-1 estimate {p1:.3f} dB, {t_learned * 1e3:.0f} ms), "
          f"Wiener on the noisy pilot {pn:.3f} dB ({t_nopilot * 1e3:.0f} ms), untrained network {pu:.3f} dB, "
          f"noisy {options.myPSNR(clean, noisy, 255):.3f} dB")
    assert pl > pn + 1.0, "the trained pilot does not improve on Wiener filtering without one"
    assert pl > pu + 3.0, "training does not improve the pilot"
