"""The MEX gateways (gbm3d_b200/mex/*.c) through a mock MATLAB runtime.

MATLAB and Octave are not installed, so the gateways are compiled with gcc
against tests/mexmock/mex.h and called from Python the way MATLAB calls a
MEX file.  Without a GPU the tests cover argument checking, option parsing
errors and the no-device error; with one, every gateway is compared with the
library's Python API, and GBM3D.m's driver loop (source/GBM3D.m:21-83) is
replayed through the gateways alone and compared with the whole-pipeline
entry point.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "mexmock"))
import harness as H  # noqa: E402

from gbm3d_b200 import options, synth  # noqa: E402


@pytest.fixture(scope="module")
def gw():
    from gbm3d_b200 import build
    build.build()
    H.build()
    return {g: H.Gateway(g) for g in H.GATEWAYS}


def _mx(o):
    """An options dict as the MATLAB struct the gateways receive."""
    mo = {k: v for k, v in o.items() if v is not None}
    mo["Wiener"] = bool(o["Wiener"])
    mo["matchSpins"] = np.array(o["matchSpins"], dtype=np.float64)
    mo["matchSpinsWie"] = np.array(o["matchSpinsWie"], dtype=np.float64)
    return mo


def _opts(profile="default", **kw):
    o = options.resolve_opts({"profile": profile})
    o.update(kw)
    return o, _mx(o)


def _cell_to_set(C, K):
    """cell(M, N) of uint32 columns -> K x M x N array and counts."""
    M, N = C.shape
    S = np.zeros((K, M, N), dtype=np.uint32)
    cnt = np.zeros((M, N), dtype=np.int32)
    for g, col in enumerate(C.items):
        i, j = g % M, g // M
        v = np.ravel(col)
        S[: v.size, i, j] = v
        cnt[i, j] = v.size
    return S, cnt


def _set_to_cell(S, cnt=None):
    K, M, N = S.shape
    items = []
    for g in range(M * N):
        i, j = g % M, g // M
        k = K if cnt is None else int(cnt[i, j])
        items.append(np.asarray(S[:k, i, j], dtype=np.uint32).reshape(-1, 1))
    return H.Cell((M, N), items)


def _psi():
    P, P2 = options.bank_from_factors(options.bior_factors())
    return np.asarray(P, dtype=np.float32), np.asarray(P2, dtype=np.float32)


# ---- no device needed ------------------------------------------------------------

def test_gateways_build_and_check_arguments(gw):
    with pytest.raises(H.MexError) as e:
        gw["matchBlocksCPU"](np.zeros((8, 8)), nargout=2)
    assert e.value.ident == "gbm3d:args" and "usage" in e.value.msg
    _, mo = _opts()
    with pytest.raises(H.MexError) as e:
        gw["matchBlocksCPU"](np.zeros((8, 8), dtype=np.float32), 25.0, mo, nargout=2)
    assert e.value.ident == "gbm3d:args" and "double" in e.value.msg
    with pytest.raises(H.MexError) as e:
        gw["matchBlocksCPU"](np.zeros((64, 64)), 25.0, dict(mo, filtType="box"), nargout=2)
    assert e.value.ident == "gbm3d:opts" and e.value.msg == "unrecognized filtering"
    with pytest.raises(H.MexError) as e:
        gw["matchBlocksWie"](np.zeros((64, 64)), np.zeros((64, 32)), 25.0, mo, nargout=3)
    assert e.value.ident == "gbm3d:args"


def test_gateway_rejects_non_separable_bank(gw):
    _, mo = _opts()
    P, P2 = _psi()
    P = P.copy()
    P[0, 1, 0, 0] += 0.3  # break the outer-product structure
    V = np.zeros((32, 32, 16), dtype=np.float32)
    S = _set_to_cell(np.full((16, 2, 2), 1, dtype=np.uint32))
    tau = 25.0 * options.getTau(3, 1)
    with pytest.raises(H.MexError) as e:
        gw["denoiseAndAggregateGPU"](V, S, tau, P, P2, mo, nargout=2)
    assert e.value.ident == "gbm3d:args" and "separable" in e.value.msg


def test_no_device_error(gw):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    _, mo = _opts()
    with pytest.raises(H.MexError) as e:
        gw["matchBlocksCPU"](np.zeros((64, 64)), 25.0, mo, nargout=2)
    assert e.value.ident == "gbm3d:cuda"


def test_filters_from_bank_host_only():
    """The C factorisation returns the exact known banks and agrees with the Python one."""
    import ctypes as C
    from gbm3d_b200._lib import gbm3d_filters, lib
    for fac in (options.bior_factors(), options.haar_factors()):
        P, P2 = [np.asarray(x, np.float32) for x in options.bank_from_factors(fac)]
        f = gbm3d_filters()
        L, Lz = P.shape[0], P.shape[2]
        rc = lib().gbm3d_filters_from_bank(P.ctypes.data_as(C.c_void_p), P2.ctypes.data_as(C.c_void_p), L, Lz,
                                           C.byref(f))
        assert rc == 0
        assert np.array_equal(np.array(f.a_lo_xy[:L]), fac["a_lo_xy"])
        assert np.array_equal(np.array(f.s_hi_xy[:L]), fac["s_hi_xy"])
    # a scaled (unknown) separable bank is split numerically
    fac = options.haar_factors()
    fac = dict(fac, a_lo_xy=fac["a_lo_xy"] * 1.5, s_lo_z=fac["s_lo_z"] * 0.5)
    P, P2 = [np.asfortranarray(x, np.float32) for x in options.bank_from_factors(fac)]
    f = gbm3d_filters()
    assert lib().gbm3d_filters_from_bank(P.ctypes.data_as(C.c_void_p), P2.ctypes.data_as(C.c_void_p), 2, 2,
                                         C.byref(f)) == 0
    Q, Q2 = options.bank_from_factors({k: np.array(getattr(f, k)[:2]) for k in fac})
    assert np.allclose(Q, P, atol=1e-6) and np.allclose(Q2, P2, atol=1e-6)


# ---- on the GPU ---------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("sigma,kw", [(10.0, {}), (0.01, {"numMin": 4}),
                                      (10.0, {"blockSize": 8, "refStride": 3, "matchSize": 24})])
def test_matchBlocksCPU_gateway(gw, sigma, kw):
    """sigma 0.01 with numMin 4: the tolerance 0.005 sigma^2 d^2 admits only the
    reference itself, so every cell is cut to numMin entries."""
    from gbm3d_b200 import api
    _, noisy = synth.noisy_image(64, 80, 10.0, seed=41)
    o, mo = _opts(**kw)
    C, V = gw["matchBlocksCPU"](noisy, sigma, mo, nargout=2)
    S, cnt = _cell_to_set(C, o["numMax"])
    Sa, Va = api.matchBlocksCPU(noisy, sigma, o)
    assert np.array_equal(cnt, Sa.count) and np.array_equal(S, np.asarray(Sa)) and np.array_equal(V, Va)
    if o["numMin"] < o["numMax"]:
        assert (cnt < o["numMax"]).any(), "the tolerance branch should shorten some cells"


@pytest.mark.gpu
def test_denoiseAndAggregateGPU_gateway_gathers_gpuarray(gw, oracle):
    from gbm3d_b200 import api
    from gbm3d_b200.api import _as_set
    _, noisy = synth.noisy_image(64, 64, 25.0, seed=42)
    o, mo = _opts()
    So, Vo, co = oracle.matchBlocksCPU(noisy, 25.0, o, prec=32)
    tau = 25.0 * options.getTau(3, 1)
    P, P2 = _psi()
    U, W = gw["denoiseAndAggregateGPU"](Vo, _set_to_cell(So, co), tau, H.GpuArray(P), H.GpuArray(P2), mo, nargout=2)
    Ua, Wa = api.denoiseAndAggregateGPU(Vo, _as_set(So, co), tau, None, None, o)
    assert np.array_equal(U, Ua) and np.array_equal(W, Wa)


@pytest.mark.gpu
def test_wiener_gateways(gw):
    from gbm3d_b200 import api
    clean, noisy = synth.noisy_image(64, 64, 25.0, seed=43)
    o, mo = _opts()
    pilot = clean + np.random.default_rng(3).normal(0, 2.0, clean.shape)
    C, V1, V2 = gw["matchBlocksWie"](pilot, noisy, 25.0, mo, nargout=3)
    Sa, V1a, V2a = api.matchBlocksWie(pilot, noisy, 25.0, o)
    S, _ = _cell_to_set(C, o["numMax"])
    assert np.array_equal(S, np.asarray(Sa)) and np.array_equal(V1, V1a) and np.array_equal(V2, V2a)
    U, W = gw["denoiseAndAggregateWieFast"](V1, V2, C, 25.0, mo, nargout=2)
    Ua, Wa = api.denoiseAndAggregateWieFast(V1a, V2a, Sa, 25.0, o)
    assert np.array_equal(U, Ua) and np.array_equal(W, Wa)
    sg = np.linspace(10, 40, 64).reshape(8, 8)
    U, W = gw["denoiseAndAggregateWieFast"](V1, V2, C, sg, mo, nargout=2)
    Ua, Wa = api.denoiseAndAggregateWieFast(V1a, V2a, Sa, sg, o)
    assert np.array_equal(U, Ua) and np.array_equal(W, Wa)
    U, W = gw["denoiseAndAggregateWie"](V1 / 255, V2 / 255, C, 25.0 / 255, mo, nargout=2)
    Ua, Wa = api.denoiseAndAggregateWie(V1a / 255, V2a / 255, Sa, 25.0 / 255, o)
    assert np.array_equal(U, Ua) and np.array_equal(W, Wa)


@pytest.mark.gpu
def test_matchBlocksGPU_gateway(gw):
    from gbm3d_b200 import api
    _, noisy = synth.noisy_image(64, 64, 25.0, seed=44)
    o, mo = _opts()
    C = gw["matchBlocksGPU"](noisy, 25.0, mo)
    S, _ = _cell_to_set(C, o["numMax"])
    assert np.array_equal(S, np.asarray(api.matchBlocksGPU(noisy, 25.0, o)))


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,profile", [(70, 90, "default"), (96, 96, "fast")])
def test_GBM3D_driver_through_gateways(gw, m, n, profile):
    """GBM3D.m:21-83 replayed with only the gateways equals the whole-pipeline entry."""
    from gbm3d_b200 import api
    _, I0 = synth.noisy_image(m, n, 25.0, seed=45)
    sigma = 25.0
    o, mo = _opts(profile)
    d = o["blockSize"]
    M, N = -(-m // d) * d, -(-n // d) * d
    I = options.myMirrorPadImage(I0, M, N)
    tau = sigma * options.getTau(o["levels"], o["tauMode"])
    P, P2 = _psi()
    nS = len(o["matchSpins"])
    U = np.zeros((M, N, nS))
    W = np.zeros((M, N, nS))
    U1 = np.zeros((M, N, nS))
    sh = lambda a, s: np.roll(a, (s, s), axis=(0, 1))  # noqa: E731  circshift(a, [s, s])
    for ii, s in enumerate(o["matchSpins"]):
        C, V = gw["matchBlocksCPU"](sh(I, s), sigma, mo, nargout=2)
        u, w = gw["denoiseAndAggregateGPU"](V, C, tau, P, P2, mo, nargout=2)
        U1[:, :, ii], W[:, :, ii] = sh(u, -s), sh(w, -s)
    U1 = U1.sum(axis=2) / W.sum(axis=2)
    for ii, s in enumerate(o["matchSpinsWie"]):
        C, V1, V2 = gw["matchBlocksWie"](sh(U1, s), sh(I, s), sigma, mo, nargout=3)
        u, w = gw["denoiseAndAggregateWieFast"](V1, V2, C, sigma, mo, nargout=2)
        U[:, :, ii], W[:, :, ii] = sh(u, -s), sh(w, -s)
    Uf = (U.sum(axis=2) / W.sum(axis=2))[:m, :n]
    Ua, out = api.GBM3D(I0, sigma, {"profile": profile})
    assert np.array_equal(U1[:m, :n], out["U1"])
    assert np.array_equal(Uf, Ua)


# ---- video gateways ----------------------------------------------------------------

def _vopts(**kw):
    o = {"blockSize": 8.0, "numMax": 16.0, "numMin": 16.0, "wname": "sym", "wnamez": "db", "order": 4.0,
         "orderz": 1.0, "levels": 3.0, "cycleSpin": 2.0, "tauMode": 2.0, "nF": 3.0,
         "matchSpins": np.array([0.0, 4.0])}
    o.update(kw)
    return o


def test_video_gateways_check_arguments(gw):
    with pytest.raises(H.MexError) as e:
        gw["matchBlocksV"](np.zeros((32, 32, 4)), 0.1, _vopts(), nargout=2)
    assert e.value.ident == "gbm3d:args" and "odd number of frames" in e.value.msg
    with pytest.raises(H.MexError) as e:
        gw["matchBlocksV"](np.zeros((32, 32, 3)), 0.1, _vopts(wname="bior"), nargout=2)
    assert e.value.ident == "gbm3d:opts" and "sym" in e.value.msg
    with pytest.raises(H.MexError) as e:
        gw["denoiseAndAggregateV"](0, np.zeros((32, 32, 16), dtype=np.float32), np.zeros((30, 32, 3)),
                                   _set_to_cell(np.ones((16, 4, 4), dtype=np.uint32)), 0.1, _vopts(), nargout=2)
    assert e.value.ident == "gbm3d:args" and "frames must be" in e.value.msg


@pytest.mark.gpu
def test_video_gateways_match_api(gw):
    from gbm3d_b200 import api
    _, noisy = synth.video(32, 40, 3, 25.0, seed=46)
    I, s = noisy / 255.0, 25.0 / 255.0
    C, V = gw["matchBlocksV"](I, s, _vopts(), nargout=2)
    S, cnt = _cell_to_set(C, 16)
    Sa, Va = api.matchBlocksV(I, s, {"blockSize": 8, "nF": 3})
    assert np.array_equal(S, np.asarray(Sa)) and np.all(cnt == 16) and np.array_equal(V, Va)
    U, out = gw["denoiseAndAggregateV"](0, V, I, C, s, _vopts(), nargout=2)
    Ua, outa = api.denoiseAndAggregateV(None, Va, I, Sa, s, {"blockSize": 8, "nF": 3})
    assert np.array_equal(U, Ua) and np.array_equal(out["K"], outa["K"])
    assert out["Z"].shape == (32, 40) and np.all(out["Z"] == 16)


@pytest.mark.gpu
def test_VBM3D_driver_through_gateways(gw):
    """VBM3D.m:24-63 replayed with only the two video gateways equals api.VBM3D
    (Y and nn single, each window's U and out.K added as float32(Y + U))."""
    from gbm3d_b200 import api
    _, noisy = synth.video(30, 44, 5, 25.0, seed=47)
    I0, sigma = noisy / 255.0, 25.0 / 255.0
    d, nF, spins = 8, 3, [0, 4]
    m, n, Kf = I0.shape
    M, N = -(-m // d) * d, -(-n // d) * d
    I2 = np.stack([options.myMirrorPadImage(I0[:, :, k], M, N) for k in range(Kf)], axis=2)
    mo = _vopts(nF=float(nF), matchSpins=np.array(spins, dtype=np.float64))
    hw = (nF - 1) // 2
    acc = np.zeros((m, n, Kf - nF + 1))
    for s in spins:
        Y = np.zeros((M, N, Kf), dtype=np.float32)
        nn = np.zeros((M, N, Kf), dtype=np.float32)
        for jj in range(hw, Kf - hw):
            I3 = np.roll(I2[:, :, jj - hw:jj + hw + 1], (s, s), axis=(0, 1))
            C, V = gw["matchBlocksV"](I3, sigma, mo, nargout=2)
            U, out = gw["denoiseAndAggregateV"](0, V, I3, C, sigma, mo, nargout=2)
            Y[:, :, jj - hw:jj + hw + 1] = (Y[:, :, jj - hw:jj + hw + 1].astype(np.float64) + U).astype(np.float32)
            nn[:, :, jj - hw:jj + hw + 1] = (nn[:, :, jj - hw:jj + hw + 1].astype(np.float64)
                                             + out["K"]).astype(np.float32)
        R = np.roll(Y / nn, (-s, -s), axis=(0, 1))
        acc += R[:m, :n, hw:Kf - hw].astype(np.float64)
    Yd = (acc / len(spins)).astype(np.float32).astype(np.float64)
    Ya, _ = api.VBM3D(I0, sigma, {"blockSize": d, "nF": nF, "matchSpins": spins})
    assert np.array_equal(Yd, Ya)
