"""Host logic and the C ABI surface (no GPU needed)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from gbm3d_b200 import options


def test_profiles_match_reference():
    d = options.setBM3Dopts("default")
    assert d["matchSpins"] == [0, 4] and d["matchSpinsWie"] == [0, 4]
    assert (d["blockSize"], d["blockSizeWie"], d["matchSize"], d["numMax"]) == (16, 8, 32, 16)
    f = options.setBM3Dopts("fast")
    assert f["matchSpins"] == [0, 4, 6] and f["matchSpinsWie"] == [0]
    s = options.setBM3Dopts("superFast")
    assert s["blockSize"] == 32 and s["Wiener"] is False
    a = options.setBM3Dopts("accuracy")
    assert a["matchSpinsWie"] == [0, 4, 6]
    assert options.setBM3Dopts("nonsense") == d


def test_checkBM3Dopts_defaults():
    o = options.checkBM3Dopts({"blockSize": 8})
    assert o["matchSize"] == 32 and o["matchSpins"] == [0, 4] and o["cycleSpin"] == 2
    o = options.checkBM3Dopts({"blockSize": 64})
    assert o["matchSize"] == 64


def test_profile_overrides_fields():
    o = options.resolve_opts({"profile": "fast", "numMax": 4})
    assert o["numMax"] == 16  # GBM3D.m:16-19 replaces every field


def test_getTau_modes():
    t = options.getTau(3, 1)
    assert np.allclose(t[:, 0], [3.3, 3.0, 2.7]) and np.allclose(t, t[:, :1])
    t2 = options.getTau(3, 2)
    assert np.allclose(t2[0], [3.3, 3.3, 3.3, 3.8, 3.8, 3.8, 4.3])
    t4 = options.getTau(2, 4)
    assert np.allclose(t4[1], [2.9] * 3 + [3.4] * 3 + [3.9])


def test_getTau_matches_oracle(oracle):
    for mode in (1, 2, 3, 4):
        assert np.array_equal(options.getTau(3, mode), oracle.get_tau(3, mode))


def test_filter_bank_roundtrip():
    Psi, Psi2 = options.getWaveFilters3Dbior()
    assert Psi.shape == (10, 10, 2, 8) and Psi.dtype == np.float32
    fac = options.factors_from_bank(Psi, Psi2)
    ref = options.bior_factors()
    for k in ref:
        assert np.array_equal(fac[k], ref[k])
    # a scaled (non-catalogued) separable bank is factorised numerically
    P3, P4 = options.bank_from_factors({k: v * (1.5 if k.startswith("a_") else 1.0) for k, v in ref.items()})
    f2 = options.factors_from_bank(P3, P4)
    Q, Q2 = options.bank_from_factors(f2)
    assert np.allclose(Q, P3, atol=1e-5) and np.allclose(Q2, P4, atol=1e-5)
    with pytest.raises(ValueError):
        bad = np.random.default_rng(0).normal(size=(10, 10, 2, 8)).astype(np.float32)
        options.factors_from_bank(bad, bad)


def test_mirror_pad():
    I = np.arange(20.0).reshape(4, 5, order="F")
    O = options.myMirrorPadImage(I, 6, 8)
    assert np.array_equal(O[:4, :5], I)
    assert np.array_equal(O[4:6, :5], np.flipud(I[2:4, :]))
    assert np.array_equal(O[:4, 5:8], np.fliplr(I[:, 2:5]))


def test_mirror_pad_matches_oracle(oracle):
    rng = np.random.default_rng(0)
    I = np.asfortranarray(rng.normal(size=(13, 11)))
    O = np.zeros((16, 16), order="F")
    oracle.lib().orc_mirror_pad(I.ctypes.data_as(C.c_void_p), 13, 11, O.ctypes.data_as(C.c_void_p), 16, 16)
    assert np.array_equal(O, options.myMirrorPadImage(I, 16, 16))


def test_psnr():
    a = np.zeros((4, 4))
    b = np.full((4, 4), 1.0)
    assert abs(options.myPSNR(a, b, 255) - 20 * np.log10(255)) < 1e-12


def test_dct_matrices_agree(oracle):
    from oracle import fft_route
    T, Ti = oracle.dct_matrices(8)
    assert np.allclose(T, fft_route.dct_matrix(8), atol=1e-15)
    assert np.allclose(Ti @ T, np.eye(8), atol=1e-14)


def test_library_builds_and_exports_every_declared_symbol():
    from gbm3d_b200 import _lib, build
    path = build.build()
    assert os.path.exists(path)
    L = C.CDLL(path)
    syms = _lib.header_symbols()
    assert len(syms) >= 18
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the binding
    assert set(syms) <= set(_lib._SIGS)
    # nm confirms the exports are plain C symbols
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    for s in syms:
        assert f" T {s}\n" in out or out.endswith(f" T {s}"), s


def test_library_option_helpers_match_host():
    """Calls that need no device: profiles, tau table and filter factors."""
    from gbm3d_b200 import _lib
    L = _lib.lib()
    for prof in ("default", "fast", "superFast", "accuracy"):
        c = _lib.gbm3d_opts()
        L.gbm3d_default_opts(prof.encode(), C.byref(c))
        o = options.setBM3Dopts(prof)
        assert (c.numMax, c.blockSize, c.blockSizeWie, c.matchSize, c.levels, c.cycleSpin) == \
            (o["numMax"], o["blockSize"], o["blockSizeWie"], o["matchSize"], o["levels"], o["cycleSpin"])
        assert list(c.matchSpins[:c.nMatchSpins]) == o["matchSpins"]
        assert list(c.matchSpinsWie[:c.nMatchSpinsWie]) == o["matchSpinsWie"]
        assert bool(c.Wiener) == o["Wiener"]
    t = np.zeros((3, 7), order="F")
    L.gbm3d_get_tau(3, 2, t.ctypes.data_as(C.c_void_p))
    assert np.array_equal(t, options.getTau(3, 2))
    f = _lib.gbm3d_filters()
    L.gbm3d_bior_filters(C.byref(f))
    ref = options.bior_factors()
    assert np.array_equal(np.array(f.a_lo_xy[:10]), ref["a_lo_xy"])
    assert np.array_equal(np.array(f.s_hi_xy[:10]), ref["s_hi_xy"])


def test_no_device_fails_loudly():
    """Without a usable CUDA device the library reports an error (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from gbm3d_b200 import _lib
    with pytest.raises(_lib.GBM3DError):
        _lib.Context(0)


def test_autotune_search_space():
    """Candidates keep patch, group and wavelet; strides never exceed the patch."""
    from gbm3d_b200 import autotune
    cs = autotune.candidates()
    assert len(cs) == len({json_key(c) for c in cs})
    for c in cs:
        assert 1 <= c["refStride"] <= 8 and 1 <= c["refStrideWie"] <= 8
        assert c["matchSpins"] in ([0], [0, 4]) and c["matchSpinsWie"][0] == 0
        assert c["cycleSpin"] in (1, 2) and c["matchSize"] in (24, 32)
        assert not ({"blockSize", "blockSizeWie", "numMax", "wname", "levels"} & set(c))
    assert not autotune.candidates(strides1=(9,))


def json_key(d):
    import json
    return json.dumps(d, sort_keys=True)


def test_autotune_select_rule():
    """The fastest row within budget - margin of the baseline wins; untimed rows never do."""
    from gbm3d_b200 import autotune
    rows = [{"baseline": True, "opts": {}, "psnr": 30.0, "ms": 100.0},
            {"opts": {"refStride": 8}, "psnr": 29.90, "ms": 10.0},   # 0.10 dB worse: out
            {"opts": {"refStride": 6}, "psnr": 29.975, "ms": 20.0},  # 0.025 dB worse: in at margin 0.02
            {"opts": {"refStride": 4}, "psnr": 30.2, "ms": 40.0},
            {"opts": {"refStride": 5}, "psnr": 29.0}]                # not timed
    assert autotune.select(rows, 0.05, 0.02)["opts"] == {"refStride": 6}
    assert autotune.select(rows, 0.05, 0.04)["opts"] == {"refStride": 4}
    assert autotune.select(rows, 0.2, 0.0)["opts"] == {"refStride": 8}
    assert autotune.select(rows[:1], 0.05)["baseline"]


def test_tuned_profile_lookup():
    """The 'tuned' profile: the largest calibrated size class not above the
    image's smaller side, the sigma class nearest in log scale, the dense
    configuration below the smallest class."""
    from gbm3d_b200 import options
    table = {"classes": [
        {"size": 512, "sigma": 10.0, "opts": {"refStride": 6, "refStrideWie": 4}},
        {"size": 512, "sigma": 25.0, "opts": {"refStride": 6, "refStrideWie": 5}},
        {"size": 2048, "sigma": 25.0, "opts": {"refStride": 8, "refStrideWie": 6, "form": "tensor"}},
        {"size": 2048, "sigma": 50.0, "opts": {"refStride": 8, "refStrideWie": 7}}]}
    o = options.tuned_opts(600, 700, 12.0, table)
    assert (o["refStride"], o["refStrideWie"]) == (6, 4)
    o = options.tuned_opts(4096, 3000, 26.0, table)
    assert (o["refStride"], o["refStrideWie"], o["form"]) == (8, 6, "tensor")
    o = options.tuned_opts(4096, 4096, 40.0, table)
    assert (o["refStride"], o["refStrideWie"]) == (8, 7)
    o = options.tuned_opts(300, 4096, 25.0, table)  # below every class: the dense configuration
    assert (o["refStride"], o["refStrideWie"], o["cycleSpin"], o["matchSpins"]) == (3, 3, 2, [0, 4])
    with pytest.raises(ValueError):
        options.resolve_opts({"profile": "tuned"})
    # sigma class rounded down: 40 -> 25 (nearest would be 50), 24 -> 10, below every class -> the smallest
    o = options.tuned_opts(4096, 4096, 40.0, table, sigma_below=True)
    assert (o["refStride"], o["refStrideWie"]) == (8, 6)
    o = options.tuned_opts(600, 700, 24.0, table, sigma_below=True)
    assert (o["refStride"], o["refStrideWie"]) == (6, 4)
    o = options.tuned_opts(600, 700, 5.0, table, sigma_below=True)
    assert (o["refStride"], o["refStrideWie"]) == (6, 4)
    o = options.tuned_opts(4096, 4096, 20.0, table, sigma_below=True)  # only 25 and 50 at 2048: the smallest
    assert (o["refStride"], o["refStrideWie"]) == (8, 6)


def test_bench_batch_rules():
    """The batched block's per-image option rules on the calibrated table:
    'calibrated' is the 'tuned' profile itself (dense below the smallest
    calibrated class), 'floor512'
    lifts small images into the 512 class, 'uniform512' gives every image the
    512 / sigma 25 set."""
    import bench
    from gbm3d_b200 import options
    assert bench.BATCH_RULE in bench.BATCH_RULES
    uniform = options.tuned_opts(512, 512, 25.0)
    small, big = (200, 240), (1500, 1200)  # small: below every calibrated size class
    sets = {r: (bench.batch_set(r, small, 40.0, uniform), bench.batch_set(r, big, 40.0, uniform))
            for r in bench.BATCH_RULES}
    assert sets["calibrated"][0]["refStride"] == 3 and sets["calibrated"][0]["cycleSpin"] == 2  # dense
    assert sets["calibrated"][1] == options.tuned_opts(1024, 1024, 50.0)  # 40 is nearer 50 than 25 in log scale
    assert sets["calibrated_sigma_below"][1] == options.tuned_opts(1024, 1024, 25.0)
    assert sets["floor512"][0] == options.tuned_opts(512, 512, 40.0)
    assert sets["uniform512"] == (uniform, uniform)
    with pytest.raises(ValueError):
        bench.batch_set("nearest", small, 25.0, uniform)


def test_mixed_option_sets():
    """A mixed submission with opts of the 'tuned' profile gives every image
    its own entry (resolved at its size and sigma by the binding); explicit
    per-image lists win, and other profiles stay call-level."""
    from gbm3d_b200 import api, options
    tuned = {"profile": "tuned"}
    o, g, c = api.mixed_option_sets(tuned, None, None, 3, 2)
    assert g == [tuned] * 3 and c == [tuned] * 2
    assert options.resolve_opts(o)["refStride"] == 3  # the dense configuration, used by no image
    own = [{"profile": "fast"}] * 3
    o, g, c = api.mixed_option_sets(tuned, own, None, 3, 1)
    assert g is own and c == [tuned]
    o, g, c = api.mixed_option_sets({"profile": "default"}, None, None, 3, 2)
    assert o == {"profile": "default"} and g is None and c is None
