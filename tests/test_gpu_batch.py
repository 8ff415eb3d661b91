"""Batched, colour, mixed and asynchronous entries, and the autotuner, on the GPU.

Batch: images of uneven sizes and noise levels denoised in one call, first
eagerly while the launch sequence is captured into a CUDA graph, then by
replaying the graph; every output must equal the single-image pipeline's bit
for bit.  Colour: the opponent-space pipeline with luma-driven matching; on a
grey image (R = G = B) the chroma channels are constant, so every output
channel must equal the grey pipeline at the luma noise level sigma / sqrt(3)
(to float rounding of the constant chroma).  Mixed submissions (grey, colour
and video in one captured graph) and the asynchronous host-stream entry must
reproduce each image's single-call result bit for bit; the autotuner's choice
must stay within its PSNR budget and run through the whole-image entry.
"""
import numpy as np
import pytest

from gbm3d_b200 import options, synth

pytestmark = pytest.mark.gpu


def _dense(**kw):
    o = options.resolve_opts({"profile": "default"})
    o.update(blockSize=8, blockSizeWie=8, matchSize=32, refStride=3, refStrideWie=3)
    o.update(kw)
    return o


@pytest.mark.parametrize("opts", [{"profile": "default"}, "dense"])
def test_batch_graph_matches_single_images(gpu, opts):
    import torch
    from gbm3d_b200 import api
    o = _dense() if opts == "dense" else options.resolve_opts(opts)
    sizes = [(96, 80), (130, 70), (64, 64), (128, 160), (70, 90)]
    sig = [10.0, 25.0, 50.0, 15.0, 35.0]
    imgs, ref = [], []
    for k, ((m, n), s) in enumerate(zip(sizes, sig)):
        _, noisy = synth.noisy_image(m, n, s, seed=60 + k)
        imgs.append(torch.from_numpy(np.asfortranarray(noisy).ravel(order="F").copy()).cuda().view(n, m))
        ref.append(api.GBM3D(noisy, s, o)[0])
    for use_graph, calls in ((False, 1), (True, 3)):  # capture, then two replays
        for _ in range(calls):
            outs = api.GBM3D_batch(imgs, sig, o, use_graph=use_graph)
            for k, (m, n) in enumerate(sizes):
                got = outs[k].cpu().numpy().reshape(-1).reshape(m, n, order="F")
                assert np.array_equal(got, ref[k]), f"image {k} (graph={use_graph})"


def test_rgb_grey_image_equals_grey_pipeline(gpu):
    from gbm3d_b200 import api
    _, noisy = synth.noisy_image(96, 96, 25.0, seed=71)
    rgb = np.stack([noisy] * 3, axis=2)
    o = _dense()
    out = api.GBM3D_rgb(rgb, 25.0, o)
    grey, _ = api.GBM3D(noisy, 25.0 / np.sqrt(3.0), o)
    for k in range(3):  # the constant chroma (offset 128) comes back up to float rounding
        assert np.abs(out[:, :, k] - grey).max() <= 1e-3


def test_rgb_denoises_colour_noise(gpu):
    from gbm3d_b200 import api
    rng = np.random.default_rng(5)
    base, other = synth.clean_image(128, 128, seed=80), synth.clean_image(128, 128, seed=81)
    # correlated channels, as in natural colour images: one structure, tinted
    clean = np.stack([0.9 * base + 0.1 * other, 0.7 * base + 30, 0.5 * base + 0.2 * other + 50], axis=2)
    noisy = clean + 25.0 * rng.standard_normal(clean.shape)
    o = _dense()
    out = api.GBM3D_rgb(noisy, 25.0, o)
    per_channel = np.stack([api.GBM3D(noisy[:, :, k], 25.0, o)[0] for k in range(3)], axis=2)
    p_rgb, p_sep = options.myPSNR(clean, out, 255), options.myPSNR(clean, per_channel, 255)
    print(f"colour: noisy {options.myPSNR(clean, noisy, 255):.2f} dB, per-channel {p_sep:.2f} dB, "
          f"opponent + luma matching {p_rgb:.2f} dB")
    assert p_rgb > options.myPSNR(clean, noisy, 255) + 4 and p_rgb > p_sep - 0.5


def test_autotune_choice_runs_within_budget(gpu):
    """A small search: the chosen options denoise the calibration image within
    budget - margin of the dense baseline and no slower than it, and they run
    through the whole-image entry point."""
    from gbm3d_b200 import api, autotune
    cands = [dict(c, matchSize=32) for c in autotune.candidates(strides1=(8,), strides2=(4, 8), searches=(32,),
                                                                 cycle_spins=(2,))]
    t = autotune.tune(size=256, sigma=25.0, cands=cands, seed=11, log=None)
    best, base = t["chosen"], t["baseline"]
    assert best["ms"] <= base["ms"]
    assert best.get("baseline") or best["psnr"] >= base["psnr"] - (t["budget_db"] - t["margin_db"])
    assert t["evaluated"] == len(cands) + 1
    clean, noisy = synth.noisy_image(256, 256, 25.0, seed=11)
    U, _ = api.GBM3D(noisy, 25.0, t["opts"])
    assert abs(options.myPSNR(clean, U, 255) - (best["psnr"])) < 1e-9


@pytest.mark.parametrize("lanes", [1, 3])
def test_mixed_batch_matches_single_entries(gpu, lanes):
    """Grey images, colour images and a video in one submission: eager, then
    captured, then replayed twice; every output equals its own single-image
    entry's bit for bit, on one lane and on three concurrent lanes."""
    from gbm3d_b200 import api
    api.context().set_lanes(lanes)
    try:
        _mixed_case()
    finally:
        api.context().set_lanes(1)


def _mixed_case():
    import torch
    from gbm3d_b200 import api
    o = _dense()
    dev = torch.device("cuda", 0)

    def col(a):
        return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)

    grey_sizes, grey_sig = [(96, 80), (64, 72), (120, 96)], [10.0, 30.0, 45.0]
    grey = [col(synth.noisy_image(m, n, s, seed=80 + k)[1]).view(n, m)
            for k, ((m, n), s) in enumerate(zip(grey_sizes, grey_sig))]
    grey_ref = [api.GBM3D(synth.noisy_image(m, n, s, seed=80 + k)[1], s, o)[0]
                for k, ((m, n), s) in enumerate(zip(grey_sizes, grey_sig))]
    rgb_sizes, rgb_sig = [(80, 64), (64, 96)], [20.0, 35.0]
    rgb, rgb_ref = [], []
    for k, ((m, n), s) in enumerate(zip(rgb_sizes, rgb_sig)):
        planes = np.stack([synth.noisy_image(m, n, s, seed=90 + 3 * k + q)[1] for q in range(3)], axis=2)
        rgb.append(tuple(col(planes[:, :, q]).view(n, m) for q in range(3)))
        rgb_ref.append(api.GBM3D_rgb(planes, s, o))
    vm, vn, vf, vs = 48, 40, 5, 25.0
    _, frames = synth.video(vm, vn, vf, vs, seed=7)
    frames = frames / 255.0
    vo = {"blockSize": 8, "nF": 3}
    video = col(frames).view(vf, vn, vm)
    video_ref = api.VBM3D(frames, vs / 255.0, vo)[0]
    for use_graph, calls in ((False, 1), (True, 3)):
        for _ in range(calls):
            g_out, c_out, v_out = api.GBM3D_mixed(grey, grey_sig, rgb, rgb_sig, video, vs / 255.0, o, vo,
                                                  use_graph=use_graph)
            for k, (m, n) in enumerate(grey_sizes):
                got = g_out[k].cpu().numpy().reshape(-1).reshape(m, n, order="F")
                assert np.array_equal(got, grey_ref[k]), f"grey image {k} (graph={use_graph})"
            for k, (m, n) in enumerate(rgb_sizes):
                for q in range(3):
                    got = c_out[k][q].cpu().numpy().reshape(-1).reshape(m, n, order="F")
                    assert np.array_equal(got, rgb_ref[k][:, :, q]), f"colour image {k} plane {q} (graph={use_graph})"
            got = v_out.cpu().numpy().reshape(-1).reshape(video_ref.shape, order="F")
            assert np.array_equal(got, video_ref), f"video (graph={use_graph})"
    # a different geometry is captured anew
    g_out, _, _ = api.GBM3D_mixed(grey[:1], grey_sig[:1], opts=o)
    m, n = grey_sizes[0]
    assert np.array_equal(g_out[0].cpu().numpy().reshape(-1).reshape(m, n, order="F"), grey_ref[0])


def test_mixed_batch_per_image_options(gpu):
    """Each image of a mixed submission with its own option set (grey_opts /
    rgb_opts: strides, spins and cycle spins differing between images) gets
    what its single-image entry gives with that set, bit for bit: eager, then
    captured and replayed, on two lanes."""
    import torch
    from gbm3d_b200 import api
    dev = torch.device("cuda", 0)

    def col(a):
        return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)

    sets = [_dense(), _dense(refStride=8, refStrideWie=4, matchSpins=[0], matchSpinsWie=[0, 2], cycleSpin=1),
            _dense(refStride=6, refStrideWie=6, matchSpins=[0], matchSpinsWie=[0], cycleSpin=2)]
    grey_sizes, grey_sig = [(96, 80), (64, 72), (120, 96)], [10.0, 30.0, 45.0]
    noisy = [synth.noisy_image(m, n, s, seed=180 + k)[1] for k, ((m, n), s) in enumerate(zip(grey_sizes, grey_sig))]
    grey = [col(x).view(n, m) for x, (m, n) in zip(noisy, grey_sizes)]
    grey_ref = [api.GBM3D(x, s, o)[0] for x, s, o in zip(noisy, grey_sig, sets)]
    rgb_sizes, rgb_sig = [(80, 64), (64, 96)], [20.0, 35.0]
    rgb_sets = [sets[1], sets[2]]
    rgb, rgb_ref = [], []
    for k, ((m, n), s) in enumerate(zip(rgb_sizes, rgb_sig)):
        planes = np.stack([synth.noisy_image(m, n, s, seed=190 + 3 * k + q)[1] for q in range(3)], axis=2)
        rgb.append(tuple(col(planes[:, :, q]).view(n, m) for q in range(3)))
        rgb_ref.append(api.GBM3D_rgb(planes, s, rgb_sets[k]))
    api.context().set_lanes(2)
    try:
        for use_graph, calls in ((False, 1), (True, 2)):
            for _ in range(calls):
                g_out, c_out, _ = api.GBM3D_mixed(grey, grey_sig, rgb, rgb_sig, opts=_dense(), use_graph=use_graph,
                                                  grey_opts=sets, rgb_opts=rgb_sets)
                for k, (m, n) in enumerate(grey_sizes):
                    got = g_out[k].cpu().numpy().reshape(-1).reshape(m, n, order="F")
                    assert np.array_equal(got, grey_ref[k]), f"grey image {k} (graph={use_graph})"
                for k, (m, n) in enumerate(rgb_sizes):
                    for q in range(3):
                        got = c_out[k][q].cpu().numpy().reshape(-1).reshape(m, n, order="F")
                        assert np.array_equal(got, rgb_ref[k][:, :, q]), f"colour image {k} plane {q}"
    finally:
        api.context().set_lanes(1)
    with pytest.raises(api.GBM3DError):
        api.GBM3D_mixed(grey, grey_sig, opts=_dense(), grey_opts=sets[:2])


def test_async_host_stream_matches_sync(gpu):
    """gbm3d_denoise_async over a stream of host images (sizes changing along
    the way) gives every image the synchronous entry's result bit for bit, and
    a non-finite input is reported at synchronisation."""
    import torch
    from gbm3d_b200 import _lib, api
    o = _dense()
    ctx = _lib.Context(0)
    sizes = [(96, 80), (96, 80), (130, 70), (96, 80), (64, 64)]
    ins, outs, refs = [], [], []
    for k, (m, n) in enumerate(sizes):
        _, noisy = synth.noisy_image(m, n, 25.0, seed=300 + k)
        ins.append(torch.from_numpy(np.asfortranarray(noisy).ravel(order="F").copy()).pin_memory())
        outs.append(torch.zeros_like(ins[-1]).pin_memory())
        refs.append(api.GBM3D(noisy, 25.0, o)[0])
    for _ in range(2):
        for (m, n), hI, hU in zip(sizes, ins, outs):
            api.GBM3D_async(hI.data_ptr(), m, n, 25.0, hU.data_ptr(), o, ctx=ctx)
        ctx.synchronize()
        for k, ((m, n), hU) in enumerate(zip(sizes, outs)):
            assert np.array_equal(hU.numpy().reshape(m, n, order="F"), refs[k]), f"image {k}"
    bad = ins[0].clone().pin_memory()
    bad[5] = float("nan")
    api.GBM3D_async(bad.data_ptr(), 96, 80, 25.0, outs[0].data_ptr(), o, ctx=ctx)
    with pytest.raises(_lib.GBM3DError):
        ctx.synchronize()
    ctx.synchronize()  # the report clears the status
    ctx.close()
