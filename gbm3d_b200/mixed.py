"""The batched form's mixed workload, timed: one submission holding 64 grey
synthetic images (sizes uniform between 200 x 300 and 2048 x 1536, sigma
uniform in [5, 50]), 8 RGB 1024 x 1024 images (opponent colour space,
luma-driven matching) and a 32-frame 1280 x 720 synthetic video (ellipses
translating 0-3 px per frame) with a +-1-frame temporal window, denoised by
gbm3d_denoise_mixed as eager launches and as one captured CUDA graph.

    python -m gbm3d_b200.mixed [--scale 1.0] [--reps 3] [--opts JSON] [--tune] [--per-image]

Grey and colour images use the dense configuration with the JSON overrides
(or, with --tune, the autotuner's choice on its calibration image, or, with
--per-image, the 'tuned' profile's set for each image's own size and sigma
class, as the bench's batched block gives them); the video
uses VBM3D.m's defaults with a 3-frame window.  --scale shrinks every image
side (a quick run).  Prints one JSON line: megapixels in the batch, device
time per submission (CUDA events on the library stream), MPix/s eager and
replayed, and the launch counts.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def _grey(args):
    from . import synth
    m, n, s, sd = args
    return synth.noisy_image(m, n, s, seed=sd)


def _video(args):
    from . import synth
    m, n, f, s, sd = args
    return synth.video(m, n, f, s, seed=sd)[1]


def workload(scale: float = 1.0, seed: int = 2024, workers: int = 0):
    """Host arrays of the mixed batch: (grey (clean, noisy) pairs, grey sigmas,
    rgb images (m x n x 3), rgb sigmas, video frames m x n x F on [0, 1],
    video sigma on [0, 1]).  Images are generated by a pool of spawned
    processes (call this before any CUDA work)."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import os
    rng = np.random.Generator(np.random.PCG64(seed))
    sz = lambda v: max(64, int(round(v * scale)))  # noqa: E731
    gjobs, gs = [], []
    for k in range(64):
        m, n = sz(rng.uniform(200, 2048)), sz(rng.uniform(300, 1536))
        s = float(rng.uniform(5, 50))
        gjobs.append((m, n, s, seed + 1 + k))
        gs.append(s)
    rjobs, rs = [], []
    for k in range(8):
        s = float(rng.uniform(5, 50))
        rjobs += [(sz(1024), sz(1024), s, seed + 100 + 3 * k + q) for q in range(3)]
        rs.append(s)
    vs = 25.0
    with cf.ProcessPoolExecutor(max_workers=workers or min(32, os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as ex:
        fv = ex.submit(_video, (sz(720), sz(1280), 32, vs, seed + 200))
        grey = list(ex.map(_grey, gjobs))
        planes = [p[1] for p in ex.map(_grey, rjobs)]
        frames = fv.result()
    rgb = [np.stack(planes[3 * k:3 * k + 3], axis=2) for k in range(8)]
    return grey, gs, rgb, rs, frames / 255.0, vs / 255.0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--opts", default="{}", help="JSON overrides of the dense configuration")
    ap.add_argument("--tune", action="store_true", help="use the autotuner's choice for the images")
    ap.add_argument("--per-image", action="store_true",
                    help="each image the 'tuned' profile's set for its own size and sigma class")
    a = ap.parse_args()

    grey_pairs, gs, rgb, rs, frames, vs = workload(a.scale)  # before any CUDA work (spawned pool)
    grey = [p[1] for p in grey_pairs]

    import torch

    from . import _lib, api, autotune, build, options
    build.build()
    ctx = _lib.Context(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    o = options.resolve_opts({"profile": "default"})
    o.update(autotune.BASELINE)
    tuned = None
    if a.tune:
        tuned = autotune.tune(ctx=ctx, log=None)
        o.update(tuned["opts"])
    o.update(json.loads(a.opts))
    vo = {"nF": 3}
    dev = torch.device("cuda", 0)

    def col(x):
        return torch.from_numpy(np.asfortranarray(x).ravel(order="F").copy()).to(dev)

    dg = [col(x).view(x.shape[1], x.shape[0]) for x in grey]
    dr = [tuple(col(x[:, :, q]).view(x.shape[1], x.shape[0]) for q in range(3)) for x in rgb]
    dv = col(frames).view(frames.shape[2], frames.shape[1], frames.shape[0])
    mpix = (sum(x.shape[0] * x.shape[1] for x in grey) + sum(3 * x.shape[0] * x.shape[1] for x in rgb)
            + frames.shape[0] * frames.shape[1] * (frames.shape[2] - 2)) / 1e6

    def timed(use_graph):
        kw = dict(use_graph=use_graph, ctx=ctx)
        if a.per_image:
            kw.update(grey_opts=[{"profile": "tuned"}] * len(dg), rgb_opts=[{"profile": "tuned"}] * len(dr))
        outs = api.GBM3D_mixed(dg, gs, dr, rs, dv, vs, o, vo, **kw)  # warm-up / capture
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.reps):
            api.GBM3D_mixed(dg, gs, dr, rs, dv, vs, o, vo, outputs=outs, **kw)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.reps, ctx.launch_count(), outs

    eager_ms, _, outs = timed(False)
    ref = [u.cpu().numpy().copy() for u in outs[0]]
    graph_ms, graph_launches, outs = timed(True)
    same = all(np.array_equal(r, u.cpu().numpy()) for r, u in zip(ref, outs[0]))
    psnr = []
    for k, (clean, x) in enumerate(grey_pairs[:4]):
        U = outs[0][k].cpu().numpy().reshape(-1).reshape(x.shape, order="F")
        psnr.append(round(float(options.myPSNR(clean, U, 255) - options.myPSNR(clean, x, 255)), 3))
    print(json.dumps({"workload": "64 grey (200x300 .. 2048x1536, sigma 5-50) + 8 RGB 1024^2 + 32-frame 1280x720 "
                                  "video, +-1 frame", "scale": a.scale, "megapixels": mpix,
                      "opts": "per image: the 'tuned' profile" if a.per_image else {
                          k: o[k] for k in ("refStride", "refStrideWie", "matchSize", "matchSpins",
                                            "matchSpinsWie", "cycleSpin", "form")},
                      "eager_ms": eager_ms, "graph_ms": graph_ms, "eager_mpix_s": mpix / (eager_ms / 1e3),
                      "graph_mpix_s": mpix / (graph_ms / 1e3), "graph_launches_per_call": graph_launches,
                      "graph_equals_eager": same,
                      "psnr_gain_db_first4": psnr, "tuned": None if tuned is None else tuned["chosen"]}))


if __name__ == "__main__":
    main()
