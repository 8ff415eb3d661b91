"""Denoise one seeded synthetic image with a given option set, a few times:
the command line used to time and profile a single configuration.

    python -m gbm3d_b200.run [--size 4096] [--sigma 25] [--calls 3] [--seed 100]
                             [--opts '{"refStride": 8, "refStrideWie": 6, ...}']
    python -m gbm3d_b200.run --video [--frames 32] [--height 720] [--width 1280]
                             [--opts '{"nF": 3}']

With --video, a seeded synthetic video goes through VBM3D (gbm3d_vbm3d_device)
with VBM3D.m's defaults and the JSON overrides (the batched configuration's
video: 32 frames of 1280 x 720, a 3-frame window), and the last call's kernel
families are printed with their CUDA-event times.

The options start from the dense configuration (patch 8, reference stride 3,
group 16, matchSize 32, match spins [0 4] + [0 4], two cycle spins) and the
JSON overrides are applied on top.  Every call runs the whole pipeline on the
device-resident image (gbm3d_denoise_device); the last call is timed with the
library's CUDA events and printed with the PSNR against the clean image.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--sigma", type=float, default=25.0)
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--seed", type=int, default=100)
    ap.add_argument("--opts", default="{}", help="JSON option overrides")
    ap.add_argument("--video", action="store_true", help="run VBM3D on a synthetic video instead")
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--height", type=int, default=720)
    ap.add_argument("--width", type=int, default=1280)
    a = ap.parse_args()
    if a.video:
        return video(a)

    import torch

    from . import _lib, api, autotune, build, options, synth
    build.build()
    ctx = _lib.Context(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    o = options.resolve_opts({"profile": "default"})
    o.update(autotune.BASELINE)
    o.update(json.loads(a.opts))
    clean, noisy = synth.noisy_image(a.size, a.size, a.sigma, seed=a.seed)
    dI = torch.from_numpy(np.asfortranarray(noisy).ravel(order="F")).cuda()
    dU = torch.empty_like(dI)
    for c in range(a.calls):
        ctx.enable_timing(c == a.calls - 1)
        api.GBM3D_device(dI.data_ptr(), a.size, a.size, a.sigma, dU.data_ptr(), o, ctx=ctx)
    st = ctx.stage_times()
    ctx.enable_timing(False)
    torch.cuda.synchronize()
    U = dU.cpu().numpy().reshape(a.size, a.size, order="F")
    print(json.dumps({"size": a.size, "sigma": a.sigma, "opts": json.loads(a.opts), "calls": a.calls,
                      "ms": st[7], "stages_ms": st, "psnr_db": float(options.myPSNR(clean, U, 255)),
                      "launches_per_call": ctx.launch_count()}))


def video(a):
    import ctypes as C

    import torch

    from . import _lib, api, build, options, synth
    m, n, F = a.height, a.width, a.frames
    vo = {"nF": 3}
    vo.update(json.loads(a.opts))
    clean, noisy = synth.video(m, n, F, a.sigma, seed=a.seed)
    build.build()
    ctx = _lib.Context(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    co = api.c_video_opts(vo)
    dI = torch.from_numpy(np.asfortranarray(noisy / 255.0).ravel(order="F").copy()).cuda()
    nout = F - co.videoFrames + 1
    dY = torch.empty(m * n * nout, dtype=torch.float64, device=dI.device)
    for c in range(a.calls):
        ctx.enable_timing(c == a.calls - 1)
        ctx.check(_lib.lib().gbm3d_vbm3d_device(ctx.h, C.c_void_p(dI.data_ptr()), m, n, F, a.sigma / 255.0,
                                                C.byref(co), C.c_void_p(dY.data_ptr())))
    st = ctx.stage_times()
    fam = {k: ctx.kernel_time(k) for k in ("match_video", "wav_analysis", "wav_synthesis", "ht_weights",
                                           "aggregate_video", "clamp", "make_pad", "video_accum", "video_out",
                                           "prep")}
    ctx.enable_timing(False)
    ctx.check(_lib.lib().gbm3d_ctx_synchronize(ctx.h))
    hw = (co.videoFrames - 1) // 2
    Y = dY.cpu().numpy().reshape(m, n, nout, order="F")
    print(json.dumps({"video": [m, n, F], "sigma": a.sigma, "opts": vo, "calls": a.calls, "ms": st[7],
                      "families_ms": {k: {"launches": v[0], "ms": v[1]} for k, v in fam.items()},
                      "psnr_db": float(options.myPSNR(clean[:, :, hw:F - hw], Y * 255.0, 255)),
                      "launches_per_call": ctx.launch_count()}))


if __name__ == "__main__":
    main()
