"""Denoise one seeded synthetic image with a given option set, a few times:
the command line used to time and profile a single configuration.

    python -m gbm3d_b200.run [--size 4096] [--sigma 25] [--calls 3] [--seed 100]
                             [--opts '{"refStride": 8, "refStrideWie": 6, ...}']

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
    a = ap.parse_args()

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


if __name__ == "__main__":
    main()
