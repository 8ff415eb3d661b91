"""Learned pilot: training, inference and the per-image fallback gate.

The network (csrc/pilot.cu) stands in for step 1 of GBM3D: it maps the noisy
image and sigma to an estimate of the step-1 (hard-threshold) output, which
the Wiener step then refines.  It is trained on (noisy, step-1 output) pairs
that this library's plain GBM3D produces on seeded synthetic images, with the
library's own forward / backward / Adam kernels; PyTorch only holds device
memory.

    python -m gbm3d_b200.pilot train [--steps N] [--out PATH]

The fallback gate: per image, on a sampled central tile, the step-1 quality of
the network and of the plain step 1 is estimated without the clean image by
recorruption (Pang et al., "Recorrupted-to-Recorrupted", 2021): with z ~ N(0,1),
y1 = y + sigma z and y2 = y - sigma z carry independent noise, so
mean((f(y1) - y2)^2) - 2 sigma^2 is an unbiased estimate of f's error at noise
level sqrt(2) sigma.  Both methods see the same y1, y2, so the common noise in
the two estimates cancels in their ratio; when the network's estimated PSNR is
more than 0.1 dB below the plain step's, the image takes the plain path.
"""
from __future__ import annotations

import argparse
import contextlib
import ctypes as C
import math
import os
import time

import numpy as np

from . import api, options, synth
from ._lib import context, lib

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights", "pilot_dense.npy")
LAYERS = [(2, 48)] + [(48, 48)] * 6 + [(48, 1)]


def dense_opts(**kw) -> dict:
    """The step-1 configuration the pilot imitates: patch 8, stride 3, group 16,
    search +-16, bior1.5 x Haar, 3 levels, 2 cycle spins, match spins [0 4]."""
    o = options.resolve_opts({"profile": "default"})
    o.update(blockSize=8, blockSizeWie=8, matchSize=32, numMax=16, numMin=16, refStride=3, refStrideWie=3)
    o.update(kw)
    return o


@contextlib.contextmanager
def shared_stream(ctx=None):
    """Run torch's work and the library's on one explicit stream, so device
    buffers torch fills are ready when the library reads them (and back)."""
    import torch
    ctx = ctx or context()
    torch.cuda.synchronize()  # work torch queued earlier (on any stream) is done
    s = torch.cuda.Stream(torch.device("cuda", ctx.device))
    ctx.set_stream(s.cuda_stream)
    try:
        with torch.cuda.stream(s):
            yield s
    finally:
        s.synchronize()
        ctx.set_stream(None)


def param_count() -> int:
    return int(lib().gbm3d_pilot_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights (the last layer scaled by 0.1), zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for li, (ci, co) in enumerate(LAYERS):
        std = math.sqrt(2.0 / (9 * ci)) * (0.1 if li == len(LAYERS) - 1 else 1.0)
        parts += [rng.normal(0, std, 9 * co * ci), np.zeros(co)]
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == param_count()
    return p


def set_params(params, ctx=None) -> None:
    ctx = ctx or context()
    p = np.ascontiguousarray(params, dtype=np.float32)
    if p.size != param_count():
        raise ValueError(f"expected {param_count()} parameters, got {p.size}")
    ctx.check(lib().gbm3d_pilot_set_params(ctx.h, p.ctypes.data_as(C.c_void_p)))


def get_params(ctx=None) -> np.ndarray:
    ctx = ctx or context()
    p = np.zeros(param_count(), dtype=np.float32)
    ctx.check(lib().gbm3d_pilot_get_params(ctx.h, p.ctypes.data_as(C.c_void_p)))
    return p


def load(path: str = WEIGHTS, ctx=None) -> np.ndarray:
    p = np.load(path).astype(np.float32)
    set_params(p, ctx)
    return p


def forward_device(img, sig, out, ctx=None) -> None:
    """img, out: torch float32 [N, H, W] on the device; sig: torch float32 [N].
    Runs on torch's current stream and returns when the output is ready."""
    import torch
    ctx = ctx or context()
    N, H, W = img.shape
    torch.cuda.current_stream().synchronize()
    ctx.check(lib().gbm3d_pilot_forward(ctx.h, C.c_void_p(img.data_ptr()), C.c_void_p(sig.data_ptr()), N, H, W,
                                        C.c_void_p(out.data_ptr())))
    ctx.check(lib().gbm3d_ctx_synchronize(ctx.h))


def pilot_image(I, sigma, ctx=None) -> np.ndarray:
    """The network's step-1 estimate of one column-major image (host arrays)."""
    import torch
    I = np.asfortranarray(I, dtype=np.float32)
    m, n = I.shape
    dev = torch.device("cuda", (ctx or context()).device)
    img = torch.from_numpy(I.ravel(order="F").copy()).to(dev).view(1, n, m)
    out = torch.empty_like(img)
    forward_device(img, torch.tensor([float(sigma)], device=dev), out, ctx)
    torch.cuda.synchronize()
    return out.view(-1).cpu().numpy().reshape(m, n, order="F").astype(np.float64)


# ---- training data: (noisy, step-1 output) pairs from the plain pipeline ---------------

def make_dataset(n_crops: int = 20000, crop: int = 128, size: int = 1024, seed: int = 7, ctx=None, log=print):
    """Crops of seeded synthetic images (sigma ~ U[5, 50] per image) and their
    plain step-1 estimates (dense configuration).  Returns torch tensors on the
    device: noisy [N, crop, crop], target [N, crop, crop], sigma [N]."""
    import torch
    ctx = ctx or context()
    dev = torch.device("cuda", ctx.device)
    per = (size // crop) ** 2
    n_img = -(-n_crops // per)
    rng = np.random.default_rng(seed)
    o1 = dense_opts(Wiener=False)
    noisy_l, tgt_l, sig_l = [], [], []
    t0 = time.time()
    for k in range(n_img):
        sigma = float(rng.uniform(5.0, 50.0))
        _, noisy = synth.noisy_image(size, size, sigma, seed=int(seed * 100003 + k))
        U1, _ = api.GBM3D(noisy, sigma, o1, ctx=ctx)
        # column-major m x n images are [n][m] row-major arrays: crops of the transpose
        nt = torch.from_numpy(np.ascontiguousarray(noisy.T, dtype=np.float32)).to(dev)
        ut = torch.from_numpy(np.ascontiguousarray(U1.T, dtype=np.float32)).to(dev)
        c = nt.unfold(0, crop, crop).unfold(1, crop, crop).reshape(-1, crop, crop)
        u = ut.unfold(0, crop, crop).unfold(1, crop, crop).reshape(-1, crop, crop)
        noisy_l.append(c.contiguous())
        tgt_l.append(u.contiguous())
        sig_l.append(torch.full((c.shape[0],), sigma, device=dev))
        if log and (k % 50 == 0 or k == n_img - 1):
            log(f"dataset: image {k + 1}/{n_img}, {time.time() - t0:.1f}s")
    return (torch.cat(noisy_l)[:n_crops].contiguous(), torch.cat(tgt_l)[:n_crops].contiguous(),
            torch.cat(sig_l)[:n_crops].contiguous())


def train(steps: int = 3000, batch: int = 32, lr: float = 1e-3, n_crops: int = 20000, crop: int = 128,
          seed: int = 0, ctx=None, data=None, log=print, params=None,
          max_seconds: float | None = None) -> tuple[np.ndarray, list]:
    """Adam on mean((pilot - step1)^2) with the library's kernels; cosine-decayed
    lr.  max_seconds bounds the wall time (the schedule then ends early)."""
    import torch
    ctx = ctx or context()
    dev = torch.device("cuda", ctx.device)
    noisy, target, sig = data if data is not None else make_dataset(n_crops, crop, ctx=ctx, log=log)
    set_params(init_params(seed) if params is None else params, ctx)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    xb = torch.empty((batch,) + tuple(noisy.shape[1:]), device=dev)
    tb = torch.empty_like(xb)
    sb = torch.empty((batch,), device=dev)
    losses = []
    loss = C.c_float(0.0)
    t0 = time.time()
    with shared_stream(ctx):
        _train_loop(ctx, steps, lr, noisy, target, sig, gen, xb, tb, sb, losses, loss, t0, log, max_seconds)
    return get_params(ctx), losses


def _train_loop(ctx, steps, lr, noisy, target, sig, gen, xb, tb, sb, losses, loss, t0, log, max_seconds=None):
    import torch
    dev = xb.device
    batch = xb.shape[0]
    for step in range(steps):
        idx = torch.randint(0, noisy.shape[0], (batch,), generator=gen).to(dev)
        torch.index_select(noisy, 0, idx, out=xb)
        torch.index_select(target, 0, idx, out=tb)
        torch.index_select(sig, 0, idx, out=sb)
        lr_t = lr * 0.5 * (1 + math.cos(math.pi * step / steps))
        ctx.check(lib().gbm3d_pilot_train_step(ctx.h, C.c_void_p(xb.data_ptr()), C.c_void_p(tb.data_ptr()),
                                               C.c_void_p(sb.data_ptr()), batch, xb.shape[1], xb.shape[2],
                                               C.c_float(max(lr_t, 1e-6)), C.byref(loss)))
        losses.append(float(loss.value))
        if max_seconds is not None and time.time() - t0 > max_seconds:
            if log:
                log(f"stopping at step {step}: {max_seconds}s budget")
            break
        if log and (step % 200 == 0 or step == steps - 1):
            log(f"step {step}: loss {np.mean(losses[-50:]):.3f} (RMSE {math.sqrt(np.mean(losses[-50:])):.3f}), "
                f"{time.time() - t0:.1f}s")


# ---- fallback gate --------------------------------------------------------------------------

def _r2r_mse(fn, y1, y2, sigma):
    """Estimated error (vs the unknown clean image) of fn at noise level sqrt(2) sigma."""
    return float(np.mean((fn(y1) - y2) ** 2)) - 2.0 * sigma ** 2


def gate(I, sigma, opts=None, tile: int = 512, threshold_db: float = 0.1, seed: int = 0, ctx=None) -> dict:
    """Per-image decision: take the network's pilot unless its estimated step-1
    PSNR on a central tile is more than threshold_db below the plain step's."""
    o = dict(opts or dense_opts())
    m, n = I.shape
    t = min(tile, m, n)
    r0, c0 = (m - t) // 2, (n - t) // 2
    y = np.asfortranarray(I[r0:r0 + t, c0:c0 + t], dtype=np.float64)
    z = np.random.default_rng(seed).standard_normal(y.shape)
    y1, y2 = np.asfortranarray(y + sigma * z), y - sigma * z
    s1 = math.sqrt(2.0) * sigma
    o1 = dict(o, Wiener=False, form="plain")
    e_plain = _r2r_mse(lambda v: api.GBM3D(v, s1, o1, ctx=ctx)[0], y1, y2, sigma)
    e_net = _r2r_mse(lambda v: pilot_image(v, s1, ctx), y1, y2, sigma)
    gap = 10.0 * math.log10(max(e_net, 1e-12) / max(e_plain, 1e-12))
    return {"mse_plain_est": e_plain, "mse_pilot_est": e_net, "gap_db": gap, "fallback": gap > threshold_db}


def GBM3D_learned(I, sigma, opts=None, ctx=None, use_gate: bool = True):
    """[U, out] with the learned pilot in place of step 1, or the plain method
    when the gate falls back (out['path'] says which)."""
    o = dict(opts or dense_opts())
    g = gate(I, sigma, o, ctx=ctx) if use_gate else {"fallback": False}
    if g["fallback"]:
        U, out = api.GBM3D(I, sigma, dict(o, form="plain"), ctx=ctx)
        out.update(path="plain", gate=g)
        return U, out
    U, out = api.GBM3D(I, sigma, dict(o, form="learned"), ctx=ctx)
    out.update(path="learned", gate=g)
    return U, out


def evaluate(size: int = 1024, sigmas=(15.0, 25.0, 50.0), seed: int = 900, ctx=None, log=print) -> list[dict]:
    """PSNR (vs the clean image) of the plain 2-step method, the learned-pilot
    method and the learned network's untrained initialisation, per sigma."""
    ctx = ctx or context()
    trained = get_params(ctx)
    rows = []
    for k, sigma in enumerate(sigmas):
        clean, noisy = synth.noisy_image(size, size, sigma, seed=seed + k)
        o = dense_opts()
        Up, outp = api.GBM3D(noisy, sigma, dict(o, form="plain"), ctx=ctx)
        Ul, outl = GBM3D_learned(noisy, sigma, o, ctx=ctx)
        Un, outn = api.GBM3D(noisy, sigma, dict(o, form="learned"), ctx=ctx)
        set_params(init_params(0), ctx)
        Uu, _ = api.GBM3D(noisy, sigma, dict(o, form="learned"), ctx=ctx)
        set_params(trained, ctx)
        row = {"sigma": sigma, "psnr_noisy": options.myPSNR(clean, noisy, 255),
               "psnr_plain": options.myPSNR(clean, Up, 255), "psnr_learned": options.myPSNR(clean, Un, 255),
               "psnr_gated": options.myPSNR(clean, Ul, 255),
               "psnr_untrained": options.myPSNR(clean, Uu, 255),
               "psnr_step1_plain": options.myPSNR(clean, outp["U1"], 255),
               "psnr_step1_learned": options.myPSNR(clean, outn["U1"], 255),
               "path": outl["path"], "gate": outl["gate"]}
        rows.append(row)
        if log:
            log(row)
    return rows


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    ev = sub.add_parser("eval")
    ev.add_argument("--size", type=int, default=1024)
    ev.add_argument("--weights", default=WEIGHTS)
    t = sub.add_parser("train")
    t.add_argument("--steps", type=int, default=3000)
    t.add_argument("--batch", type=int, default=32)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--crops", type=int, default=20000)
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--out", default=WEIGHTS)
    t.add_argument("--max-seconds", type=float, default=None)
    a = ap.parse_args()
    from . import build
    build.build()
    if a.cmd == "eval":
        load(a.weights)
        evaluate(a.size)
        return
    params, losses = train(a.steps, a.batch, a.lr, a.crops, seed=a.seed, max_seconds=a.max_seconds)
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    np.save(a.out, params)
    print(f"saved {a.out}: final loss {np.mean(losses[-100:]):.4f}")


if __name__ == "__main__":
    main()
