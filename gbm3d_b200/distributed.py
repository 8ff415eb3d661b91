"""Tiled GBM3D (GBM3D_distributed) and its multi-GPU sharding.

Host-side restatement of source/GBM3D_distributed.m:15-120 with
utilities/getBM3D_distribution.m:10-48 and utilities/makeInterpWindow.m:8-13:
the image is cut into (256+k) x (256+k) tiles overlapping by k = blockSize,
each tile x match spin is denoised with the reference's four hot-path
functions, and the tiles are stitched with linear ramp windows.

Sharding: with torch.distributed initialised and world size N > 1, work item
ii (a tile x spin row of the distribution table) runs on rank ii mod N.  The
per-item results are all-gathered and every rank stitches all items in table
order, so the result does not depend on N (bit-identical to one rank); the
step-2 search needs the whole step-1 estimate, which every rank then holds.
The all-gather is the only exchange; items are independent otherwise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable

import numpy as np

from . import options as _opt


def getBM3D_distribution(m: int, n: int, matchSpins, k: int):
    """Rows (R1, R2, R3, R4, spin) with 1-based inclusive tile bounds, tile side d0 = 256+k
    (getBM3D_distribution.m:10-48)."""
    d0 = 256 + k
    xcnt = math.ceil((n - k) / (d0 - k))
    ycnt = math.ceil((m - k) / (d0 - k))
    R = []
    for i in range(ycnt):
        iy = i * (d0 - k)
        for j in range(xcnt):
            ix = j * (d0 - k)
            for s in matchSpins:
                r1, r2, r3, r4 = iy + 1, iy + d0, ix + 1, ix + d0
                if r4 >= n:
                    r3 = min(n - math.ceil((n - r3 + 1) / k) * k + 1, n - 2 * k + 1)
                if r2 >= m:
                    r1 = min(m - math.ceil((m - r1 + 1) / k) * k + 1, m - 2 * k + 1)
                R.append([r1, min(r2, m), r3, min(r4, n), int(s)])
    return np.array(R, dtype=np.int64).reshape(-1, 5), d0, k


def makeInterpWindow(a: int, b: int, k: int) -> np.ndarray:
    """Linear ramps of length k on all four sides (makeInterpWindow.m:8-13)."""
    w = np.ones((a, b))
    ramp = np.linspace(0.01, 1, k)
    w[:k, :] *= ramp[:, None]
    w[:, :k] *= ramp[None, :]
    w[a - k:, :] *= ramp[::-1][:, None]
    w[:, b - k:] *= ramp[::-1][None, :]
    return w


@dataclass
class Backend:
    """The four per-tile functions (CUDA drop-ins by default)."""
    step1: Callable  # (Ilocal, sigma, tau, opts) -> (U, W)
    step2: Callable  # (pilot_local, noisy_local, sigma, opts) -> (U, W)


def cuda_backend(ctx=None) -> Backend:
    from . import api

    def step1(I, sigma, tau, opts):
        S, V = api.matchBlocksCPU(I, sigma, opts, ctx=ctx)
        return api.denoiseAndAggregateGPU(V, S, tau, None, None, opts, ctx=ctx)

    def step2(P, I, sigma, opts):
        S, V1, V2 = api.matchBlocksWie(P, I, sigma, opts, ctx=ctx)
        return api.denoiseAndAggregateWieFast(V1, V2, S, sigma, opts, ctx=ctx)

    return Backend(step1, step2)


def _dist():
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
            return dist
    except ImportError:
        pass
    return None


def _run_items(items, fn, dist):
    """Run fn(ii) for the work items of this rank and gather every item's result."""
    if dist is None:
        return [fn(ii) for ii in items]
    rank, world = dist.get_rank(), dist.get_world_size()
    mine = {ii: fn(ii) for ii in items if ii % world == rank}
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    out = {}
    for part in gathered:
        out.update(part)
    return [out[ii] for ii in items]


def _stitch(R, results, m, n, d0, k):
    U2 = np.zeros((m, n))
    norm = np.zeros((m, n))
    mwin = makeInterpWindow(d0, d0, k)
    for ii, (U, W) in enumerate(results):
        r1, r2, r3, r4 = (int(v) for v in R[ii, :4])
        ny, nx = r2 - r1 + 1, r4 - r3 + 1
        win = mwin if (ny == d0 and nx == d0) else makeInterpWindow(ny, nx, k)
        U2[r1 - 1:r2, r3 - 1:r4] += U * win
        norm[r1 - 1:r2, r3 - 1:r4] += win * W
    return U2, norm


def _shift(a, s):
    return np.roll(a, (s, s), axis=(0, 1))


def GBM3D_distributed(I, sigma, opts: dict | None = None, backend: Backend | None = None):
    """[U, out] = GBM3D_distributed(I, sigma, opts) (source/GBM3D_distributed.m:1)."""
    o = _opt.resolve_opts(opts)
    I = np.asarray(I, dtype=np.float64)
    m, n = I.shape
    k = int(o["blockSize"])
    if m < 256 + k or n < 256 + k:  # GBM3D_distributed.m:24-27
        from . import api
        return api.GBM3D(I, sigma, o)
    be = backend or cuda_backend()
    dist = _dist()
    tau = sigma * _opt.getTau(int(o["levels"]), int(o["tauMode"]))
    R, d0, _ = getBM3D_distribution(m, n, o["matchSpins"], k)
    RW, _, _ = getBM3D_distribution(m, n, o["matchSpinsWie"], k)

    def step1(ii):
        r1, r2, r3, r4, s = (int(v) for v in R[ii])
        U, W = be.step1(_shift(I[r1 - 1:r2, r3 - 1:r4], s), sigma, tau, o)
        return _shift(U, -s), _shift(W, -s)

    res1 = _run_items(list(range(len(R))), step1, dist)
    U2, norm = _stitch(R, res1, m, n, d0, k)
    U2 = U2 / norm
    out = {"U2": U2}
    if not o["Wiener"]:
        return U2, out

    def step2(ii):
        r1, r2, r3, r4, s = (int(v) for v in RW[ii])
        U, W = be.step2(_shift(U2[r1 - 1:r2, r3 - 1:r4], s), _shift(I[r1 - 1:r2, r3 - 1:r4], s), sigma, o)
        return _shift(U, -s), _shift(W, -s)

    res2 = _run_items(list(range(len(RW))), step2, dist)
    Uf, norm2 = _stitch(RW, res2, m, n, d0, k)
    return Uf / norm2, out
