"""Tiled GBM3D (GBM3D_distributed) and its multi-GPU sharding.

Restatement of source/GBM3D_distributed.m:15-120 with
utilities/getBM3D_distribution.m:10-48 and utilities/makeInterpWindow.m:8-13:
the image is cut into (256+k) x (256+k) tiles overlapping by k = blockSize,
each tile x match spin is denoised with the reference's four hot-path
functions, and the tiles are stitched with linear ramp windows.

Two drivers with the same result:
  * on the device (the default with a GPU): one library call per step runs
    this rank's tiles (gbm3d_tiles_device) and one call stitches them
    (gbm3d_tiles_stitch_device); images and tiles stay in device memory;
  * on the host through a Backend of per-tile functions (the CUDA drop-ins
    with host copies, or the CPU oracle in the tests).

Sharding: with torch.distributed initialised and world size N > 1, work item
ii (a tile x spin row of the distribution table) runs on rank ii mod N.  The
per-item tiles are packed into fixed (2, tile, tile) float64 slots and
all-gathered as one tensor (NCCL on the GPU, gloo on the CPU), and every rank
stitches all items in table order, so the result does not depend on N
(bit-identical to one rank); the step-2 search needs the whole step-1
estimate, which every rank then holds.  The all-gather is the only exchange.
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


def _gather_slots(mine, n_items: int, dist, like):
    """Every item's slot, in table order, from the slots each rank computed:
    rank r holds items r, r + N, ... in order (mine: [n_mine, 2, tile, tile]).
    One all_gather of equal-sized tensors (counts padded to the largest)."""
    import torch
    world = dist.get_world_size()
    cap = -(-n_items // world)
    buf = torch.zeros((cap,) + tuple(mine.shape[1:]), dtype=mine.dtype, device=mine.device)
    buf[:mine.shape[0]] = mine
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    full = torch.empty((n_items,) + tuple(mine.shape[1:]), dtype=mine.dtype, device=mine.device)
    for r in range(world):
        idx = list(range(r, n_items, world))
        if idx:
            full[idx] = parts[r][:len(idx)]
    return full


def _run_items(items, fn, dist, tile):
    """Run fn(ii) -> (U, W) for the work items of this rank and return every
    item's (U, W) in table order (host arrays)."""
    if dist is None:
        return [fn(ii) for ii in items]
    import torch
    rank, world = dist.get_rank(), dist.get_world_size()
    res = {ii: fn(ii) for ii in items if ii % world == rank}
    mine = torch.zeros((len(res), 2, tile, tile), dtype=torch.float64)
    shapes = {}
    for q, ii in enumerate(sorted(res)):
        U, W = res[ii]
        shapes[ii] = U.shape
        mine[q, 0].view(-1)[:U.size] = torch.from_numpy(np.asfortranarray(U).ravel(order="F"))
        mine[q, 1].view(-1)[:W.size] = torch.from_numpy(np.asfortranarray(W).ravel(order="F"))
    full = _gather_slots(mine, len(items), dist, mine).numpy()
    return full, shapes


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


def _unpack(full, R, ii):
    r1, r2, r3, r4 = (int(v) for v in R[ii, :4])
    ny, nx = r2 - r1 + 1, r4 - r3 + 1
    U = full[ii, 0].reshape(-1)[:ny * nx].reshape((ny, nx), order="F")
    W = full[ii, 1].reshape(-1)[:ny * nx].reshape((ny, nx), order="F")
    return U, W


def _host_items(R, fn, dist, d0):
    out = _run_items(list(range(len(R))), fn, dist, d0)
    if dist is None:
        return out
    full, _ = out
    return [_unpack(full, R, ii) for ii in range(len(R))]


def GBM3D_distributed(I, sigma, opts: dict | None = None, backend: Backend | None = None, ctx=None):
    """[U, out] = GBM3D_distributed(I, sigma, opts) (source/GBM3D_distributed.m:1).
    Without a backend the tiles run on the device (gbm3d_tiles_device)."""
    o = _opt.resolve_opts(opts)
    I = np.asarray(I, dtype=np.float64)
    m, n = I.shape
    k = int(o["blockSize"])
    if m < 256 + k or n < 256 + k:  # GBM3D_distributed.m:24-27
        from . import api
        return api.GBM3D(I, sigma, o)
    dist = _dist()
    if backend is None:
        return _device_driver(I, sigma, o, dist, ctx)
    be = backend
    tau = sigma * _opt.getTau(int(o["levels"]), int(o["tauMode"]))
    R, d0, _ = getBM3D_distribution(m, n, o["matchSpins"], k)
    RW, _, _ = getBM3D_distribution(m, n, o["matchSpinsWie"], k)

    def step1(ii):
        r1, r2, r3, r4, s = (int(v) for v in R[ii])
        U, W = be.step1(_shift(I[r1 - 1:r2, r3 - 1:r4], s), sigma, tau, o)
        return _shift(U, -s), _shift(W, -s)

    res1 = _host_items(R, step1, dist, d0)
    U2, norm = _stitch(R, res1, m, n, d0, k)
    U2 = U2 / norm
    out = {"U2": U2}
    if not o["Wiener"]:
        return U2, out

    def step2(ii):
        r1, r2, r3, r4, s = (int(v) for v in RW[ii])
        U, W = be.step2(_shift(U2[r1 - 1:r2, r3 - 1:r4], s), _shift(I[r1 - 1:r2, r3 - 1:r4], s), sigma, o)
        return _shift(U, -s), _shift(W, -s)

    res2 = _host_items(RW, step2, dist, d0)
    Uf, norm2 = _stitch(RW, res2, m, n, d0, k)
    return Uf / norm2, out


def _device_driver(I, sigma, o, dist, ctx=None):
    """The tiled driver on the device: per step one gbm3d_tiles_device call over
    this rank's items, one all_gather of the item slots (N > 1), one
    gbm3d_tiles_stitch_device call in table order."""
    import ctypes as C

    import torch

    from . import api
    from ._lib import context, lib
    ctx = ctx or context()
    dev = torch.device("cuda", ctx.device)
    m, n = I.shape
    k = int(o["blockSize"])
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist is not None else (0, 1)
    tau = np.asfortranarray(sigma * _opt.getTau(int(o["levels"]), int(o["tauMode"])))
    ramp = np.ascontiguousarray(np.linspace(0.01, 1, k))
    co = api.c_opts(o)
    dI = torch.from_numpy(np.asfortranarray(I).ravel(order="F").copy()).to(dev)
    torch.cuda.synchronize(dev)

    def step(spins, pilot):
        R, d0, _ = getBM3D_distribution(m, n, spins, k)
        table = np.ascontiguousarray(R, dtype=np.int32)
        mine = np.ascontiguousarray(table[rank::world])
        slots = torch.empty((mine.shape[0], 2, d0, d0), dtype=torch.float64, device=dev)
        ctx.check(lib().gbm3d_tiles_device(
            ctx.h, C.c_void_p(dI.data_ptr()), C.c_void_p(pilot.data_ptr()) if pilot is not None else None, m, n,
            float(sigma), tau.ctypes.data_as(C.c_void_p), C.byref(co), mine.ctypes.data_as(C.c_void_p),
            mine.shape[0], d0, C.c_void_p(slots.data_ptr())))
        full = _gather_slots(slots, len(table), dist, slots) if dist is not None else slots
        torch.cuda.synchronize(dev)
        U = torch.empty_like(dI)
        ctx.check(lib().gbm3d_tiles_stitch_device(
            ctx.h, C.c_void_p(full.data_ptr()), table.ctypes.data_as(C.c_void_p), len(table), d0, m, n, k,
            ramp.ctypes.data_as(C.c_void_p), C.c_void_p(U.data_ptr())))
        return U

    U2 = step(o["matchSpins"], None)
    out = {"U2": U2.cpu().numpy().reshape((m, n), order="F")}
    if not o["Wiener"]:
        return out["U2"], out
    U = step(o["matchSpinsWie"], U2)
    return U.cpu().numpy().reshape((m, n), order="F"), out


# ---- the strip form: one image split by columns over the ranks ---------------------

def strip_bounds(n: int, parts: int) -> list[tuple[int, int]]:
    """Column ranges [lo, hi) of `parts` near-equal contiguous strips covering 0..n."""
    if parts < 1 or parts > n:
        raise ValueError("strip count must be in 1..n")
    return [(r * n // parts, (r + 1) * n // parts) for r in range(parts)]


def _gather_strips(mine, bounds, world, dist):
    """Every strip, in column order, from the strips each rank computed: rank r
    holds strips r, r + N, ... (mine: list of (hi - lo, m) tensors, column-major
    strips).  One all_gather of equal-sized tensors (widths padded to the widest,
    counts to the largest)."""
    import torch
    m = mine[0].shape[1] if mine else 0
    cap_w = max(hi - lo for lo, hi in bounds)
    cap_n = -(-len(bounds) // world)
    like = mine[0]
    buf = torch.zeros((cap_n, cap_w, m), dtype=like.dtype, device=like.device)
    for q, t in enumerate(mine):
        buf[q, :t.shape[0]] = t
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = []
    for s, (lo, hi) in enumerate(bounds):
        out.append(parts[s % world][s // world, :hi - lo])
    return out


def GBM3D_strips(I, sigma, opts: dict | None = None, strips: int | None = None, strip_fn=None, ctx=None):
    """GBM3D on one image split into column strips, one GPU per strip.

    Every rank holds the whole noisy image and computes whole strips: strip s
    (of `strips`, the world size by default) runs on rank s mod N.  A strip is
    computed by gbm3d_denoise_strip_device, which restricts every stage to the
    columns its consumers read (the strip plus the halo of the spin shifts,
    search windows and wavelet filters), so each strip is bit-identical to the
    same columns of the whole-image GBM3D; the only exchange is the final
    all_gather of the strips (NCCL between GPUs, gloo on the CPU).  This is not
    the reference's tiled driver (GBM3D_distributed, with its overlapping tiles
    and ramp stitching, which changes the result); it splits the work of
    source/GBM3D.m:22-83 itself.

    strip_fn(I, sigma, opts, lo, hi) -> m x (hi - lo) host array replaces the
    device call (the CPU tests pass the oracle here).  Returns the m x n result
    on every rank.
    """
    import torch
    I = np.asarray(I, dtype=np.float64)
    m, n = I.shape
    o = _opt.resolve_opts(opts, shape=(m, n), sigma=sigma)
    dist = _dist()
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist is not None else (0, 1)
    bounds = strip_bounds(n, strips or world)
    mine_idx = list(range(rank, len(bounds), world))
    if strip_fn is not None:
        mine = [torch.from_numpy(np.ascontiguousarray(np.asarray(strip_fn(I, sigma, o, lo, hi), np.float64).T))
                for lo, hi in (bounds[s] for s in mine_idx)]
    else:
        from . import api
        from ._lib import context
        ctx = ctx or context()
        dev = torch.device("cuda", ctx.device)
        dI = torch.from_numpy(np.asfortranarray(I).ravel(order="F").copy()).to(dev)
        torch.cuda.synchronize(dev)
        mine = []
        for s in mine_idx:
            lo, hi = bounds[s]
            t = torch.empty((hi - lo, m), dtype=torch.float64, device=dev)
            api.GBM3D_strip_device(dI.data_ptr(), m, n, sigma, lo, hi, t.data_ptr(), o, ctx=ctx)
            mine.append(t)
        ctx.synchronize()
    if dist is not None:
        if not mine:  # more ranks than strips: this rank still takes part in the gather
            like = torch.zeros((1, m), dtype=torch.float64,
                               device=dI.device if strip_fn is None else "cpu")
            mine = [like[:0]]
        got = _gather_strips(mine, bounds, world, dist)
    else:
        got = mine
    U = np.empty((m, n))
    for (lo, hi), t in zip(bounds, got):
        U[:, lo:hi] = t.cpu().numpy().T
    return U
