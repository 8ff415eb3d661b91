"""Seeded synthetic test images.

The reference measures on no public dataset and ships one photo only, so
seeded synthetic images stand in: a linear-gradient background, 40 random
ellipses of uniform intensity in [0, 255] and 3 sinusoidal texture patches
with a period of 4-16 px, plus additive white Gaussian noise.  numpy's PCG64
generator makes every image reproducible from its seed.
"""
from __future__ import annotations

import numpy as np


def clean_image(m: int, n: int, seed: int = 0, n_ellipses: int = 40, n_textures: int = 3) -> np.ndarray:
    """m x n float64 clean image on a 0-255 scale (column-major)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    yy, xx = np.meshgrid(np.arange(m, dtype=np.float64), np.arange(n, dtype=np.float64), indexing="ij")
    g0, gy, gx = rng.uniform(40, 120), rng.uniform(-60, 60), rng.uniform(-60, 60)
    img = g0 + gy * yy / max(m - 1, 1) + gx * xx / max(n - 1, 1)
    for _ in range(n_ellipses):
        cy, cx = rng.uniform(0, m), rng.uniform(0, n)
        ry = rng.uniform(0.02, 0.2) * m
        rx = rng.uniform(0.02, 0.2) * n
        th = rng.uniform(0, np.pi)
        val = rng.uniform(0, 255)
        c, s = np.cos(th), np.sin(th)
        # only the ellipse's bounding box (2 px of margin) is tested: the same
        # elementwise arithmetic as over the whole grid, on fewer pixels
        ey, ex = np.hypot(ry * c, rx * s), np.hypot(ry * s, rx * c)
        r0, r1 = max(int(np.floor(cy - ey)) - 2, 0), min(int(np.ceil(cy + ey)) + 3, m)
        c0, c1 = max(int(np.floor(cx - ex)) - 2, 0), min(int(np.ceil(cx + ex)) + 3, n)
        if r0 >= r1 or c0 >= c1:
            continue
        by, bx = yy[r0:r1, c0:c1], xx[r0:r1, c0:c1]
        u = ((by - cy) * c + (bx - cx) * s) / ry
        v = (-(by - cy) * s + (bx - cx) * c) / rx
        img[r0:r1, c0:c1][u * u + v * v <= 1.0] = val
    for _ in range(n_textures):
        h = int(rng.uniform(0.1, 0.3) * m) + 1
        w = int(rng.uniform(0.1, 0.3) * n) + 1
        y0 = int(rng.integers(0, max(m - h, 1)))
        x0 = int(rng.integers(0, max(n - w, 1)))
        period = rng.uniform(4, 16)
        th = rng.uniform(0, np.pi)
        amp = rng.uniform(20, 60)
        base = rng.uniform(60, 190)
        py, px = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
        phase = 2 * np.pi * (py * np.cos(th) + px * np.sin(th)) / period
        img[y0:y0 + h, x0:x0 + w] = base + amp * np.sin(phase)
    return np.asfortranarray(np.clip(img, 0, 255))


def noisy_image(m: int, n: int, sigma: float, seed: int = 0, dtype=np.float64):
    """(clean, noisy) pair; noise is N(0, sigma^2) from an independent stream."""
    clean = clean_image(m, n, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 1_000_003))
    noisy = clean + sigma * rng.standard_normal((m, n))
    return clean, np.asfortranarray(noisy.astype(dtype))


def colored_noisy_image(m: int, n: int, sigma: float, omega: float = 1.0, seed: int = 0):
    """(clean, noisy, sigmaPSD): white noise of std sigma filtered by a unit-sum
    circular Gaussian of width omega (scripts/mainTestColoredNoise.m builds its
    test noise this way), and its power spectrum sigma^2 |g_hat|^2, the matrix
    sigma that GBM3D.m takes for coloured noise."""
    from .options import gaussian_psf_hat
    clean = clean_image(m, n, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 2_000_003))
    ghat = gaussian_psf_hat((m, n), omega)
    w = sigma * rng.standard_normal((m, n))
    noise = np.real(np.fft.ifft2(np.fft.fft2(w) * ghat))
    psd = sigma ** 2 * np.abs(ghat) ** 2
    return clean, np.asfortranarray(clean + noise), np.asfortranarray(psd)


def video(m: int, n: int, frames: int, sigma: float, seed: int = 0, n_ellipses: int = 40):
    """(clean, noisy) m x n x frames on a 0-255 scale: a gradient background and
    ellipses that each translate by a fixed (dy, dx) of 0-3 px per frame."""
    rng = np.random.Generator(np.random.PCG64(seed))
    yy, xx = np.meshgrid(np.arange(m, dtype=np.float64), np.arange(n, dtype=np.float64), indexing="ij")
    g0, gy, gx = rng.uniform(40, 120), rng.uniform(-60, 60), rng.uniform(-60, 60)
    ell = []
    for _ in range(n_ellipses):
        ell.append((rng.uniform(0, m), rng.uniform(0, n), rng.uniform(0.02, 0.2) * m, rng.uniform(0.02, 0.2) * n,
                    rng.uniform(0, np.pi), rng.uniform(0, 255), rng.uniform(-3, 3), rng.uniform(-3, 3)))
    clean = np.zeros((m, n, frames))
    for f in range(frames):
        img = g0 + gy * yy / max(m - 1, 1) + gx * xx / max(n - 1, 1)
        for cy, cx, ry, rx, th, val, vy, vx in ell:
            c, s = np.cos(th), np.sin(th)
            # bounding box of the moved ellipse, 2 px of margin (see clean_image)
            ey, ex = np.hypot(ry * c, rx * s), np.hypot(ry * s, rx * c)
            ccy, ccx = cy + vy * f, cx + vx * f
            r0, r1 = max(int(np.floor(ccy - ey)) - 2, 0), min(int(np.ceil(ccy + ey)) + 3, m)
            c0, c1 = max(int(np.floor(ccx - ex)) - 2, 0), min(int(np.ceil(ccx + ex)) + 3, n)
            if r0 >= r1 or c0 >= c1:
                continue
            by, bx = yy[r0:r1, c0:c1], xx[r0:r1, c0:c1]
            u = ((by - cy - vy * f) * c + (bx - cx - vx * f) * s) / ry
            v = (-(by - cy - vy * f) * s + (bx - cx - vx * f) * c) / rx
            img[r0:r1, c0:c1][u * u + v * v <= 1.0] = val
        clean[:, :, f] = img
    noise = np.random.Generator(np.random.PCG64(seed + 3_000_017)).standard_normal((m, n, frames))
    return np.asfortranarray(clean), np.asfortranarray(clean + sigma * noise)
