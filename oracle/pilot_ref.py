"""CPU reference of the learned pilot network — TEST INFRASTRUCTURE ONLY.

The CUDA kernels (gbm3d_b200/csrc/pilot.cu) run the network with bf16
operands and fp32 accumulation on the tensor cores; this module runs the same
network in float64 with the same bf16 rounding of inputs, weights and
activations, and its backward pass by plain calculus, so the GPU forward and
the GPU gradients can be checked against it.  It is never part of the
product path.

Network: input (noisy/255, sigma/255); 7 x [3x3 conv, 48 ch, bias, ReLU];
3x3 conv to 1 channel + bias = r; pilot = noisy - 255 r.  Convolutions are
correlations with zero padding: y[p] = sum_{dy,dx} x[p + (dy-1, dx-1)] W[3dy+dx]^T + b.
Parameters: per layer W [9][out][in] then b [out], concatenated.
"""
from __future__ import annotations

import numpy as np

LAYERS = [(2, 48)] + [(48, 48)] * 6 + [(48, 1)]


def param_count():
    return sum(9 * co * ci + co for ci, co in LAYERS)


def unpack(params):
    out, o = [], 0
    for ci, co in LAYERS:
        W = params[o:o + 9 * co * ci].reshape(9, co, ci)
        o += 9 * co * ci
        b = params[o:o + co]
        o += co
        out.append((W, b))
    return out


def init_params(seed=0):
    """He-normal weights, zero biases; the last layer starts small."""
    rng = np.random.default_rng(seed)
    parts = []
    for li, (ci, co) in enumerate(LAYERS):
        std = np.sqrt(2.0 / (9 * ci)) * (0.1 if li == len(LAYERS) - 1 else 1.0)
        parts += [rng.normal(0, std, 9 * co * ci), np.zeros(co)]
    return np.concatenate(parts).astype(np.float32)


def bf16(x):
    """Round to bfloat16 (nearest even) and back to float64."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _shift(x, dy, dx):
    """x[n, y + dy, x + dx, :] with zeros outside."""
    N, H, W, C = x.shape
    out = np.zeros_like(x)
    ys, yd = (slice(dy, H), slice(0, H - dy)) if dy >= 0 else (slice(0, H + dy), slice(-dy, H))
    xs, xd = (slice(dx, W), slice(0, W - dx)) if dx >= 0 else (slice(0, W + dx), slice(-dx, W))
    out[:, yd, xd, :] = x[:, ys, xs, :]
    return out


def conv(x, W, b=None):
    y = 0.0
    for t in range(9):
        y = y + _shift(x, t // 3 - 1, t % 3 - 1) @ W[t].T
    return y if b is None else y + b


def forward(params, img, sig, rounding=True):
    """img: [N, H, W] float; sig: [N].  Returns (pilot, acts) with acts[l] the
    input of layer l, bf16-rounded like the kernels' (rounding=False: exact
    float64 arithmetic, for finite-difference checks of the backward pass)."""
    rnd = (lambda a: bf16(np.asarray(a, np.float32))) if rounding else (lambda a: np.asarray(a, np.float64))
    Ws = [(rnd(W), np.asarray(b, np.float64)) for W, b in unpack(np.asarray(params, np.float64 if not rounding
                                                                             else np.float32))]
    img = np.asarray(img, np.float64)
    x = np.stack([img / 255.0, np.broadcast_to(np.asarray(sig, np.float64)[:, None, None] / 255.0, img.shape)], -1)
    x = rnd(x)
    acts = [x]
    for l, (W, b) in enumerate(Ws):
        y = conv(x, W, b)
        if l < len(Ws) - 1:
            x = rnd(np.maximum(y, 0))
            acts.append(x)
    r = y[..., 0]
    return img - 255.0 * r, acts


def gradients(params, img, sig, target, rounding=True):
    """Gradient of mean((pilot - target)^2) w.r.t. the parameters (float64),
    through the (bf16-rounded) forward activations, and the loss."""
    rnd = (lambda a: bf16(np.asarray(a, np.float32))) if rounding else (lambda a: np.asarray(a, np.float64))
    Ws = [(rnd(W), b) for W, b in unpack(np.asarray(params, np.float64 if not rounding else np.float32))]
    pilot, acts = forward(params, img, sig, rounding)
    P = pilot.size
    g = (-255.0 * 2.0 * (pilot - np.asarray(target, np.float64)) / P)[..., None]  # d loss / d r
    grads = [None] * len(Ws)
    for l in range(len(Ws) - 1, -1, -1):
        x = acts[l]
        W, _ = Ws[l]
        dW = np.zeros(W.shape)
        for t in range(9):
            xs = _shift(x, t // 3 - 1, t % 3 - 1)
            dW[t] = np.einsum("nhwo,nhwi->oi", g, xs)
        grads[l] = (dW, g.sum(axis=(0, 1, 2)))
        if l == 0:
            break
        dx = 0.0
        for t in range(9):  # transpose of the correlation
            dx = dx + _shift(g @ W[t], -(t // 3 - 1), -(t % 3 - 1))
        g = dx * (x > 0)
    flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
    return flat, float(np.mean((pilot - target) ** 2))
