"""Test infrastructure: CPU restatement of the radiance-cache MLP.

The radiance cache has no counterpart in the reference (the reference's path
tracer ends every path after `bounces` vertices, src/shaders/pathtrace.wgsl
and VoxelBench/pipeline/core.cpp); this module states the network the CUDA
kernels in voxelrt_b200/csrc/k_mlp.cu compute, so that tests can check them:

* input encoding of a query (position in metres, normal, albedo): the
  position divided by the world extent, then for 12 octaves k and each axis
  sin/cos(2*pi * 2^k * frac(p / 2)), followed by normal, albedo, 1, 0
  (80 features), rounded to bf16.  Octave 0 uses the project's own sincos
  (om_sincos in vrt_oracle.cpp, the same code the kernels run); octave k+1
  follows from octave k by sin 2a = (sin a cos a) * 2 and
  cos 2a = (cos a - sin a)(cos a + sin a) in fp32, as the kernels evaluate
  them, so the features are bit-exact;
* 80 -> 64 -> 64 -> 64 -> 3 ReLU network without biases; weights and hidden
  activations bf16, sums in fp32 (fp64 here);
* loss: mean over samples of sum_c (o_c - y_c)^2 / (o_c^2 + 0.01), the
  denominator held constant, so dL/do_c = 2 (o_c - y_c) / (o_c^2 + 0.01) / n;
* Adam with b1 0.9, b2 0.99, eps 1e-8 on fp32 master weights.

`forward`/`gradient` follow the kernels' bf16 roundings (the GPU parity
checks); `forward64`/`gradient64` are the exact fp64 network used to pin the
analytic gradient against finite differences.
"""
from __future__ import annotations

import numpy as np

from . import math_eval

N_IN, N_HID, N_OUT_PAD, N_OUT = 80, 64, 16, 3
SHAPES = [(N_IN, N_HID), (N_HID, N_HID), (N_HID, N_HID), (N_HID, N_OUT_PAD)]
N_PARAMS = sum(a * b for a, b in SHAPES)   # 14336
N_FREQS = 12
TWO_PI_F32 = np.float32(6.28318548)


def bf16_round(x) -> np.ndarray:
    """Round-to-nearest-even to bf16, returned as float32 values."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    out = (r << 16).astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    if nan.any():
        out = out.copy()
        out[nan] = np.nan
    return out


def bf16_bits(x) -> np.ndarray:
    return (bf16_round(x).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def unpack(params: np.ndarray) -> list[np.ndarray]:
    """Flat parameter vector -> [W0 (80x64), W1, W2 (64x64), W3 (64x16)]."""
    out, off = [], 0
    for k, n in SHAPES:
        out.append(np.asarray(params[off:off + k * n]).reshape(k, n))
        off += k * n
    return out


def pack(ws: list[np.ndarray]) -> np.ndarray:
    return np.concatenate([np.asarray(w).ravel() for w in ws])


def encode(q9: np.ndarray, extent: float) -> np.ndarray:
    """n x 80 float32 features (bf16 values), as the kernels compute them."""
    q = np.ascontiguousarray(q9, np.float32).reshape(-1, 9)
    n = q.shape[0]
    f = np.zeros((n, N_IN), np.float32)
    x = (q[:, :3] / np.float32(extent)) * np.float32(0.5)
    t = x - np.floor(x)
    arg = (TWO_PI_F32 * t).astype(np.float32)
    sn = math_eval(0, arg.ravel()).reshape(n, 3)
    cs = math_eval(1, arg.ravel()).reshape(n, 3)
    for k in range(N_FREQS):
        f[:, 6 * k:6 * k + 3] = sn
        f[:, 6 * k + 3:6 * k + 6] = cs
        # octave k+1 by the double-angle identities, in the kernels' fp32 order
        sn, cs = (sn * cs) * np.float32(2.0), (cs - sn) * (cs + sn)
    f[:, 72:78] = q[:, 3:9]
    f[:, 78] = 1.0
    return bf16_round(f)


def forward(feat: np.ndarray, params: np.ndarray):
    """Returns (o: n x 16 fp64, acts: [A0..A3] bf16-valued, masks [3])."""
    ws = [bf16_round(w).astype(np.float64) for w in unpack(params)]
    a = np.asarray(feat, np.float64)
    acts, masks = [a], []
    for l in range(3):
        h = a @ ws[l]
        masks.append(h > 0)
        a = bf16_round(np.maximum(h, 0.0).astype(np.float32)).astype(np.float64)
        acts.append(a)
    o = a @ ws[3]
    return o, acts, masks


def loss_and_grad_out(o: np.ndarray, y3: np.ndarray):
    """Per-sample loss sum and bf16 dL/do (unscaled by 1/n), as the kernel forms them."""
    o32 = np.asarray(o[:, :N_OUT], np.float32)
    d = o32 - np.asarray(y3, np.float32)
    den = o32 * o32 + np.float32(0.01)
    g = np.zeros((o.shape[0], N_OUT_PAD), np.float32)
    g[:, :N_OUT] = bf16_round((np.float32(2.0) * d) / den)
    loss = float(np.sum((d.astype(np.float64) ** 2) / den.astype(np.float64)))
    return loss, g


def gradient(feat: np.ndarray, y3: np.ndarray, params: np.ndarray):
    """(mean loss, flat gradient of the mean loss) with the kernels' roundings."""
    n = feat.shape[0]
    ws = [bf16_round(w).astype(np.float64) for w in unpack(params)]
    o, acts, masks = forward(feat, params)
    loss, g = loss_and_grad_out(o, y3)
    dy = g.astype(np.float64)
    grads = [None] * 4
    grads[3] = acts[3].T @ dy
    dx = dy @ ws[3].T
    for l in (2, 1, 0):
        dh = bf16_round(np.where(masks[l], dx, 0.0).astype(np.float32)).astype(np.float64)
        grads[l] = acts[l].T @ dh
        if l > 0:
            dx = dh @ ws[l].T
    return loss / n, pack(grads) / n


def forward64(feat, params):
    ws = unpack(np.asarray(params, np.float64))
    a = np.asarray(feat, np.float64)
    for l in range(3):
        a = np.maximum(a @ ws[l], 0.0)
    return a @ ws[3]


def loss64(feat, y3, params) -> float:
    """Mean relative L2 loss with the denominator evaluated at `params`."""
    o = forward64(feat, params)[:, :N_OUT]
    den = o * o + 0.01
    return float(np.mean(np.sum((o - y3) ** 2 / den, axis=1)))


def gradient64(feat, y3, params):
    """Exact fp64 gradient of the mean loss (denominator constant)."""
    n = feat.shape[0]
    ws = unpack(np.asarray(params, np.float64))
    a = np.asarray(feat, np.float64)
    acts, hs = [a], []
    for l in range(3):
        h = a @ ws[l]
        hs.append(h)
        a = np.maximum(h, 0.0)
        acts.append(a)
    o = a @ ws[3]
    dy = np.zeros_like(o)
    oc = o[:, :N_OUT]
    dy[:, :N_OUT] = 2.0 * (oc - y3) / (oc * oc + 0.01)
    grads = [None] * 4
    grads[3] = acts[3].T @ dy
    dx = dy @ ws[3].T
    for l in (2, 1, 0):
        dh = np.where(hs[l] > 0, dx, 0.0)
        grads[l] = acts[l].T @ dh
        dx = dh @ ws[l].T
    return pack(grads) / n


def adam(w, m, v, g, step: int, lr: float, b1=0.9, b2=0.99, eps=1e-8):
    """One fp32 Adam step (output-layer pad columns forced to 0)."""
    f = np.float32
    b1, b2, eps, lr = f(b1), f(b2), f(eps), f(lr)
    g = np.asarray(g, np.float32)
    w = np.asarray(w, np.float32).copy()
    m = b1 * np.asarray(m, np.float32) + (f(1) - b1) * g
    v = b2 * np.asarray(v, np.float32) + (f(1) - b2) * g * g
    bc1 = f(1) - f(np.float64(b1) ** step)
    bc2 = f(1) - f(np.float64(b2) ** step)
    w = w - lr * (m / bc1) / (np.sqrt(v / bc2) + eps)
    off3 = N_PARAMS - N_HID * N_OUT_PAD
    pad = (np.arange(N_HID * N_OUT_PAD) % N_OUT_PAD) >= N_OUT
    w[off3:][pad] = 0.0
    return w, m, v
