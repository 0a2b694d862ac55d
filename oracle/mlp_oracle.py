"""NumPy restatement of the learned initialiser's network (forward, loss, backward, Adam).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the tensor-core network kernels
(fdt_b200/csrc/bpx_mlp.cu, bpx_gemm.cu).  The product never imports this module.

The network has no counterpart in the reference; this file restates the library's own
definition: BF16 weights and activations (round-to-nearest-even), products summed in higher
precision (float64 here, FP32 in the tensor cores), biases and pre-activations in FP32, exact
(erf) GELU, the loss of bpx_mlp_train_step_dev and bias-corrected Adam.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

WIDTH, HIDDEN, NOUT = 256, 4, 32


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even); returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def geometry(ndir: int):
    nin = (ndir + 7) // 8 * 8
    k = [nin] + [WIDTH] * HIDDEN
    n = [WIDTH] * HIDDEN + [NOUT]
    woff, boff, o = [], [], 0
    for l in range(HIDDEN + 1):
        woff.append(o)
        o += k[l] * n[l]
        boff.append(o)
        o += n[l]
    return nin, k, n, woff, boff, o


def unpack(params: np.ndarray, ndir: int):
    nin, k, n, woff, boff, _ = geometry(ndir)
    W = [params[woff[l] : woff[l] + n[l] * k[l]].reshape(n[l], k[l]) for l in range(HIDDEN + 1)]
    b = [params[boff[l] : boff[l] + n[l]] for l in range(HIDDEN + 1)]
    return W, b


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def _ident(x):
    return np.asarray(x, np.float64)


def forward(params: np.ndarray, ndir: int, x: np.ndarray, exact: bool = False):
    """x: [B][nin] bf16 values (float32).  Returns (out [B][32], cache).  exact=True drops every
    BF16/FP32 rounding (float64 throughout), which makes the loss smooth for finite differences."""
    r = _ident if exact else bf16
    f32 = np.float64 if exact else np.float32
    W, b = unpack(params, ndir)
    a = [np.asarray(x, f32)]
    z = []
    for l in range(HIDDEN):
        zz = (a[-1].astype(np.float64) @ r(W[l]).astype(np.float64).T).astype(f32) + b[l]
        z.append(zz)
        a.append(r(gelu(zz.astype(np.float64)).astype(f32)))
    out = (a[-1].astype(np.float64) @ r(W[HIDDEN]).astype(np.float64).T).astype(f32) + b[HIDDEN]
    return out, (a, z)


def loss_grad(out: np.ndarray, t: np.ndarray, tw: np.ndarray, exact: bool = False):
    """Mean loss over the batch and dL/dout (rounded to bf16 as the kernel stores it)."""
    B = out.shape[0]
    o, tt, w = out.astype(np.float64), t.astype(np.float64), tw.astype(np.float64)
    g = np.zeros_like(o)
    scal = [j for j in range(NOUT) if not (3 <= j < 12)]
    e = o[:, scal] - tt[:, scal]
    L = (w[:, scal] * e * e).sum(axis=1)
    g[:, scal] = 2.0 * w[:, scal] * e / B
    for k in range(3):
        u = o[:, 3 + 3 * k : 6 + 3 * k]
        v = tt[:, 3 + 3 * k : 6 + 3 * k]
        wd = w[:, 3 + 3 * k]
        uu = (u * u).sum(axis=1)
        uv = (u * v).sum(axis=1)
        L += wd * (uu * uu - 2.0 * uv * uv + 1.0)
        g[:, 3 + 3 * k : 6 + 3 * k] = (4.0 * wd * uu)[:, None] * u / B - (4.0 * wd * uv)[:, None] * v / B
    return float(L.mean()), (g if exact else bf16(g.astype(np.float32)))


def backward(params: np.ndarray, ndir: int, cache, dz_out: np.ndarray, exact: bool = False) -> np.ndarray:
    """Gradient of the mean loss with respect to the flat parameter vector."""
    r = _ident if exact else bf16
    f32 = np.float64 if exact else np.float32
    W, _ = unpack(params, ndir)
    nin, k, n, woff, boff, total = geometry(ndir)
    a, z = cache
    grads = np.zeros(total, np.float64)
    g = dz_out.astype(np.float64)
    for l in range(HIDDEN, -1, -1):
        grads[woff[l] : woff[l] + n[l] * k[l]] = (g.T @ a[l].astype(np.float64)).ravel()
        grads[boff[l] : boff[l] + n[l]] = g.sum(axis=0)
        if l == 0:
            break
        da = g @ r(W[l]).astype(np.float64)
        g = r((da.astype(f32) * gelu_grad(z[l - 1].astype(np.float64)).astype(f32))).astype(np.float64)
    return grads


def adam(p, g, m, v, lr, b1, b2, eps, step):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1, c2 = 1.0 / (1.0 - b1**step), 1.0 / (1.0 - b2**step)
    return p - lr * (m * c1) / (np.sqrt(v * c2) + eps), m, v
