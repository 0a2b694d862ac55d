"""The network oracle pinned by its own mathematics (no GPU).

The learned initialiser has no counterpart in the reference, so the oracle of its kernels
(oracle/mlp_oracle.py) is pinned analytically: with every rounding switched off, its backward pass
must match central finite differences of its loss, and its BF16 rounding must be round-to-nearest-
even as the tensor-core kernels apply it.
"""
import numpy as np

from oracle import mlp_oracle as M


def _setup(seed=0, ndir=20, batch=6):
    rng = np.random.default_rng(seed)
    nin, k, n, woff, boff, total = M.geometry(ndir)
    p = np.zeros(total)
    for l in range(M.HIDDEN + 1):
        p[woff[l] : woff[l] + n[l] * k[l]] = rng.normal(size=n[l] * k[l]) / np.sqrt(k[l])
        p[boff[l] : boff[l] + n[l]] = 0.1 * rng.normal(size=n[l])
    x = np.zeros((batch, nin))
    x[:, :ndir] = rng.uniform(0.1, 1.0, size=(batch, ndir))
    t = rng.normal(size=(batch, M.NOUT))
    for kk in range(3):
        v = rng.normal(size=(batch, 3))
        t[:, 3 + 3 * kk : 6 + 3 * kk] = v / np.linalg.norm(v, axis=1, keepdims=True)
    tw = rng.uniform(0.2, 1.0, size=(batch, M.NOUT))
    return p, x, t, tw, ndir


def _loss(p, x, t, tw, ndir):
    out, _ = M.forward(p, ndir, x, exact=True)
    return M.loss_grad(out, t, tw, exact=True)[0]


def test_backward_matches_finite_differences():
    p, x, t, tw, ndir = _setup()
    out, cache = M.forward(p, ndir, x, exact=True)
    _, g_out = M.loss_grad(out, t, tw, exact=True)
    g = M.backward(p, ndir, cache, g_out, exact=True)
    nin, k, n, woff, boff, total = M.geometry(ndir)
    rng = np.random.default_rng(1)
    idx = list(rng.integers(0, total, size=40)) + [woff[0], boff[0], woff[4] + 5, boff[4] + 3, boff[4] + 20]
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (_loss(pp, x, t, tw, ndir) - _loss(pm, x, t, tw, ndir)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, 1.0 + 2**-9, -2.5, 3.0e-5, 65504.0], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # tie between 1 and 1+2^-7 goes to the even mantissa (1.0)
    assert r[2] == np.float32(1.0 + 2**-6)  # tie goes up to the even mantissa
    assert r[3] == 1.0
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-5) <= 3.0e-5 * 2**-8
    assert r[6] == 65536.0


def test_adam_step_matches_closed_form():
    p, g = np.array([1.0, -2.0]), np.array([0.5, -0.25])
    q, m, v = M.adam(p, g, np.zeros(2), np.zeros(2), 1e-3, 0.9, 0.999, 1e-8, 1)
    # first step of bias-corrected Adam moves each parameter by lr * sign(g)
    assert np.allclose(q, p - 1e-3 * np.sign(g), atol=1e-9)
