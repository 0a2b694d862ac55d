"""CPU checks of the posterior-mean labels of the initialiser's training set (learned.py)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from fdt_b200 import learned
from fdt_b200.abi import Options


def _records(ns, n, K, th, ph, f, seed=0):
    rng = np.random.default_rng(seed)
    rec = np.zeros((6 + 3 * K, ns, n), np.float32)
    rec[0] = 1e-3 + 1e-4 * rng.standard_normal((ns, n))   # d
    rec[1] = 0.02                                           # f0
    rec[2] = 5e-4                                           # tau
    rec[3] = 3e-4                                           # d_std
    rec[5] = 1000.0 + rng.standard_normal((ns, n))          # S0
    for k in range(K):
        rec[6 + 3 * k] = th[k]
        rec[7 + 3 * k] = ph[k]
        rec[8 + 3 * k] = f[k]
    return rec


def test_mean_labels_scalars_and_layout():
    o = Options.make(model=2, nfibres=2, rician=1, f0=1)
    rec = _records(10, 7, 2, th=[np.full((10, 7), 0.7), np.full((10, 7), 1.9)],
                   ph=[np.full((10, 7), 0.3), np.full((10, 7), -2.0)], f=[0.5, 0.2])
    params, tau = learned.state_mean_from_records(o, torch.from_numpy(rec))
    assert params.shape == (7, o.nparams_fit)
    p = params.numpy()
    np.testing.assert_allclose(p[:, 0], rec[5].mean(0), rtol=1e-6)            # S0
    np.testing.assert_allclose(p[:, 1], rec[0].mean(0), rtol=1e-5)            # d
    np.testing.assert_allclose(p[:, 2], 3e-4, rtol=1e-6)                      # d_std
    np.testing.assert_allclose(p[:, 3], 0.5, rtol=1e-6)                       # f1
    np.testing.assert_allclose(p[:, 4], 0.7, atol=1e-5)                       # th1
    np.testing.assert_allclose(p[:, 5], 0.3, atol=1e-5)                       # ph1
    np.testing.assert_allclose(p[:, 6], 0.2, rtol=1e-6)                       # f2
    v = lambda t, f: np.array([np.sin(t) * np.cos(f), np.sin(t) * np.sin(f), np.cos(t)])  # noqa: E731
    # fibre 2 (theta 1.9 > pi/2) comes back as the antipode with theta < pi/2
    np.testing.assert_allclose(np.abs(v(p[0, 7], p[0, 8]) @ v(1.9, -2.0)), 1.0, atol=1e-6)
    assert p[0, 7] <= np.pi / 2
    np.testing.assert_allclose(p[:, 9], 0.02, rtol=1e-6)                      # f0
    np.testing.assert_allclose(tau.numpy(), 5e-4, rtol=1e-6)


def test_mean_direction_ignores_sign_flips():
    """Samples of one axis drawn as v or -v (theta -> pi - theta, phi -> phi + pi) average to it."""
    o = Options.make(model=1, nfibres=1)
    rng = np.random.default_rng(2)
    th0, ph0 = 0.4, 1.1
    flip = rng.random((20, 5)) < 0.5
    th = np.where(flip, np.pi - th0, th0) + 0.01 * rng.standard_normal((20, 5))
    ph = np.where(flip, ph0 + np.pi, ph0) + 0.01 * rng.standard_normal((20, 5))
    rec = _records(20, 5, 1, th=[th], ph=[ph], f=[0.6])
    params, _ = learned.state_mean_from_records(o, torch.from_numpy(rec))
    p = params.numpy()
    u = np.array([np.sin(p[:, 3]) * np.cos(p[:, 4]), np.sin(p[:, 3]) * np.sin(p[:, 4]), np.cos(p[:, 3])])
    w = np.array([np.sin(th0) * np.cos(ph0), np.sin(th0) * np.sin(ph0), np.cos(th0)])
    assert np.all(np.abs(w @ u) > np.cos(np.deg2rad(1.0)))
