"""The learned initialiser's network kernels against the NumPy oracle (oracle/mlp_oracle.py).

Forward pass, loss, every parameter gradient and the Adam step of the tensor-core implementation
are compared with the oracle on the same BF16 inputs and FP32 parameters.  The two sum the BF16
products in different orders (FP32 in TMEM against float64), so a hidden activation can round to
the neighbouring BF16 value; the bounds are relative Frobenius errors: 1e-2 for outputs, 2e-2 for
gradients, 1e-3 for the loss.
"""
import numpy as np
import pytest

from fdt_b200.abi import Options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _problem(ndir, batch, seed):
    from fdt_b200 import learned
    from oracle import mlp_oracle as M

    rng = np.random.default_rng(seed)
    p = learned.init_params(ndir, seed)
    k, n, woff, boff, total = learned.geometry(ndir)
    for l in range(5):
        p[boff[l] : boff[l] + n[l]] = 0.05 * rng.normal(size=n[l])
    nin = learned.nin(ndir)
    x = np.zeros((batch, nin), np.float32)
    x[:, :ndir] = rng.uniform(0.05, 1.2, size=(batch, ndir))
    x = M.bf16(x)
    t = rng.normal(size=(batch, 32)).astype(np.float32)
    for kk in range(3):
        v = rng.normal(size=(batch, 3))
        t[:, 3 + 3 * kk : 6 + 3 * kk] = v / np.linalg.norm(v, axis=1, keepdims=True)
    tw = rng.uniform(0.0, 1.0, size=(batch, 32)).astype(np.float32)
    return p, x, t, tw


@pytest.mark.parametrize("ndir,batch", [(64, 300), (279, 200), (288, 517)])
def test_forward_matches_oracle(torch, ndir, batch):
    from fdt_b200 import learned, lib
    from oracle import mlp_oracle as M

    p, x, _, _ = _problem(ndir, batch, 3)
    xd = torch.from_numpy(x).to(torch.bfloat16).cuda()
    out = learned.forward(p, ndir, xd).cpu().numpy()
    assert lib.poll_error() == 0
    ref, _ = M.forward(p, ndir, x)
    assert _rel(out, ref) < 1e-2


@pytest.mark.parametrize("ndir,batch", [(64, 300), (288, 1000)])
def test_gradients_match_oracle(torch, ndir, batch):
    import ctypes as C

    from fdt_b200 import learned, lib
    from oracle import mlp_oracle as M

    p, x, t, tw = _problem(ndir, batch, 5)
    L = lib.load()
    pd = torch.from_numpy(p).cuda()
    g = torch.zeros_like(pd)
    loss = torch.zeros(1, device="cuda")
    xd = torch.from_numpy(x).to(torch.bfloat16).cuda()
    td, wd = torch.from_numpy(t).cuda(), torch.from_numpy(tw).cuda()
    rc = L.bpx_mlp_train_step_dev(ndir, pd.data_ptr(), g.data_ptr(), batch, xd.data_ptr(), td.data_ptr(), wd.data_ptr(),
                                  loss.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.bpx_last_error()
    torch.cuda.synchronize()
    assert lib.poll_error() == 0
    out, cache = M.forward(p, ndir, x)
    lref, dz = M.loss_grad(out, t, tw)
    gref = M.backward(p, ndir, cache, dz)
    assert abs(loss.item() - lref) <= 1e-3 * abs(lref)
    gg = g.cpu().numpy()
    k, n, woff, boff, total = learned.geometry(ndir)
    for l in range(5):
        w = slice(woff[l], woff[l] + n[l] * k[l])
        b = slice(boff[l], boff[l] + n[l])
        assert _rel(gg[w], gref[w]) < 2e-2, ("W", l, _rel(gg[w], gref[w]))
        assert _rel(gg[b], gref[b]) < 2e-2, ("b", l, _rel(gg[b], gref[b]))


def test_adam_matches_oracle(torch):
    import ctypes as C

    from fdt_b200 import lib
    from oracle import mlp_oracle as M

    rng = np.random.default_rng(9)
    n = 100003
    p = rng.normal(size=n).astype(np.float32)
    gr = rng.normal(size=n).astype(np.float32)
    m = (0.1 * rng.normal(size=n)).astype(np.float32)
    v = np.abs(0.1 * rng.normal(size=n)).astype(np.float32)
    pd, gd, md, vd = (torch.from_numpy(a.copy()).cuda() for a in (p, gr, m, v))
    L = lib.load()
    rc = L.bpx_mlp_adam_dev(n, pd.data_ptr(), gd.data_ptr(), md.data_ptr(), vd.data_ptr(), 1e-3, 0.9, 0.999, 1e-8, 7,
                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    # the kernel takes the hyper-parameters as FP32 numbers (1 - 0.999f is 1.3e-5 away from 0.001),
    # so the float64 oracle gets the same values; what remains is FP32 rounding of the updates,
    # which cancel near zero (absolute bounds) -- |g| <= ~5, weights 0.1 and 0.001
    f = lambda x: float(np.float32(x))  # noqa: E731
    pr, mr, vr = M.adam(p.astype(np.float64), gr.astype(np.float64), m.astype(np.float64), v.astype(np.float64),
                        f(1e-3), f(0.9), f(0.999), f(1e-8), 7)
    assert np.allclose(pd.cpu().numpy(), pr, rtol=1e-5, atol=1e-6)
    assert np.allclose(md.cpu().numpy(), mr, rtol=1e-5, atol=1e-7)
    assert np.allclose(vd.cpu().numpy(), vr, rtol=1e-5, atol=1e-8)


def test_decode_inverts_targets(torch):
    """Targets made from a fitted state, fed back as network outputs, decode to that state."""
    from fdt_b200 import learned, lib, synth

    opts = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1)
    prot = synth.three_shell(9, 30)
    data, _ = synth.make_volume(2000, prot, 3, True, 25.0, seed=13)
    d = lib.to_device(data)
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    lib.prepare_data(d)
    params, tau, status = lib.fit(opts, d, bv, bl)
    x, s0 = learned.features(d, bv, bl)
    # adapted widths of realistic size per slot (f0, tau, d, d_std, R, S0, (th, ph, f) x 3)
    lo = torch.tensor([1e-3, 0.0, 1e-5, 1e-5, 0.01, 0.0] + [0.01, 0.01, 0.005] * 3, device="cuda")
    hi = torch.tensor([2e-2, 0.0, 2e-4, 2e-4, 0.05, 0.0] + [0.5, 0.5, 0.05] * 3, device="cuda")
    props = lo[:, None] + (hi - lo)[:, None] * torch.rand((15, 2000), device="cuda")
    props[1] = tau * (0.01 + 0.19 * torch.rand(2000, device="cuda"))
    props[5] = s0 * (0.005 + 0.045 * torch.rand(2000, device="cuda"))
    import ctypes as C

    L = lib.load()
    t = torch.empty((2000, 32), device="cuda")
    w = torch.empty((2000, 32), device="cuda")
    rc = L.bpx_mlp_targets_dev(C.byref(opts), 2000, params.data_ptr(), tau.data_ptr(), props.data_ptr(), s0.data_ptr(),
                               t.data_ptr(), w.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    p2, tau2, props2, st2 = learned.decode(opts, t, s0)
    P, P2 = params.cpu().numpy(), p2.cpu().numpy()
    # voxels inside the decoder's clip ranges (fractions 0.001..0.95, sum < 0.98, d < 0.0049)
    fr = P[:, [3, 6, 9]]
    ok = (fr[:, 0] > 0.01) & (fr.max(1) < 0.95) & (P[:, 1] < 0.0049) & ((fr.sum(1) + np.maximum(P[:, 12], 0.001)) < 0.97)
    assert ok.mean() > 0.5
    assert np.allclose(P2[ok, 0], P[ok, 0], rtol=1e-5)
    assert np.allclose(P2[ok, 1], P[ok, 1], rtol=1e-5)
    for k in range(3):
        f = P[ok, 3 + 3 * k]
        big = f > 0.001
        assert np.allclose(P2[ok, 3 + 3 * k][big], f[big], rtol=1e-5, atol=1e-6)
        th, ph = P[ok, 4 + 3 * k], P[ok, 5 + 3 * k]
        th2, ph2 = P2[ok, 4 + 3 * k], P2[ok, 5 + 3 * k]
        v = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
        v2 = np.stack([np.sin(th2) * np.cos(ph2), np.sin(th2) * np.sin(ph2), np.cos(th2)], 1)
        assert np.all(np.abs((v * v2).sum(1)) > 1 - 1e-5)
    assert np.allclose(tau2.cpu().numpy()[ok], tau.cpu().numpy()[ok], rtol=1e-4)
    pr, pr2 = props.cpu().numpy(), props2.cpu().numpy()
    for q in (0, 1, 2, 3, 5, 6, 7, 8, 14):
        assert np.allclose(pr2[q][ok], pr[q][ok], rtol=1e-4), q


def test_training_reduces_loss(torch):
    """A short training run on forward-model voxels: the loss falls, and on held-out voxels the
    error of the well-determined outputs (f1, d, the first fibre's direction) drops well below
    that of the untrained network.  (The total loss keeps a floor: the state labels are means of
    ten chain samples and the width labels single chain states.)"""
    from fdt_b200 import learned, lib, synth

    opts = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1)
    prot = synth.three_shell(9, 30)
    ts = learned.make_training_set(opts, prot.bvecs, prot.bvals, 20480, seed=21, chunk=8192)
    assert float(ts.tweights[:, 0].mean()) > 0.9
    ho = 4096
    tr = learned.TrainingSet(ts.x[:-ho], ts.targets[:-ho], ts.tweights[:-ho], ts.ndir)
    p0 = learned.output_bias_from_targets(tr, learned.init_params(tr.ndir, 0))
    p1, losses = learned.train(tr, steps=400, batch=1024, lr=2e-3, params=p0, log_every=50)
    assert lib.poll_error() == 0
    assert np.isfinite(losses[-1][1]) and losses[-1][1] < 0.9 * losses[0][1], losses
    xt, tt = ts.x[-ho:].contiguous(), ts.targets[-ho:]

    def errors(p):
        out = learned.forward(p, ts.ndir, xt)
        f1 = float(((out[:, 0] - tt[:, 0]) ** 2).mean())
        d = float(((out[:, 12] - tt[:, 12]) ** 2).mean())
        u, v = out[:, 3:6], tt[:, 3:6]
        c = ((u * v).sum(1).abs() / u.norm(dim=1).clamp_min(1e-9)).clamp(max=1.0)
        return f1, d, float(torch.rad2deg(torch.acos(c)).median())

    e0, e1 = errors(p0), errors(p1)
    assert e1[0] < 0.5 * e0[0] and e1[1] < 0.5 * e0[1], (e0, e1)
    assert e1[2] < 0.5 * e0[2], (e0, e1)


def test_targets_drop_non_finite_labels(torch):
    """A labelling chain that met a non-finite state must not poison training: its non-finite
    labels become zero targets with zero weight (a direction as a whole)."""
    import ctypes as C

    from fdt_b200 import lib

    opts = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1)
    n = 4
    p = torch.tensor([[1000.0, 1e-3, 3e-4, 0.5, 1.0, 2.0, 0.2, 0.5, 0.3, 0.05, 2.0, 1.0, 0.01]] * n, device="cuda")
    p[1, 1] = float("nan")  # d
    p[2, 4] = float("inf")  # theta of fibre 1
    tau = torch.full((n,), 6e-4, device="cuda")
    tau[3] = float("nan")
    s0 = torch.full((n,), 1000.0, device="cuda")
    t = torch.empty((n, 32), device="cuda")
    w = torch.empty((n, 32), device="cuda")
    rc = lib.load().bpx_mlp_targets_dev(C.byref(opts), n, p.data_ptr(), tau.data_ptr(), None, s0.data_ptr(),
                                       t.data_ptr(), w.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    t, w = t.cpu().numpy(), w.cpu().numpy()
    assert np.all(np.isfinite(t)) and np.all(np.isfinite(w))
    assert w[0, 12] == 1.0 and w[1, 12] == 0.0 and t[1, 12] == 0.0
    assert np.all(w[2, 3:6] == 0.0) and np.all(t[2, 3:6] == 0.0) and w[2, 6] > 0.0
    assert w[3, 16] == 0.0 and w[0, 16] > 0.0
