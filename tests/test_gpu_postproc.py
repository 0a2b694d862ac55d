"""bedpostx_postproc arithmetic on the GPU (bpx_postproc_dev) against a NumPy restatement of
make_dyadic_vectors.cc:60-92 (mean dyadic tensor, principal eigenvector, 1 - max|eigenvalue|) and
of the fslmaths / maskdyads steps of CUDA/bedpostx_postproc_gpu.sh:20-49, on the outputs of a
short chain.  Tolerances: means and dispersions 1e-5 absolute (FP64 sums of FP32 samples),
eigenvectors (stored in FP32) within 0.05 degrees (sign-free)."""
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


def test_postproc_matches_numpy(torch):
    from fdt_b200 import lib, synth

    opts = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=100, njumps=200, sampleevery=10)
    prot = synth.three_shell(9, 30)
    y, _ = synth.make_volume(600, prot, 3, True, 20.0, seed=5)
    out = lib.xfibres_dev(opts, lib.to_device(y), lib.to_device(prot.bvecs), lib.to_device(prot.bvals))
    pp = lib.postproc(opts, out, 0.05)
    torch.cuda.synchronize()
    th, ph = out["th"].cpu().numpy().astype(np.float64), out["ph"].cpu().numpy().astype(np.float64)
    mf = out["mean_f"].cpu().numpy()
    dy = out["dyads"].cpu().numpy()
    K, ns, n = th.shape
    assert np.allclose(pp["mean_th"].cpu().numpy(), th.mean(1), atol=1e-5)
    assert np.allclose(pp["mean_ph"].cpu().numpy(), ph.mean(1), atol=1e-5)
    assert np.allclose(pp["mean_fsum"].cpu().numpy(), mf.sum(0), atol=1e-5)
    disp = pp["dispersion"].cpu().numpy()
    for k in range(K):
        v = np.stack([np.sin(th[k]) * np.cos(ph[k]), np.sin(th[k]) * np.sin(ph[k]), np.cos(th[k])], -1)  # [ns][n][3]
        T = np.einsum("sni,snj->nij", v, v) / ns
        w, V = np.linalg.eigh(T)
        assert np.allclose(disp[k], 1.0 - np.abs(w).max(1), atol=1e-5)
        pv = V[:, :, -1]
        c = np.abs((pv * dy[k].T).sum(1))
        assert np.all(c > np.cos(np.deg2rad(0.05))), k  # dyads are stored in FP32
    thr, modf = pp["dyads_thr"].cpu().numpy(), pp["dyads_modf"].cpu().numpy()
    for k in range(1, K):
        keep = (mf[k] >= 0.05) & (mf[k] != 0)
        want = dy[k] * keep[None, :]
        assert np.array_equal(thr[k], want)
        ratio = np.where(mf[0] != 0, mf[k] / np.where(mf[0] != 0, mf[0], 1), 0)
        assert np.allclose(modf[k], want * ratio[None, :], rtol=1e-6, atol=1e-7)
