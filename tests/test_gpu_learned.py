"""The learned form end to end, and what the trained network gains (ablation).

Uses the committed initialiser for the whole-brain protocol (288 measurements).  On held-out
forward-model voxels:
  * the learned pipeline through the host-buffer entry equals the device entry;
  * started from the network's state and proposal widths with a burn-in of 200, the chain's
    posterior agrees with the plain LM-initialised chain (burn-in 1000): median dyad-1 difference
    below 1 degree, and fractions within 2 Monte-Carlo standard errors nearly as often as two
    plain chains with different seeds agree with each other;
  * ablation -- the same short chain started without the network (the data-independent state the
    network's output biases encode, with initialise_props widths) misses the plain chain's
    dyads by several times more, and the learned pipeline takes a fraction of the plain
    pipeline's time.
"""
import time

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


@pytest.fixture(scope="module")
def setup(torch):
    from fdt_b200 import learned, lib, synth

    params, meta = learned.load_weights(learned.default_weights_path("whole_brain"))
    prot = synth.three_shell(18, 90)
    assert int(meta["ndir"]) == prot.ndir
    data, _ = synth.make_volume(4096, prot, 3, True, 25.0, seed=777)
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    base = dict(model=2, nfibres=3, rician=1, f0=1, ardf0=1)
    plain = lib.xfibres_dev(Options.make(**base, seed=11), lib.to_device(data), bv, bl)
    return dict(params=params, prot=prot, data=data, bv=bv, bl=bl, base=base, plain=plain)


def test_learned_host_entry_matches_device_entry(torch, setup):
    import ctypes as C

    from fdt_b200 import learned, lib
    from fdt_b200.abi import Volume

    s = setup
    o = Options.make(**s["base"], nburn=200, njumps=250, seed=5)
    n = 1000
    y = np.ascontiguousarray(s["data"][:n])
    dev = learned.xfibres_learned(o, lib.to_device(y), s["bv"], s["bl"], s["params"], freeze=0)
    t, oo = lib.alloc_outputs(o, n, device="cpu")
    v = Volume()
    v.nvox, v.ndir = y.shape
    bvh = np.ascontiguousarray(s["prot"].bvecs, np.float32)
    blh = np.ascontiguousarray(s["prot"].bvals, np.float32)
    v.data, v.bvecs, v.bvals = y.ctypes.data, bvh.ctypes.data, blh.ctypes.data
    v.grad = None
    v.voxel_offset = 0
    p = np.ascontiguousarray(s["params"], np.float32)
    rc = lib.load().bpx_xfibres_learned_host(C.byref(o), C.byref(v), p.ctypes.data, 0, C.byref(oo))
    assert rc == 0, lib.load().bpx_last_error()
    for k in ("th", "ph", "f", "mean_d", "mean_S0", "dyads"):
        assert np.allclose(t[k].numpy(), dev[k].cpu().numpy(), rtol=1e-6, atol=0), k


def test_learned_start_matches_plain_and_beats_no_network(torch, setup):
    import ctypes as C

    from fdt_b200 import learned, lib

    s = setup
    o = Options.make(**s["base"])
    lo = Options.make(**s["base"], nburn=200, seed=12)
    t0 = time.perf_counter()
    learned_out = learned.xfibres_learned(lo, lib.to_device(s["data"]), s["bv"], s["bl"], s["params"], freeze=0)
    torch.cuda.synchronize()
    t_learned = time.perf_counter() - t0
    t0 = time.perf_counter()
    plain2 = lib.xfibres_dev(Options.make(**s["base"], seed=13), lib.to_device(s["data"]), s["bv"], s["bl"])
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    acc = learned.summary(o, learned_out, s["plain"])
    ref = learned.summary(o, plain2, s["plain"])
    assert acc["dyad_median_deg"][0] < 1.0, acc
    assert acc["f_within_2se"][0] >= ref["f_within_2se"][0] - 0.15, (acc, ref)
    assert acc["d_rel_median"] < 0.05, acc

    # ablation: the same short chain without the network -- every voxel starts from the state the
    # output biases alone encode (the training set's mean) with the reference's initial widths
    d = lib.to_device(s["data"])
    lib.prepare_data(d)
    x, s0 = learned.features(d, s["bv"], s["bl"])
    k, n, woff, boff, total = learned.geometry(s["prot"].ndir)
    bias_only = np.zeros_like(s["params"])
    bias_only[boff[4] : boff[4] + 32] = s["params"][boff[4] : boff[4] + 32]
    bias_only[boff[4] + 3 : boff[4] + 12] = np.tile([0.0, 0.0, 1.0], 3)  # a fixed direction per fibre
    out = learned.forward(bias_only, s["prot"].ndir, x)
    p0, tau0, _, st0 = learned.decode(lo, out, s0)
    rec, _ = lib.mcmc_ex(lo, d, s["bv"], s["bl"], p0, tau0, props_in=None, freeze=0, status=st0)
    naive = lib.finish(lo, rec)
    abl = learned.summary(o, naive, s["plain"])
    # the network's start beats the data-independent one on both dyads and on f1's agreement
    assert abl["dyad_median_deg"][0] > 2.5 * acc["dyad_median_deg"][0], (abl, acc)
    assert abl["dyad_median_deg"][1] > 2.0 * acc["dyad_median_deg"][1], (abl, acc)
    assert acc["f_within_2se"][0] > abl["f_within_2se"][0] + 0.15, (abl, acc)
    assert t_learned < 0.75 * t_plain, (t_learned, t_plain)
