"""The learned form end to end, and what the trained network gains (ablation).

Uses the committed initialiser for the whole-brain protocol (288 measurements).  On held-out
forward-model voxels:
  * the learned pipeline through the host-buffer entry equals the device entry;
  * its posterior against the plain LM-initialised chain, against a long chain, and against the
    method without the network at the same burn-in, with Monte-Carlo standard errors from
    independent chains (see the second test for what is and is not reached).
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
    data, truth = synth.make_volume(4096, prot, 3, True, 25.0, seed=777)
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    base = dict(model=2, nfibres=3, rician=1, f0=1, ardf0=1)
    return dict(params=params, prot=prot, data=data, truth=truth, bv=bv, bl=bl, base=base)


def test_learned_host_entry_matches_device_entry(torch, setup, monkeypatch):
    import ctypes as C

    monkeypatch.setenv("BPX_HOST_CHUNK", "300")  # four sub-volumes through the two buffer sets

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


def test_learned_form_against_plain_gold_and_the_method_without_the_network(torch, setup):
    """Posterior agreement with 8 independent chains per voxel and form (agreement.compare):
      * learned (network start and widths, burn-in 200) against the plain chain (burn-in 1000):
        supported dyads within a median 1 degree; f and d means within 2 Monte-Carlo SE in most
        voxels -- measured 0.75/0.78/0.67 (f1-f3) and 0.76 (d) on the whole-brain configuration,
        where two plain chains at different seeds agree in 0.95/0.95/0.97 and 0.95: the learned form
        does NOT reach the plain form's agreement, which the bounds below record rather than hide;
      * the method without the network at the same burn-in (LM start, the reference's widths,
        burn-in 200) against a long chain (burn-in 5000, 12500 jumps): the learned form is about as
        close to it (f1 within 0.08), so what the network buys is time -- the LM fits it replaces
        (more than 1.8x the voxels/s of the LM start at burn-in 200);
      * against the ground truth of these synthetic voxels (agreement.truth_errors), the learned
        form's posterior means are at least as accurate as the plain form's and the LM start's at
        burn-in 200 for the two largest fibres (f error and dyad angle) -- measured on 4096
        whole-brain voxels: f1 0.0145 vs 0.0164 (plain), first dyad 1.27 vs 1.37 degrees."""
    from fdt_b200 import learned, lib

    s = setup
    n = 1024
    d = lib.to_device(s["data"][:n])
    lib.prepare_data(d)
    o = Options.make(**s["base"])
    sets = learned.posterior_study(o, d, s["bv"], s["bl"], s["params"], R=8, seed=300)
    rep = learned.study_report(sets, s["truth"])
    yard, acc, lm = (rep["vs_plain"][k] for k in ("plain_other_seed", "learned", "lm_burnin200"))
    print("learned vs plain", acc, "\nplain vs plain", yard, "\nLM burn-in 200 vs plain", lm)
    print("vs gold", rep["vs_gold"])
    assert min(yard["f_within_2se"]) >= 0.90 and yard["d_within_2se"] >= 0.90, yard  # the statistic itself
    assert acc["dyad_median_deg_supported"] < 1.0, acc
    assert acc["f_within_2se"][0] >= 0.62 and acc["f_within_2se"][1] >= 0.62, acc
    assert acc["d_within_2se"] >= 0.60, acc
    g = rep["vs_gold"]
    assert g["learned"]["f_within_2se"][0] >= g["lm_burnin200"]["f_within_2se"][0] - 0.08, g
    assert g["learned"]["dyad_median_deg_supported"] < 1.0, g
    t = rep["vs_truth"]
    print("vs truth", t)
    for k in (0, 1):
        for other in ("plain", "lm_burnin200"):
            assert t["learned"]["f_abs_median"][k] <= 1.1 * t[other]["f_abs_median"][k], (k, other, t)
            assert t["learned"]["dyad_deg_median"][k] <= 1.1 * t[other]["dyad_deg_median"][k], (k, other, t)

    # speed: the learned pipeline against the LM-started chain at the same burn-in
    lo = Options.make(**s["base"], nburn=200, seed=12)
    y = s["data"]
    for _ in range(2):  # second pass timed (first loads modules, grows workspaces)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        learned.xfibres_learned(lo, lib.to_device(y), s["bv"], s["bl"], s["params"], freeze=0)
        torch.cuda.synchronize()
        t_learned = time.perf_counter() - t0
        t0 = time.perf_counter()
        lib.xfibres_dev(lo, lib.to_device(y), s["bv"], s["bl"])
        torch.cuda.synchronize()
        t_lm200 = time.perf_counter() - t0
    assert t_lm200 > 1.8 * t_learned, (t_learned, t_lm200)
