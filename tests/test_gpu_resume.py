"""Checkpoint and resume of the chain (bpx_mcmc_stretch_dev): a chain run as consecutive stretches,
each started from the previous one's state, widths and acceptance counts, equals one run bit for bit."""
import numpy as np
import pytest

from fdt_b200 import synth
from fdt_b200.abi import Options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def lib(torch):
    from fdt_b200 import lib as L

    L.load()
    return L


@pytest.mark.parametrize("kw,cuts", [
    (dict(model=2, nfibres=3, rician=1, f0=1, ardf0=1), [53]),    # mid recording, between two width updates
    (dict(model=1, nfibres=2), [40, 77]),                          # at the end of the burn-in, mid recording
    (dict(model=3, nfibres=2, rician=1), [1, 119]),                # after one iteration, before the last
], ids=["m2_ric_f0", "m1", "m3_ric"])
def test_stretches_reproduce_one_chain(torch, lib, kw, cuts):
    o = Options.make(nburn=40, njumps=80, sampleevery=8, updateproposalevery=10, **kw)
    prot = synth.three_shell(9, 30) if o.model >= 2 else synth.single_shell_64()
    y, _ = synth.make_volume(96, prot, o.nfibres, o.model >= 2, 25.0, seed=5)
    d = torch.from_numpy(np.ascontiguousarray(y, np.float32)).cuda()
    bv = torch.from_numpy(np.ascontiguousarray(prot.bvecs, np.float32)).cuda()
    bl = torch.from_numpy(np.ascontiguousarray(prot.bvals, np.float32)).cuda()
    if o.rician:
        lib.prepare_data(d)
    p, t, _ = lib.fit(o, d, bv, bl)
    total = o.nburn + o.njumps

    rec_one, state_one = lib.mcmc_stretch(o, d, bv, bl, 0, total, params=p, tau=t)
    assert torch.equal(rec_one, lib.mcmc(o, d, bv, bl, p, t))  # the whole chain as one stretch

    rec, state, begin = None, None, 0
    for end in cuts + [total]:
        rec, state = lib.mcmc_stretch(o, d, bv, bl, begin, end, params=p if begin == 0 else None,
                                      tau=t if begin == 0 else None, state=state, records=rec)
        begin = end
    torch.cuda.synchronize()
    assert torch.equal(rec, rec_one)
    for key in ("state", "props", "acc"):
        assert torch.equal(state[key], state_one[key]), key
