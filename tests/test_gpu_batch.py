"""The batched form (bpx_batch_*) against per-item runs, and the autotuner.

Items of mixed models, fibre counts and measurement counts (two of them sharing a bucket, so
their voxels are packed together) run as one CUDA-graph launch; every output must equal the
plain per-item pipeline (bpx_xfibres_dev) with the bucket's launch layout exactly -- the chains
are keyed by each item's own voxel indices, so packing changes nothing -- and a replay of the
graph must give the same outputs again.
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


def _items(torch):
    from fdt_b200 import lib, synth

    spec = [  # model, nfibres, ndir, nvox, voxel_offset
        (1, 1, 33, 300, 0),
        (2, 3, 65, 410, 1000),
        (2, 2, 65, 257, 0),
        (1, 2, 129, 333, 77),
        (2, 3, 65, 129, 5000),
    ]
    items = []
    for i, (model, K, M, n, off) in enumerate(spec):
        prot = synth.truncated_three_shell(M)
        y, _ = synth.make_volume(n, prot, K, model == 2, 20.0, seed=100 + i)
        items.append(dict(data=lib.to_device(y), host=y, bvecs=lib.to_device(prot.bvecs),
                          bvals=lib.to_device(prot.bvals), model=model, nfibres=K, voxel_offset=off))
    # items 1 and 4 share model, K, ndir and (so that they form one bucket) the same b-matrix tensors
    items[4]["bvecs"], items[4]["bvals"] = items[1]["bvecs"], items[1]["bvals"]
    return items


def test_batch_equals_per_item_runs(torch):
    from fdt_b200 import lib

    opts = Options.make(rician=1, f0=1, ardf0=1, nburn=60, njumps=100, sampleevery=10)
    items = _items(torch)
    batch = lib.Batch(opts, items, autotune=True)
    bks = batch.buckets()
    assert len(bks) == 4 and sum(b["voxels"] for b in bks) == sum(int(it["data"].shape[0]) for it in items)
    assert any(b["items"] == 2 for b in bks)
    for b in bks:
        assert b["tpv"] * b["mpl"] >= b["ndir"]
    outs = [{k: v.clone() for k, v in o.items()} for o in batch.run()]
    torch.cuda.synchronize()
    outs2 = batch.run()
    torch.cuda.synchronize()
    for i, it in enumerate(items):
        # the same launch layout as the item's bucket: another threads-per-voxel sums the likelihood
        # terms in another order, and the chains then agree statistically, not bit for bit
        bk = [b for b in bks if (b["model"], b["nfibres"], b["ndir"]) == (it["model"], it["nfibres"],
                                                                           int(it["data"].shape[1]))][0]
        o = Options.make(rician=1, f0=1, ardf0=1, nburn=60, njumps=100, sampleevery=10, model=it["model"],
                         nfibres=it["nfibres"], mcmc_tpv=bk["tpv"], mcmc_mpl=bk["mpl"])
        ref = lib.xfibres_dev(o, lib.to_device(it["host"]), it["bvecs"], it["bvals"], voxel_offset=it["voxel_offset"])
        for k in ("th", "ph", "f", "mean_d", "mean_S0", "mean_f", "dyads", "status"):
            a, b = outs[i][k].cpu().numpy(), ref[k].cpu().numpy()
            assert np.array_equal(a, b), (i, k)
            assert np.array_equal(outs2[i][k].cpu().numpy(), a), (i, k, "replay")
    batch.close()


def test_autotuner_picks_a_covering_layout(torch):
    from fdt_b200 import lib, synth

    prot = synth.truncated_three_shell(129)
    opts = Options.make(model=2, nfibres=2, rician=1)
    tpv, mpl, t = lib.autotune_layout(opts, lib.to_device(prot.bvecs), lib.to_device(prot.bvals), sample=1024)
    assert tpv * mpl >= 129 and (tpv, mpl) in t
    assert all(v > 0 for v in t.values()) and len(t) >= 2
    assert t[(tpv, mpl)] == min(t.values())


def test_learned_items_in_a_batch_equal_the_learned_pipeline(torch):
    """Items started from the initialiser network run in the same graph as LM-started items and
    give exactly what the standalone learned pipeline gives with the bucket's layout."""
    from fdt_b200 import learned, lib, synth

    params, meta = learned.load_weights(learned.default_weights_path("whole_brain"))
    prot = synth.three_shell(18, 90)
    mlp = torch.from_numpy(params).cuda()
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    ys = [synth.make_volume(n, prot, 3, True, 25.0, seed=400 + n)[0] for n in (700, 300)]
    opts = Options.make(rician=1, f0=1, ardf0=1, nburn=300, njumps=100, sampleevery=10)
    items = [
        dict(data=lib.to_device(ys[0]), bvecs=bv, bvals=bl, model=2, nfibres=3, mlp=mlp, nburn=80, freeze=0),
        dict(data=lib.to_device(ys[1]), bvecs=bv, bvals=bl, model=2, nfibres=3, voxel_offset=9000),
        dict(data=lib.to_device(ys[1]), bvecs=bv, bvals=bl, model=2, nfibres=3, mlp=mlp, nburn=80, freeze=2,
             voxel_offset=9000),
    ]
    batch = lib.Batch(opts, items, autotune=False)
    bks = batch.buckets()
    assert len(bks) == 3
    outs = batch.run()
    torch.cuda.synchronize()
    assert lib.poll_error() == 0
    lay = (bks[0]["tpv"], bks[0]["mpl"])
    for i, (n_b, fr) in [(0, (80, 0)), (2, (80, 2))]:
        o = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=n_b, njumps=100, sampleevery=10,
                         mcmc_tpv=lay[0], mcmc_mpl=lay[1])
        off = items[i].get("voxel_offset", 0)
        ref = learned.xfibres_learned(o, lib.to_device(ys[0 if i == 0 else 1]), bv, bl, mlp, freeze=fr,
                                      out=None) if off == 0 else None
        if off:
            d = lib.to_device(ys[1])
            t, oo = lib.alloc_outputs(o, d.shape[0])
            import ctypes as C

            vol = lib.make_volume(d, bv, bl, voxel_offset=off)
            rc = lib.load().bpx_xfibres_learned_dev(C.byref(o), C.byref(vol), mlp.data_ptr(), fr, C.byref(oo),
                                                    C.c_void_p(torch.cuda.current_stream().cuda_stream))
            assert rc == 0
            ref = t
        for k in ("th", "ph", "f", "mean_d", "dyads", "status"):
            assert np.array_equal(outs[i][k].cpu().numpy(), ref[k].cpu().numpy()), (i, k)
    o = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=300, njumps=100, sampleevery=10,
                     mcmc_tpv=bks[1]["tpv"], mcmc_mpl=bks[1]["mpl"])
    ref = lib.xfibres_dev(o, lib.to_device(ys[1]), bv, bl, voxel_offset=9000)
    for k in ("th", "f", "dyads"):
        assert np.array_equal(outs[1][k].cpu().numpy(), ref[k].cpu().numpy()), (1, k)
    batch.close()
