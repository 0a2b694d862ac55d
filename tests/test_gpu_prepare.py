"""remove_NonPositive_entries on the GPU (bpx_prepare_data_dev) against the oracle, bit for bit.

The reference (CUDA/xfibres_gpu.cu:350-367) replaces every non-positive sample of a voxel whose
maximum is positive by the voxel's smallest positive sample, and leaves voxels that are all
positive, or all non-positive, as they are.  The GPU kernel must give exactly the oracle's floats.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _volume(nvox: int, ndir: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    y = rng.uniform(1.0, 1000.0, (nvox, ndir)).astype(np.float32)
    kind = np.arange(nvox) % 6
    # 0: all positive; 1: a few non-positive samples; 2: half non-positive; 3: all non-positive;
    # 4: all zero; 5: one positive sample among zeros and negatives
    few = rng.random((nvox, ndir)) < 0.05
    y[kind == 1] = np.where(few[kind == 1], -rng.uniform(0, 10, few[kind == 1].shape), y[kind == 1])
    half = rng.random((nvox, ndir)) < 0.5
    y[kind == 2] = np.where(half[kind == 2], np.where(half[kind == 2] & (rng.random((nvox, ndir))[kind == 2] < 0.5), 0.0, -3.0), y[kind == 2])
    y[kind == 3] = -rng.uniform(0, 5, ((kind == 3).sum(), ndir))
    y[kind == 4] = 0.0
    sel = np.where(kind == 5)[0]
    y[sel] = np.where(rng.random((len(sel), ndir)) < 0.5, 0.0, -1.0)
    y[sel, rng.integers(0, ndir, len(sel))] = 7.5
    return np.ascontiguousarray(y, np.float32)


@pytest.mark.parametrize("nvox,ndir", [(1, 7), (61, 33), (600, 288), (97, 512), (0, 64)])
def test_prepare_data_bit_exact(torch, nvox, ndir):
    from fdt_b200 import lib

    y = _volume(nvox, ndir, seed=nvox * 1000 + ndir)
    want = O.prepare_data(y)
    d = lib.to_device(y) if nvox else torch.zeros((0, ndir), device="cuda")
    lib.prepare_data(d)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    if nvox >= 6:
        # the cases the rule distinguishes are all present and behave as the reference's rule says
        kind = np.arange(nvox) % 6
        assert np.array_equal(got[kind == 0], y[kind == 0])
        assert np.array_equal(got[kind == 3], y[kind == 3]) and np.array_equal(got[kind == 4], y[kind == 4])
        assert np.all(got[(kind == 1) | (kind == 2) | (kind == 5)] > 0)
        assert np.all(got[kind == 5] == 7.5)
