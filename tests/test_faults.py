"""Host-side fault injection (no GPU): damaged inputs to the bedpostx driver end in a clear error
naming the file or the mismatch, before any device work."""
import os

import numpy as np
import pytest

from fdt_b200 import bedpostx, nifti, synth
from fdt_b200.abi import Options


def _subject(d, shape=(4, 3, 2), M=16, mask_shape=None):
    prot = synth.single_shell_64()
    rng = np.random.default_rng(1)
    data = rng.uniform(100, 1000, size=shape + (M,)).astype(np.float32)
    nifti.write(os.path.join(d, "data.nii.gz"), data)
    nifti.write(os.path.join(d, "nodif_brain_mask.nii.gz"), np.ones(mask_shape or shape, np.uint8))
    np.savetxt(os.path.join(d, "bvecs"), prot.bvecs[:, :M])
    np.savetxt(os.path.join(d, "bvals"), prot.bvals[None, :M])
    return data


def test_a_consistent_subject_reads(tmp_path):
    data = _subject(str(tmp_path))
    y, mask, hdr, bvecs, bvals = bedpostx.read_subject(str(tmp_path))
    assert y.shape == (int(np.prod(data.shape[:3])), data.shape[3]) and bvecs.shape == (3, 16)


def test_mask_data_mismatch(tmp_path):
    _subject(str(tmp_path), mask_shape=(4, 3, 3))
    with pytest.raises(ValueError, match="different spatial shapes"):
        bedpostx.read_subject(str(tmp_path))


def test_bvecs_bvals_count_mismatch(tmp_path):
    _subject(str(tmp_path))
    np.savetxt(os.path.join(str(tmp_path), "bvals"), np.ones((1, 15)))
    with pytest.raises(ValueError, match="do not match the 16 volumes"):
        bedpostx.read_subject(str(tmp_path))


def test_missing_mask(tmp_path):
    _subject(str(tmp_path))
    os.remove(os.path.join(str(tmp_path), "nodif_brain_mask.nii.gz"))
    with pytest.raises(FileNotFoundError, match="nodif_brain_mask"):
        bedpostx.read_subject(str(tmp_path))


@pytest.mark.parametrize("damage,match", [
    (lambda raw: raw[:200], "too short"),
    (lambda raw: raw[:-40], "truncated"),
    (lambda raw: raw[:344] + b"xx1\x00" + raw[348:], "magic"),
    (lambda raw: raw[:70] + np.int16(1234).tobytes() + raw[72:], "datatype"),
])
def test_damaged_nifti(tmp_path, damage, match):
    p = os.path.join(str(tmp_path), "v.nii")
    nifti.write(p, np.ones((3, 3, 3), np.float32))
    raw = open(p, "rb").read()
    open(p, "wb").write(damage(raw))
    with pytest.raises(ValueError, match=match):
        nifti.read(p)


def test_truncated_part_file(tmp_path):
    o = Options.make(model=1, nfibres=1, njumps=10, sampleevery=5)
    n, ns = 10, 2
    out = {"th": np.zeros((1, ns, n)), "ph": np.zeros((1, ns, n)), "f": np.zeros((1, ns, n))}
    for key in bedpostx.MEAN_KEYS.values():
        out[key] = np.zeros(n)
    bedpostx.write_parts(str(tmp_path), out, o, 2)
    f = os.path.join(str(tmp_path), "diff_parts", "data_part_0001", "th1samplesJ")
    raw = open(f, "rb").read()
    open(f, "wb").write(raw[:-8])
    with pytest.raises(ValueError, match="expected 10 values, found 9"):
        bedpostx.join_parts(str(tmp_path), "th1samples", n, ns, 2)
