"""The bedpostx driver end to end on a small synthetic subject (NIfTI in, NIfTI out): the merged
and post-processed volumes equal the library's outputs placed at the mask's voxels, and rebuilding
the merged volumes from the part files (merge_parts_gpu semantics) gives the same volumes."""
import os

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


def test_subject_directory_run_and_merge(torch, tmp_path):
    from fdt_b200 import bedpostx, nifti, synth

    prot = synth.truncated_three_shell(65)
    shape = (9, 8, 5)
    mask = np.zeros(shape, np.float32)
    x, y, z = np.meshgrid(*[np.linspace(-1, 1, s) for s in shape], indexing="ij")
    mask[(x**2 + y**2 + z**2) < 0.8] = 1
    n = int(mask.sum())
    vox, _ = synth.make_volume(n, prot, 2, True, 25.0, seed=3)
    data4 = nifti.from_matrix(vox, mask)
    subj = tmp_path / "subj"
    subj.mkdir()
    hdr = nifti.Header(dim=(4,) + shape + (65, 1, 1, 1), pixdim=(1.0, 2.0, 2.0, 2.0, 1.0, 1, 1, 1))
    nifti.write(str(subj / "data.nii.gz"), data4, like=hdr)
    nifti.write(str(subj / "nodif_brain_mask.nii.gz"), mask, like=hdr)
    np.savetxt(subj / "bvecs", prot.bvecs)
    np.savetxt(subj / "bvals", prot.bvals[None, :])
    argv = [str(subj), "--nf", "2", "--model", "2", "--rician", "--f0", "--ardf0", "--bi", "100", "--nj", "200",
            "--se", "10", "--parts", "3"]
    bedpostx.main(argv)
    out = str(subj) + ".bedpostX"
    opts = Options.make(model=2, nfibres=2, rician=1, f0=1, ardf0=1, nburn=100, njumps=200, sampleevery=10)
    host = bedpostx.run(str(subj), opts, outdir=str(tmp_path / "direct"))
    f1, h = nifti.read(os.path.join(out, "merged_f1samples.nii.gz"))
    assert f1.shape == shape + (20,) and h.pixdim[1] == 2.0
    assert np.array_equal(nifti.to_matrix(f1, mask), host["f"][0].T)
    for name in ("dyads1", "dyads2", "dyads2_thr0.05", "dyads2_thr0.05_modf2", "dyads1_dispersion", "mean_fsumsamples",
                 "mean_th1samples", "mean_f2samples", "mean_d_stdsamples", "mean_tausamples", "mean_f0samples",
                 "nodif_brain_mask"):
        assert os.path.exists(os.path.join(out, name + ".nii.gz")), name
    d1, _ = nifti.read(os.path.join(out, "dyads1.nii.gz"))
    assert np.allclose(nifti.to_matrix(d1, mask), host["dyads"][0].T)
    # merge_parts_gpu semantics: rebuild the merged volumes from the part files
    merged_before = nifti.read(os.path.join(out, "merged_ph2samples.nii.gz"))[0]
    os.remove(os.path.join(out, "merged_ph2samples.nii.gz"))
    bedpostx.main(argv[:1] + ["merge"] + argv[1:])
    merged_after = nifti.read(os.path.join(out, "merged_ph2samples.nii.gz"))[0]
    assert np.array_equal(merged_after, merged_before)


def test_gradnonlin_reads_grad_dev_in_mask_order(torch, tmp_path):
    """--gradnonlin reads grad_dev (X x Y x Z x 9) at the mask's voxels and corrects the b-matrix
    per voxel on the device: the driver's outputs equal the library run on the per-voxel b-matrix
    of the same tensors taken voxel by voxel here."""
    from fdt_b200 import bedpostx, lib, nifti, synth

    prot = synth.truncated_three_shell(33)
    shape = (6, 5, 3)
    mask = np.zeros(shape, np.float32)
    mask[1:5, 1:4, :] = 1
    n = int(mask.sum())
    vox, _ = synth.make_volume(n, prot, 1, False, 30.0, seed=8)
    rng = np.random.default_rng(4)
    grad = (0.02 * rng.normal(size=shape + (9,))).astype(np.float32)
    subj = tmp_path / "g"
    subj.mkdir()
    hdr = nifti.Header(dim=(4,) + shape + (33, 1, 1, 1))
    nifti.write(str(subj / "data.nii.gz"), nifti.from_matrix(vox, mask), like=hdr)
    nifti.write(str(subj / "nodif_brain_mask.nii.gz"), mask, like=hdr)
    nifti.write(str(subj / "grad_dev.nii.gz"), grad, like=hdr)
    np.savetxt(subj / "bvecs", prot.bvecs)
    np.savetxt(subj / "bvals", prot.bvals[None, :])
    o = Options.make(model=1, nfibres=1, nburn=50, njumps=100, sampleevery=10, gradnonlin=1)
    got = bedpostx.run(str(subj), o, outdir=str(tmp_path / "out"))
    idx = np.argwhere(mask.transpose(2, 1, 0) != 0)[:, ::-1]  # x fastest
    gm = np.stack([grad[i, j, k] for i, j, k in idx])
    bv, bl = lib.gradnonlin(lib.to_device(gm), lib.to_device(prot.bvecs), lib.to_device(prot.bvals))
    want = lib.xfibres_dev(o, lib.to_device(vox), bv, bl)
    for k in ("th", "ph", "f", "mean_d"):
        assert np.array_equal(got[k], want[k].cpu().numpy()), k
