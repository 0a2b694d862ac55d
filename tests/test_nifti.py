"""Host side of the bedpostx driver (no GPU): NIfTI-1 read/write, FSL's masked-voxel order, and the
part-file layout of Samples::save / merge_parts_gpu (raw float64 [nsamples][part voxels])."""
import gzip
import os
import struct

import numpy as np
import pytest

from fdt_b200 import bedpostx, nifti
from fdt_b200.abi import Options


@pytest.mark.parametrize("ext", [".nii", ".nii.gz"])
def test_roundtrip_keeps_data_and_geometry(tmp_path, ext):
    rng = np.random.default_rng(0)
    a = rng.normal(size=(5, 4, 3, 7)).astype(np.float32)
    like = nifti.Header(dim=(4, 5, 4, 3, 7, 1, 1, 1), pixdim=(1.0, 2.0, 2.0, 2.5, 3.0, 1, 1, 1), qform_code=1,
                        sform_code=1, quatern=(0.0, 0.0, 0.0, -10.0, -12.0, 5.0),
                        srow=((2.0, 0.0, 0.0, -10.0), (0.0, 2.0, 0.0, -12.0), (0.0, 0.0, 2.5, 5.0)))
    p = str(tmp_path / ("x" + ext))
    nifti.write(p, a, like=like, cal=(-1.0, 1.0))
    b, h = nifti.read(p)
    assert b.shape == a.shape and np.array_equal(b, a)
    assert h.dim[:5] == (4, 5, 4, 3, 7)
    assert h.pixdim[1:4] == (2.0, 2.0, 2.5)
    assert h.sform_code == 1 and h.srow[2][3] == 5.0
    assert (h.cal_min, h.cal_max) == (-1.0, 1.0)
    raw = (gzip.open(p, "rb") if ext.endswith(".gz") else open(p, "rb")).read()
    assert struct.unpack("<i", raw[:4])[0] == 348 and raw[344:348] == b"n+1\x00"
    assert struct.unpack("<f", raw[108:112])[0] == 352.0
    assert len(raw) == 352 + a.size * 4
    # x fastest in the file
    assert struct.unpack("<f", raw[352 + 4 : 356 + 4])[0] == a[1, 0, 0, 0]


def test_scaled_integer_data_reads_as_float(tmp_path):
    a = np.arange(24, dtype=np.int16).reshape(2, 3, 4)
    p = str(tmp_path / "i.nii")
    nifti.write(p, a)
    raw = bytearray(open(p, "rb").read())
    struct.pack_into("<2f", raw, 112, 0.5, 3.0)  # scl_slope, scl_inter
    open(p, "wb").write(bytes(raw))
    b, _ = nifti.read(p)
    assert np.allclose(b, a * 0.5 + 3.0)


def test_mask_order_is_x_fastest_and_inverts():
    mask = np.zeros((4, 3, 2))
    mask[1, 0, 0] = mask[3, 2, 1] = mask[0, 1, 0] = 1
    idx = nifti.mask_indices(mask)
    assert list(idx) == [1, 4, 3 + 4 * 2 + 12]  # (1,0,0), (0,1,0), (3,2,1) in x-fastest order
    vol = np.random.default_rng(1).normal(size=(4, 3, 2, 5)).astype(np.float32)
    m = nifti.to_matrix(vol, mask)
    assert m.shape == (3, 5) and np.array_equal(m[0], vol[1, 0, 0]) and np.array_equal(m[2], vol[3, 2, 1])
    back = nifti.from_matrix(m, mask)
    assert np.array_equal(back[mask != 0], vol[mask != 0]) and np.all(back[mask == 0] == 0)


def test_part_files_join_like_merge_parts(tmp_path):
    opts = Options.make(model=2, nfibres=2, rician=1, f0=1, njumps=30, sampleevery=10)
    n, ns, K = 101, 3, 2
    rng = np.random.default_rng(2)
    out = {k: rng.normal(size=(K, ns, n)).astype(np.float32) for k in ("th", "ph", "f")}
    for k in ("mean_d", "mean_dstd", "mean_f0", "mean_tau", "mean_S0"):
        out[k] = rng.normal(size=n).astype(np.float32)
    bedpostx.write_parts(str(tmp_path), out, opts, 4)
    f = tmp_path / "diff_parts" / "data_part_0003" / "f2samplesJ"
    assert os.path.getsize(f) == ns * (n - 3 * (n // 4)) * 8  # the last part takes the remainder
    j = bedpostx.join_parts(str(tmp_path), "f2samples", n, ns, 4)
    assert j.shape == (ns, n) and np.array_equal(j, out["f"][1].astype(np.float64))
    m = bedpostx.join_parts(str(tmp_path), "mean_tausamples", n, 1, 4)
    assert np.array_equal(m[0], out["mean_tau"].astype(np.float64))
    names = [x[1] for x in bedpostx.joined_names(opts)]
    assert "mean_d_stdsamples" in names and "mean_f0samples" in names and "merged_ph2samples" in names
    assert "mean_Rsamples" not in names
