"""bedpostx on one subject directory with libbpx.so: the host driver around the GPU path.

    python -m fdt_b200.bedpostx SUBJDIR [--nf 3] [--model 2] [--rician] [--f0] [--ardf0] ...

Reads SUBJDIR/{data, nodif_brain_mask}.nii.gz, bvecs and bvals (the inputs bedpostx_gpu reads;
grad_dev with --gradnonlin),
runs the per-voxel path on the GPU (LM-initialised, or --learned WEIGHTS for the learned start),
the bedpostx_postproc arithmetic on the GPU, and writes into SUBJDIR.bedpostX/ the files
merge_parts_gpu and bedpostx_postproc_gpu.sh produce:

  merged_{th,ph,f}{k}samples, mean_{th,ph,f}{k}samples, mean_dsamples, mean_d_stdsamples (model >= 2),
  mean_Rsamples (model 3), mean_f0samples (--f0), mean_tausamples (--rician), mean_S0samples,
  dyads{k}, dyads{k}_dispersion, dyads{k}_thr0.05 and dyads{k}_thr0.05_modf{k} (k >= 2),
  mean_fsumsamples, nodif_brain_mask.

--parts P additionally writes the reference's part files (diff_parts/data_part_XXXX/<name>J:
raw float64 [nsamples][voxels of the part], Samples::save / join_Parts layout,
CUDA/samples.cu:231-260, merge_parts_gpu.cc:17-82), and `merge` rebuilds the merged volumes from
such part files the way merge_parts_gpu does.
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from . import nifti
from .abi import Options

# (part-file name, output name, display max, display min) as merge_parts_gpu.cc:123-160 joins them;
# -10 means the data's own maximum / minimum
def joined_names(opts: Options) -> list[tuple[str, str, float, float]]:
    n = [("mean_dsamples", "mean_dsamples", -10, 0)]
    if opts.model >= 2:
        n.append(("mean_d_stdsamples", "mean_d_stdsamples", -10, 0))
        if opts.model == 3:
            n.append(("mean_Rsamples", "mean_Rsamples", 1, 0))
    if opts.f0:
        n.append(("mean_f0samples", "mean_f0samples", 1, 0))
    if opts.rician:
        n.append(("mean_tausamples", "mean_tausamples", -10, 0))
    n.append(("mean_S0samples", "mean_S0samples", -10, 0))
    for k in range(1, opts.nfibres + 1):
        n += [(f"th{k}samples", f"merged_th{k}samples", -10, -10), (f"ph{k}samples", f"merged_ph{k}samples", -10, -10),
              (f"f{k}samples", f"merged_f{k}samples", 1, 0)]
    return n


MEAN_KEYS = {"mean_dsamples": "mean_d", "mean_d_stdsamples": "mean_dstd", "mean_Rsamples": "mean_R",
             "mean_f0samples": "mean_f0", "mean_tausamples": "mean_tau", "mean_S0samples": "mean_S0"}


def part_rows(outputs: dict, name: str) -> np.ndarray:
    """[nt][nvox] rows of one part file from host outputs (nt = nsamples or 1)."""
    if name in MEAN_KEYS:
        return np.asarray(outputs[MEAN_KEYS[name]])[None, :]
    for key in ("th", "ph", "f"):
        if name.startswith(key) and name.endswith("samples") and name[len(key) : -len("samples")].isdigit():
            return np.asarray(outputs[key])[int(name[len(key) : -len("samples")]) - 1]
    raise KeyError(name)


def read_text_matrix(path: str) -> np.ndarray:
    return np.atleast_2d(np.loadtxt(path, dtype=np.float64))


def read_subject(subjdir: str):
    """(data [nvox][M] float32, mask, header of data, bvecs [3][M], bvals [M])."""
    def find(base):
        for ext in (".nii.gz", ".nii"):
            if os.path.exists(os.path.join(subjdir, base + ext)):
                return os.path.join(subjdir, base + ext)
        raise FileNotFoundError(os.path.join(subjdir, base + ".nii.gz"))

    data4, hdr = nifti.read(find("data"))
    mask, _ = nifti.read(find("nodif_brain_mask"))
    if mask.shape != data4.shape[:3]:
        raise ValueError("mask and data have different spatial shapes")
    bvecs = read_text_matrix(os.path.join(subjdir, "bvecs"))
    bvals = read_text_matrix(os.path.join(subjdir, "bvals"))
    M = data4.shape[3]
    if bvecs.shape == (M, 3):
        bvecs = bvecs.T
    bvals = bvals.reshape(-1)
    if bvecs.shape != (3, M) or bvals.size != M:
        raise ValueError(f"bvecs/bvals do not match the {M} volumes of data")
    y = nifti.to_matrix(data4, mask).astype(np.float32)
    return y, mask, hdr, bvecs.astype(np.float32), bvals.astype(np.float32)


def read_grad_dev(subjdir: str, mask: np.ndarray) -> np.ndarray:
    """grad_dev (X x Y x Z x 9, the gradient-nonlinearity tensor per voxel) at the mask's voxels:
    [nvox][9], the rows split_parts_gpu takes with grad.matrix(mask) (CUDA/split_parts_gpu.cc:114-120)."""
    for ext in (".nii.gz", ".nii"):
        p = os.path.join(subjdir, "grad_dev" + ext)
        if os.path.exists(p):
            g, _ = nifti.read(p)
            if g.shape[:3] != mask.shape or g.ndim != 4 or g.shape[3] != 9:
                raise ValueError("grad_dev must be X x Y x Z x 9 over the mask's grid")
            return nifti.to_matrix(g, mask).astype(np.float32)
    raise FileNotFoundError(os.path.join(subjdir, "grad_dev.nii.gz"))


def write_parts(outdir: str, outputs: dict, opts: Options, nparts: int) -> None:
    """The reference's part files: diff_parts/data_part_XXXX/<name>J, float64 [nt][part voxels]."""
    nvox = int(np.asarray(outputs["mean_d"]).shape[0])
    size = nvox // nparts
    for p in range(nparts):
        lo = p * size
        hi = nvox if p == nparts - 1 else lo + size
        d = os.path.join(outdir, "diff_parts", f"data_part_{p:04d}")
        os.makedirs(d, exist_ok=True)
        for name, _, _, _ in joined_names(opts):
            rows = part_rows(outputs, name)[:, lo:hi].astype(np.float64)
            rows.tofile(os.path.join(d, name + "J"))


def join_parts(outdir: str, name: str, nvox: int, nt: int, nparts: int) -> np.ndarray:
    """merge_parts_gpu.cc:17-82 join_Parts: [nt][nvox] from the parts' <name>J files."""
    size = nvox // nparts
    cols = []
    for p in range(nparts):
        n = nvox - (nparts - 1) * size if p == nparts - 1 else size
        f = os.path.join(outdir, "diff_parts", f"data_part_{p:04d}", name + "J")
        a = np.fromfile(f, dtype=np.float64, count=n * nt)
        if a.size != n * nt:
            raise ValueError(f"{f}: expected {n * nt} values, found {a.size}")
        cols.append(a.reshape(nt, n))
    return np.concatenate(cols, axis=1)


def _display(arr: np.ndarray, mx: float, mn: float) -> tuple[float, float]:
    a = np.asarray(arr)
    return (float(a.min()) if mn == -10 else mn, float(a.max()) if mx == -10 else mx)


def write_merged(outdir: str, rows_of, opts: Options, mask: np.ndarray, hdr: nifti.Header) -> None:
    """The merged_* and mean_* volumes (merge_parts_gpu's outputs) from rows_of(name) -> [nt][nvox]."""
    for name, out, mx, mn in joined_names(opts):
        rows = np.asarray(rows_of(name), dtype=np.float32)
        vol = nifti.from_matrix(rows.T if rows.shape[0] > 1 else rows[0], mask)
        nifti.write(os.path.join(outdir, out + ".nii.gz"), vol, like=hdr, cal=_display(vol, mx, mn))


def write_postproc(outdir: str, outputs: dict, post: dict, opts: Options, mask: np.ndarray, hdr: nifti.Header) -> None:
    """bedpostx_postproc_gpu.sh outputs from the GPU post-processing arrays."""
    K = opts.nfibres
    for k in range(K):
        kk = k + 1
        for key, name in (("mean_th", f"mean_th{kk}samples"), ("mean_ph", f"mean_ph{kk}samples")):
            v = nifti.from_matrix(np.asarray(post[key])[k], mask)
            nifti.write(os.path.join(outdir, name + ".nii.gz"), v, like=hdr, cal=_display(v, -10, -10))
        v = nifti.from_matrix(np.asarray(outputs["mean_f"])[k], mask)
        nifti.write(os.path.join(outdir, f"mean_f{kk}samples.nii.gz"), v, like=hdr, cal=(0.0, 1.0))
        dy = nifti.from_matrix(np.asarray(outputs["dyads"])[k].T, mask)
        nifti.write(os.path.join(outdir, f"dyads{kk}.nii.gz"), dy, like=hdr, cal=(-1.0, 1.0))
        v = nifti.from_matrix(np.asarray(post["dispersion"])[k], mask)
        nifti.write(os.path.join(outdir, f"dyads{kk}_dispersion.nii.gz"), v, like=hdr, cal=(0.0, 1.0))
        if kk >= 2:
            t = nifti.from_matrix(np.asarray(post["dyads_thr"])[k].T, mask)
            nifti.write(os.path.join(outdir, f"dyads{kk}_thr0.05.nii.gz"), t, like=hdr, cal=(-1.0, 1.0))
            m = nifti.from_matrix(np.asarray(post["dyads_modf"])[k].T, mask)
            nifti.write(os.path.join(outdir, f"dyads{kk}_thr0.05_modf{kk}.nii.gz"), m, like=hdr)
    v = nifti.from_matrix(np.asarray(post["mean_fsum"]), mask)
    nifti.write(os.path.join(outdir, "mean_fsumsamples.nii.gz"), v, like=hdr)
    nifti.write(os.path.join(outdir, "nodif_brain_mask.nii.gz"), (np.asarray(mask) != 0).astype(np.float32), like=hdr)


def run(subjdir: str, opts: Options, learned_weights: str | None = None, nparts: int = 0,
        outdir: str | None = None, freeze: int = 0) -> dict:
    """The whole subject on the current GPU; returns host copies of the outputs."""
    import torch

    from . import learned, lib

    t0 = time.time()
    y, mask, hdr, bvecs, bvals = read_subject(subjdir)
    outdir = outdir or subjdir.rstrip("/") + ".bedpostX"
    os.makedirs(outdir, exist_ok=True)
    d = lib.to_device(y)
    bv, bl = lib.to_device(bvecs), lib.to_device(bvals)
    if opts.gradnonlin:  # per-voxel corrected b-matrix on the device (correct_bvals_bvecs)
        bv, bl = lib.gradnonlin(lib.to_device(read_grad_dev(subjdir, mask)), bv, bl)
    if learned_weights:
        params, meta = learned.load_weights(learned_weights)
        if int(meta["ndir"]) != y.shape[1]:
            raise SystemExit(f"{learned_weights} was trained for {int(meta['ndir'])} measurements, data have {y.shape[1]}")
        out = learned.xfibres_learned(opts, d, bv, bl, params, freeze=freeze)
    else:
        out = lib.xfibres_dev(opts, d, bv, bl)
    post = lib.postproc(opts, out, 0.05)
    torch.cuda.synchronize()
    t_gpu = time.time() - t0
    host = {k: v.cpu().numpy() for k, v in out.items()}
    posth = {k: v.cpu().numpy() for k, v in post.items()}
    write_merged(outdir, lambda name: part_rows(host, name), opts, mask, hdr)
    write_postproc(outdir, host, posth, opts, mask, hdr)
    if nparts > 0:
        write_parts(outdir, host, opts, nparts)
    print(f"{y.shape[0]} voxels, {y.shape[1]} measurements: GPU path {t_gpu:.1f} s; outputs in {outdir}")
    return host


def merge(subjdir: str, opts: Options, nparts: int, outdir: str | None = None) -> None:
    """merge_parts_gpu: the merged_* / mean_* volumes from part files."""
    outdir = outdir or subjdir.rstrip("/") + ".bedpostX"
    _, mask, hdr, _, _ = read_subject(subjdir)
    nvox = int((np.asarray(mask) != 0).sum())
    ns = opts.nsamples

    def rows_of(name):
        return join_parts(outdir, name, nvox, 1 if name.startswith("mean_") else ns, nparts)

    write_merged(outdir, rows_of, opts, mask, hdr)


def options_from_args(a) -> Options:
    return Options.make(model=a.model, nfibres=a.nf, fudge=a.fudge, njumps=a.nj, nburn=a.bi, sampleevery=a.se,
                        updateproposalevery=a.upe, no_ard=int(a.noard), all_ard=int(a.allard), nonlin=int(a.nonlinear),
                        cnonlin=int(not a.nonlinear), rician=int(a.rician), f0=int(a.f0), ardf0=int(a.ardf0),
                        gradnonlin=int(a.gradnonlin), seed=a.seed)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("subjdir")
    ap.add_argument("command", nargs="?", default="run", choices=["run", "merge"])
    ap.add_argument("--nf", type=int, default=3, help="number of fibres per voxel")
    ap.add_argument("--model", type=int, default=2, choices=[1, 2, 3])
    ap.add_argument("--fudge", type=float, default=1.0, help="ARD weight")
    ap.add_argument("--nj", type=int, default=1250, help="jumps")
    ap.add_argument("--bi", type=int, default=1000, help="burn-in")
    ap.add_argument("--se", type=int, default=25, help="sample every")
    ap.add_argument("--upe", type=int, default=40, help="update proposal every")
    ap.add_argument("--seed", type=int, default=8665904)
    ap.add_argument("--noard", action="store_true")
    ap.add_argument("--allard", action="store_true")
    ap.add_argument("--nonlinear", action="store_true", help="PVM_single start instead of PVM_single_c")
    ap.add_argument("--rician", action="store_true")
    ap.add_argument("--f0", action="store_true")
    ap.add_argument("--ardf0", action="store_true")
    ap.add_argument("--gradnonlin", action="store_true", help="per-voxel b-matrix from SUBJDIR/grad_dev")
    ap.add_argument("--learned", default=None, help="initialiser weights: learned start (use --bi 200)")
    ap.add_argument("--freeze", type=int, default=0, choices=[0, 1, 2])
    ap.add_argument("--parts", type=int, default=0, help="also write (run) or read (merge) this many part files")
    a = ap.parse_args(argv)
    opts = options_from_args(a)
    if a.command == "merge":
        if a.parts < 1:
            raise SystemExit("merge needs --parts")
        merge(a.subjdir, opts, a.parts)
    else:
        run(a.subjdir, opts, a.learned, a.parts, freeze=a.freeze)


if __name__ == "__main__":
    main()
