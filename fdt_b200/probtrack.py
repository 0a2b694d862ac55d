"""probtrackx on a bedpostx directory, on the GPU (bpx_probtrack_dev): simple and seedmask modes.

    python -m fdt_b200.probtrack SUBJECT.bedpostX --seeds SEEDS --out OUTDIR [-o fdt_paths] [-P 5000]
        [-S 2000] [--steplength 0.5] [--cthr 0.2] [--fibthresh 0.01] [--distthresh 0] [--randfib 0]
        [--fibst 1] [--usef] [--sampvox] [--pd] [-l] [--modeuler] [--seed N] [--avoid MASK]
        [--stop MASK] [--waypoints MASK|LIST] [--targetmasks LIST --os2t] [--omatrix2 --lrmask MASK]
        [--omatrix1] [--prefdir VOL4D] [--network] [--mask2 MASK]

Reads merged_th{k}samples, merged_ph{k}samples, merged_f{k}samples and nodif_brain_mask (NIfTI-1)
as probtrackx does (probtrackx.cc:25-96, tractvolsx.h:55-97) and tracks from the seeds:
  * SEEDS a text file of points (one per row, voxel coordinates x y z): simple mode
    (ptx_simple.cc:16-70, as run with --opd): one path distribution per point,
    OUTDIR/<out>_<x>_<y>_<z>.nii.gz, counts reset between points;
  * SEEDS a NIfTI mask on the diffusion grid: seedmask mode (ptx_seedmask.cc): every voxel with a
    non-zero value is a seed point, in z, y, x order, and OUTDIR/<out>.nii.gz sums them all.
  * --network with SEEDS a text file naming several masks: network mode (ptx_nmasks.cc): each
    mask's voxels are seeds in turn, keeping only streamlines that reach the union of the other
    masks (one extra waypoint mask); OUTDIR/<out>.nii.gz sums all, waytotal has one line per mask;
  * SEEDS a mask and --mask2 a second one: twomasks mode (ptx_twomasks.cc), the same with two.
OUTDIR/waytotal holds the number of kept streamlines over all seeds (Counter::save_total).
--targetmasks LIST --os2t (a text file naming up to 32 masks one per line) adds
OUTDIR/seeds_to_<mask>.nii.gz: at every seed voxel, the kept streamlines from it that enter the
mask (Counter::update_seedcounts, save_seedcounts; streamlines.cc:700-748, 900-930).
--omatrix2 --lrmask MASK (a mask on a tract-space grid of its own voxel size, in line with the
diffusion grid) adds OUTDIR/fdt_matrix2.nii.gz, seeds x tract-space voxels: for every seed, the
kept streamlines from it through each voxel of the mask, and its coordinate and lookup files
(Counter::initialise_matrix2, update_matrix2_row, save_matrix2; streamlines.cc:515-560, 772-808,
970-980).
--omatrix1 (seedmask mode) adds OUTDIR/fdt_matrix1.nii.gz, seeds x seeds: for every seed, the kept
streamlines from it through each seed voxel (its path distribution read at the seed mask), and
coords_for_fdt_matrix1 (Counter::initialise_matrix1, update_matrix1, save_matrix1;
streamlines.cc:493-510, 751-770, 963-968).  The reference clears its path distribution after each
seed when it builds matrix1, so its fdt_paths comes out empty then; here fdt_paths keeps the sum.
--prefdir VOL4D (x, y, z components per voxel) makes every step after a streamline's first take the
fibre closest to the voxel's preferred direction, where it is non-zero (streamlines.cc:286-291,
tractvolsx.h:209-225).
--avoid rejects a half that enters the mask, --stop ends a half where it enters it, and --waypoints
(one mask, or a text file naming up to 32 masks one per line) keeps only streamlines whose halves
together passed every mask (streamlines.cc:112-145, 279-330); all on the diffusion grid.
The seed coordinates are taken in the volume's voxel grid as stored (the reference converts NIfTI
voxel coordinates to its internal convention, which is the identity for neurological storage).
"""
from __future__ import annotations

import argparse
import glob
import os

import numpy as np

from . import lib, nifti
from .abi import TrackOptions


def read_samples(bpx_dir: str):
    """(th, ph, f [K][nsamples][nz][ny][nx] float32, mask [nz][ny][nx], header, voxel size)."""
    mask, hdr = nifti.read(os.path.join(bpx_dir, "nodif_brain_mask.nii.gz"))
    K = len(glob.glob(os.path.join(bpx_dir, "merged_th*samples.nii.gz")))
    if K == 0:
        raise FileNotFoundError(f"{bpx_dir}: no merged_th1samples")
    vols = {}
    for q in ("th", "ph", "f"):
        arr = []
        for k in range(1, K + 1):
            a, _ = nifti.read(os.path.join(bpx_dir, f"merged_{q}{k}samples.nii.gz"))
            if a.ndim == 3:
                a = a[..., None]
            if a.shape[:3] != mask.shape[:3]:
                raise ValueError(f"merged_{q}{k}samples: grid {a.shape[:3]} differs from the mask's {mask.shape[:3]}")
            arr.append(np.transpose(np.asarray(a, np.float32), (3, 2, 1, 0)))  # [ns][z][y][x]
        vols[q] = np.ascontiguousarray(np.stack(arr))
    m = np.ascontiguousarray(np.transpose(np.asarray(mask, np.float32).reshape(mask.shape[:3]), (2, 1, 0)))
    vs = tuple(float(x) for x in hdr.pixdim[1:4])
    return vols["th"], vols["ph"], vols["f"], m, hdr, vs


def read_mask(path: str, grid: tuple[int, int, int]) -> np.ndarray:
    """A mask on the diffusion grid as float32 [nz][ny][nx]."""
    a, _ = nifti.read(path)
    if a.shape[:3] != grid:
        raise ValueError(f"{path}: grid {a.shape[:3]} differs from the mask's {grid}")
    return np.ascontiguousarray(np.transpose(np.asarray(a, np.float32).reshape(grid), (2, 1, 0)))


def waypoint_files(arg: str) -> list[str]:
    """--waypoints: one image, or a text file naming one image per line (probtrackx's read_masks)."""
    if arg.endswith((".nii", ".nii.gz")):
        return [arg]
    base = os.path.dirname(os.path.abspath(arg))
    names = [ln.strip() for ln in open(arg) if ln.strip()]
    return [n if os.path.isabs(n) else os.path.join(base, n) for n in names]


def read_prefdir(path: str, grid: tuple[int, int, int]) -> np.ndarray:
    """--prefdir: a 4D NIfTI [x][y][z][3] of preferred directions on the diffusion grid, as float32
    [3][nz][ny][nx] (read_volume4D of streamlines.cc:124-125)."""
    a, _ = nifti.read(path)
    if a.ndim != 4 or a.shape[:3] != grid or a.shape[3] != 3:
        raise ValueError(f"{path}: expected a 4D volume of 3 components on the grid {grid}, got {a.shape}")
    return np.ascontiguousarray(np.transpose(np.asarray(a, np.float32), (3, 2, 1, 0)))


def seed_points(arg: str, grid: tuple[int, int, int]) -> tuple[np.ndarray, bool]:
    """(seed points [n][3] as voxel x y z, per_seed): a text file of points (simple mode, one
    output per point) or a NIfTI mask whose non-zero voxels, in z, y, x order, are the seeds
    (seedmask mode, one output over all)."""
    if arg.endswith((".nii", ".nii.gz")):
        m = read_mask(arg, grid)  # [z][y][x]
        zyx = np.argwhere(np.abs(m) > 0)
        return np.ascontiguousarray(zyx[:, ::-1].astype(np.float32)), False
    pts = np.loadtxt(arg, ndmin=2)
    if pts.shape[1] != 3 and pts.shape[0] == 3:
        pts = pts.T
    return np.ascontiguousarray(pts, np.float32), True


def run(bpx_dir: str, seeds, opts: TrackOptions, outdir: str, avoid: str | None = None,
        stop: str | None = None, waypoints: str | None = None, outname: str = "fdt_paths",
        targets: str | None = None, lrmask: str | None = None, omatrix1: bool = False,
        prefdir: str | None = None) -> tuple[np.ndarray, int]:
    """Tracks from `seeds` (a seed file or mask path, or an array of points for simple mode) and
    writes the path distributions and waytotal; returns (paths [x][y][z], or [nseeds][x][y][z] in
    simple mode, waytotal)."""
    import torch

    th, ph, f, m, hdr, vs = read_samples(bpx_dir)
    grid = m.shape[::-1]
    seeds_arg = seeds
    if isinstance(seeds, str):
        seeds, per_seed = seed_points(seeds, grid)
    else:
        seeds, per_seed = np.ascontiguousarray(seeds, np.float32).reshape(-1, 3), True
    opts.per_seed = int(per_seed)
    dev = [lib.to_device(a) for a in (th, ph, f, m)]
    extra = {}
    if avoid:
        extra["avoid"] = lib.to_device(read_mask(avoid, grid))
    if stop:
        extra["stop"] = lib.to_device(read_mask(stop, grid))
    if waypoints:
        extra["waypoints"] = [read_mask(w, grid) for w in waypoint_files(waypoints)]
    target_files = waypoint_files(targets) if targets else []
    if target_files:
        extra["targets"] = [read_mask(t, grid) for t in target_files]
    if lrmask:
        lr, lr_hdr = nifti.read(lrmask)
        lr_zyx = np.ascontiguousarray(np.transpose(np.asarray(lr, np.float32).reshape(lr.shape[:3]), (2, 1, 0)))
        extra["matrix2"] = (lr_zyx, tuple(float(x) for x in lr_hdr.pixdim[1:4]))
    if prefdir:
        extra["prefdir"] = read_prefdir(prefdir, grid)
    if omatrix1:
        if per_seed or not isinstance(seeds_arg, str):
            raise ValueError("--omatrix1 needs a seed mask (seedmask mode)")
        # the columns: the seed voxels, in the order seed_points gives the seeds (z, y, x)
        extra["matrix1"] = (np.abs(read_mask(seeds_arg, grid)) > 0).astype(np.float32)
    res = lib.probtrack(opts, *dev, seeds, voxel_size=vs, **extra)
    paths, way = res[0], res[1]
    torch.cuda.synchronize()
    os.makedirs(outdir, exist_ok=True)

    def save(vol_zyx: np.ndarray, name: str) -> np.ndarray:
        vol = np.transpose(vol_zyx, (2, 1, 0))  # back to [x][y][z]
        # an int32 volume, as the reference saves its volume<int> m_prob
        nifti.write(os.path.join(outdir, name + ".nii.gz"), vol.astype(np.int32), like=hdr,
                    cal=(float(vol.min()), float(vol.max())))
        return vol

    p = paths.cpu().numpy()
    if per_seed:
        # Counter::save_pathdist(add): the basename, then _x_y_z as the seed file gives them
        vols = np.stack([save(p[i], f"{outname}_{x:g}_{y:g}_{z:g}") for i, (x, y, z) in enumerate(seeds)])
    else:
        vols = save(p, outname)
    with open(os.path.join(outdir, "waytotal"), "w") as fh:
        fh.write(f"{way}\n")
    if target_files:
        # seeds_to_<target>: each seed's count at its (rounded) voxel, float as the reference saves it
        s2t = res[2]
        idx = np.floor(seeds + 0.5).astype(np.int64)
        inside = np.all((idx >= 0) & (idx < np.array(grid)), axis=1)
        for t, name in enumerate(target_files):
            vol = np.zeros(grid, np.float32)
            vol[idx[inside, 0], idx[inside, 1], idx[inside, 2]] = s2t[t][inside]
            stem = os.path.basename(name)
            for ext in (".nii.gz", ".nii"):
                if stem.endswith(ext):
                    stem = stem[: -len(ext)]
            nifti.write(os.path.join(outdir, f"seeds_to_{stem}.nii.gz"), vol, like=hdr,
                        cal=(0.0, float(opts.nparticles)))
    if lrmask:
        save_matrix2(outdir, res[2 + bool(target_files)], seeds, lr_zyx, lr_hdr)
    if omatrix1:
        save_matrix1(outdir, res[-1], seeds)
    return vols, way


def save_matrix1(outdir: str, m1: np.ndarray, seeds: np.ndarray) -> None:
    """Counter::save_matrix1 (streamlines.cc:963-968): fdt_matrix1 (seeds along x, seed-voxel columns
    along y, int32 as the reference's volume<int>) and coords_for_fdt_matrix1 (each seed's voxel
    x y z)."""
    m1 = np.asarray(m1, np.int32)
    nifti.write(os.path.join(outdir, "fdt_matrix1.nii.gz"), m1[:, :, None], cal=(0.0, float(m1.max(initial=0))))
    seed_vox = np.floor(np.asarray(seeds, np.float64) + 0.5).astype(np.int32)
    nifti.write(os.path.join(outdir, "coords_for_fdt_matrix1.nii.gz"), seed_vox[:, :, None])


def save_matrix2(outdir: str, m2: np.ndarray, seeds: np.ndarray, lr_zyx: np.ndarray, lr_hdr) -> None:
    """Counter::save_matrix2 (streamlines.cc:970-980): fdt_matrix2 (seeds along x, tract-space
    columns along y), coords_for_fdt_matrix2 (each seed's voxel x y z), tract_space_coords_for_fdt_matrix2
    (each column's tract-space voxel), lookup_tractspace_fdt_matrix2 (each tract-space voxel's
    column, 0 outside the mask); int32 as the reference's volume<int>."""
    m2 = np.asarray(m2, np.int32)
    nifti.write(os.path.join(outdir, "fdt_matrix2.nii.gz"), m2[:, :, None], cal=(0.0, float(m2.max(initial=0))))
    seed_vox = np.floor(np.asarray(seeds, np.float64) + 0.5).astype(np.int32)
    nifti.write(os.path.join(outdir, "coords_for_fdt_matrix2.nii.gz"), seed_vox[:, :, None])
    inside = lr_zyx != 0
    tract = np.ascontiguousarray(np.argwhere(inside)[:, ::-1].astype(np.int32))  # z, y, x order -> x y z
    nifti.write(os.path.join(outdir, "tract_space_coords_for_fdt_matrix2.nii.gz"), tract[:, :, None])
    lut = np.maximum(lib.matrix2_lookup(lr_zyx), 0)
    nifti.write(os.path.join(outdir, "lookup_tractspace_fdt_matrix2.nii.gz"), np.transpose(lut, (2, 1, 0)),
                like=lr_hdr, cal=(0.0, float(lut.max(initial=0))))


def run_network(bpx_dir: str, mask_list, opts: TrackOptions, outdir: str, avoid: str | None = None,
                stop: str | None = None, waypoints: str | None = None,
                outname: str = "fdt_paths", prefdir: str | None = None) -> tuple[np.ndarray, list[int]]:
    """Network mode (ptx_nmasks.cc; with two masks, twomasks mode, ptx_twomasks.cc): for each mask
    of the list (a text file naming them, or a list of paths), its voxels (z, y, x order) are the
    seeds and the union of the other masks is one more waypoint mask (Streamliner::add_waymask);
    the path counts of all masks add into one volume and waytotal has one entry per mask."""
    import torch

    th, ph, f, m, hdr, vs = read_samples(bpx_dir)
    grid = m.shape[::-1]
    names = waypoint_files(mask_list) if isinstance(mask_list, str) else list(mask_list)
    masks = [np.abs(read_mask(n, grid)) > 0 for n in names]
    if len(masks) < 2:
        raise ValueError("network mode needs at least two masks")
    dev = [lib.to_device(a) for a in (th, ph, f, m)]
    extra = {}
    if avoid:
        extra["avoid"] = lib.to_device(read_mask(avoid, grid))
    if stop:
        extra["stop"] = lib.to_device(read_mask(stop, grid))
    if prefdir:
        extra["prefdir"] = read_prefdir(prefdir, grid)
    user_ways = [read_mask(w, grid) for w in waypoint_files(waypoints)] if waypoints else []
    if len(user_ways) > 31:
        raise ValueError("network mode takes at most 31 waypoint masks of its own")
    opts.per_seed = 0
    total = np.zeros(m.shape, np.int64)
    ways = []
    for i, mi in enumerate(masks):
        others = np.zeros(m.shape, bool)
        for j, mj in enumerate(masks):
            if j != i:
                others |= mj
        seeds = np.ascontiguousarray(np.argwhere(mi)[:, ::-1].astype(np.float32))
        paths, way = lib.probtrack(opts, *dev, seeds, voxel_size=vs, waypoints=user_ways + [others.astype(np.float32)],
                                   **extra)
        torch.cuda.synchronize()
        total += paths.cpu().numpy()
        ways.append(way)
    os.makedirs(outdir, exist_ok=True)
    vol = np.transpose(total.astype(np.int32), (2, 1, 0))
    nifti.write(os.path.join(outdir, outname + ".nii.gz"), vol, like=hdr, cal=(float(vol.min()), float(vol.max())))
    with open(os.path.join(outdir, "waytotal"), "w") as fh:
        fh.write("".join(f"{w}\n" for w in ways))
    return vol, ways


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("bpx_dir")
    ap.add_argument("--seeds", required=True,
                    help="text file of seed points (voxel x y z per row: simple mode) or a seed mask (seedmask mode)")
    ap.add_argument("--out", required=True, help="output directory")
    ap.add_argument("-o", "--outname", default="fdt_paths", help="basename of the path distributions")
    ap.add_argument("-P", "--nsamples", type=int, default=5000)
    ap.add_argument("-S", "--nsteps", type=int, default=2000)
    ap.add_argument("--steplength", type=float, default=0.5)
    ap.add_argument("-c", "--cthr", type=float, default=0.2)
    ap.add_argument("--fibthresh", type=float, default=0.01)
    ap.add_argument("--distthresh", type=float, default=0.0)
    ap.add_argument("--randfib", type=int, default=0)
    ap.add_argument("--fibst", type=int, default=1)
    ap.add_argument("-f", "--usef", action="store_true")
    ap.add_argument("--sampvox", action="store_true")
    ap.add_argument("--pd", action="store_true", help="correct the path distribution for the length of the pathways")
    ap.add_argument("-l", "--loopcheck", action="store_true", help="perform loopchecks on paths")
    ap.add_argument("--modeuler", action="store_true", help="use modified Euler streamlining")
    ap.add_argument("--seed", type=int, default=8665904)
    ap.add_argument("--avoid", help="reject pathways passing through this mask")
    ap.add_argument("--stop", help="stop tracking at locations given by this mask")
    ap.add_argument("--waypoints", help="waypoint mask, or a text file listing waypoint masks")
    ap.add_argument("--targetmasks", help="text file listing target masks (seeds_to_targets)")
    ap.add_argument("--os2t", action="store_true", help="output seeds_to_targets")
    ap.add_argument("--omatrix2", action="store_true", help="output matrix2 (seeds x tract-space voxels)")
    ap.add_argument("--lrmask", help="tract-space (low resolution) mask for matrix2")
    ap.add_argument("--omatrix1", action="store_true", help="output matrix1 (seeds x seed voxels; seedmask mode)")
    ap.add_argument("--prefdir", help="4D volume of preferred directions (x, y, z) on the diffusion grid")
    ap.add_argument("--network", action="store_true", help="network mode: --seeds lists several masks")
    ap.add_argument("--mask2", help="second seed mask (twomasks mode, with a seed mask)")
    a = ap.parse_args(argv)
    o = TrackOptions.make(nparticles=a.nsamples, nsteps=a.nsteps, steplength=a.steplength, c_thr=a.cthr,
                          fibthresh=a.fibthresh, distthresh=a.distthresh, randfib=a.randfib, fibst=a.fibst,
                          usef=int(a.usef), sampvox=int(a.sampvox), pathdist=int(a.pd), loopcheck=int(a.loopcheck),
                          modeuler=int(a.modeuler), seed=a.seed)
    if a.os2t and not a.targetmasks:
        ap.error("--os2t needs --targetmasks")
    if a.omatrix2 and not a.lrmask:
        ap.error("--omatrix2 needs --lrmask")
    if a.network or a.mask2:
        if a.os2t or a.omatrix2 or a.omatrix1:
            ap.error("seeds_to_targets, matrix1 and matrix2 are not available in multiple seed tractography")
        masks = [a.seeds, a.mask2] if a.mask2 else a.seeds
        _, ways = run_network(a.bpx_dir, masks, o, a.out, avoid=a.avoid, stop=a.stop, waypoints=a.waypoints,
                              outname=a.outname, prefdir=a.prefdir)
        print("waytotal " + " ".join(map(str, ways)))
        return
    if a.omatrix1 and not a.seeds.endswith((".nii", ".nii.gz")):
        ap.error("--omatrix1 needs a seed mask (seedmask mode)")
    _, way = run(a.bpx_dir, a.seeds, o, a.out, avoid=a.avoid, stop=a.stop, waypoints=a.waypoints, outname=a.outname,
                 targets=a.targetmasks if a.os2t else None, lrmask=a.lrmask if a.omatrix2 else None,
                 omatrix1=a.omatrix1, prefdir=a.prefdir)
    print(f"waytotal {way}")


if __name__ == "__main__":
    main()
