"""probtrackx simple mode on the GPU (bpx_probtrack_dev) against the CPU oracle, exactly.

Both draw every step's random numbers from the same counter-based stream and do the same
single-precision operations in the same order, so fdt_paths and waytotal must be identical, bit for
bit (integer counts), for every option the kernel takes: the first fibre chosen by --fibst or at
random (--randfib 1/2/3), --usef, --sampvox, --distthresh (the two-pass halves), the avoid, stop
and waypoint masks, --pd, --modeuler, --loopcheck (also on circling tracts, where it acts), short
and long step counts, and on the outputs of this library's own bedpostx run.
"""
import numpy as np
import pytest

from fdt_b200 import synth
from fdt_b200.abi import Options, TrackOptions
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


CASES = [
    ("default", dict()),
    ("randfib1", dict(randfib=1)),
    ("randfib2", dict(randfib=2)),
    ("randfib3", dict(randfib=3)),
    ("usef", dict(usef=1)),
    ("sampvox_fibst2", dict(sampvox=1, fibst=2)),
    ("distthresh", dict(distthresh=6.0)),
    ("short_steps_low_cthr", dict(nsteps=20, c_thr=0.0)),
    ("steplength_1mm", dict(steplength=1.0)),
    ("avoid", dict(masks=("avoid",))),
    ("stop", dict(masks=("stop",))),
    ("waypoints", dict(masks=("waypoints",))),
    ("all_masks_distthresh", dict(masks=("avoid", "stop", "waypoints"), distthresh=4.0)),
    ("pathdist", dict(pathdist=1)),
    ("pathdist_waypoints", dict(pathdist=1, masks=("waypoints",))),
    ("modeuler", dict(modeuler=1)),
    ("modeuler_randfib2_usef", dict(modeuler=1, randfib=2, usef=1)),
    ("loopcheck_low_cthr", dict(loopcheck=1, c_thr=0.05)),
    ("everything", dict(modeuler=1, loopcheck=1, pathdist=1, distthresh=3.0, masks=("avoid", "stop", "waypoints"))),
    ("per_seed", dict(per_seed=1)),
    ("per_seed_pathdist_waypoints", dict(per_seed=1, pathdist=1, masks=("waypoints",))),
]


def _masks(mask, which):
    """Planes across the synthetic field's x-running tracts (nz, ny, nx = 10, 16, 20): avoid at
    x = 17, stop at x = 3, two waypoints at x = 8 and x = 12 (each changes the oracle's counts)."""
    out = {}
    if "avoid" in which:
        out["avoid"] = np.zeros_like(mask)
        out["avoid"][:, :, 17] = 1.0
    if "stop" in which:
        out["stop"] = np.zeros_like(mask)
        out["stop"][:, :, 3] = 2.0
    if "waypoints" in which:
        a, b = np.zeros_like(mask), np.zeros_like(mask)
        a[:, :, 8] = 1.0
        b[:, :, 12] = 1.0
        out["waypoints"] = [a, b]
    return out


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_tracking_equals_oracle(torch, name, kw):
    from fdt_b200 import lib

    lib.load()
    th, ph, f, mask = synth.fibre_field((20, 16, 10), nsamples=12, seed=4)
    seeds = np.array([[5.0, 8.0, 5.0], [14.0, 7.0, 4.6], [10.3, 3.2, 5.5], [0.0, 0.0, 0.0]], np.float32)
    kw = dict(kw)
    masks = _masks(mask, kw.pop("masks", ()))
    o = TrackOptions.make(nparticles=200, nsteps=kw.pop("nsteps", 300), seed=17, **kw)
    want_p, want_w = O.probtrack(o, th, ph, f, mask, seeds, voxel_size=(2.0, 2.0, 2.5), **masks)
    dev = [lib.to_device(a) for a in (th, ph, f, mask)]
    dmasks = {k: (lib.to_device(v) if k != "waypoints" else v) for k, v in masks.items()}
    got_p, got_w = lib.probtrack(o, *dev, seeds, voxel_size=(2.0, 2.0, 2.5), **dmasks)
    torch.cuda.synchronize()
    got_p = got_p.cpu().numpy()
    assert got_w == want_w, (name, got_w, want_w)
    assert np.array_equal(got_p, want_p), (name, np.argwhere(got_p != want_p)[:5])
    assert want_p.sum() > 0


def test_tracking_on_bedpostx_outputs_equals_oracle(torch):
    from fdt_b200 import lib, nifti

    lib.load()
    # a small volume through this library's bedpostx, its merged samples tracked from two seeds
    shape = (12, 10, 6)
    mask = synth.ellipsoid_mask(shape, 400)
    n = int(mask.sum())
    prot = synth.three_shell(9, 90)
    y, _ = synth.make_volume(n, prot, 2, True, 25.0, seed=8)
    o = Options.make(model=2, nfibres=2, nburn=100, njumps=200, sampleevery=10)
    out = lib.xfibres_dev(o, lib.to_device(y), lib.to_device(prot.bvecs), lib.to_device(prot.bvals))
    torch.cuda.synchronize()
    K, ns = 2, o.nsamples
    vols = {}
    for k in ("th", "ph", "f"):
        a = out[k].cpu().numpy()  # [K][ns][n]
        # merged_{k}{fibre}samples as volumes [x][y][z][ns], stored [fibre][ns][z][y][x]
        v = np.stack([nifti.from_matrix(a[kk].T, mask) for kk in range(K)])  # [K][x][y][z][ns]
        vols[k] = np.ascontiguousarray(np.transpose(v, (0, 4, 3, 2, 1)), np.float32)
    m = np.ascontiguousarray(np.transpose(mask.astype(np.float32), (2, 1, 0)))
    seeds = np.array([[6.0, 5.0, 3.0], [4.0, 4.0, 2.0]], np.float32)
    t = TrackOptions.make(nparticles=300, nsteps=400, seed=5)
    want_p, want_w = O.probtrack(t, vols["th"], vols["ph"], vols["f"], m, seeds)
    got_p, got_w = lib.probtrack(t, *(lib.to_device(vols[k]) for k in ("th", "ph", "f")), lib.to_device(m), seeds)
    torch.cuda.synchronize()
    assert got_w == want_w and np.array_equal(got_p.cpu().numpy(), want_p)


def test_probtrack_cli_with_masks_equals_oracle(torch, tmp_path):
    """python -m fdt_b200.probtrack on a bedpostX directory with --avoid, --stop and a waypoint list,
    in simple mode (a seed file: one path distribution per point) and seedmask mode (a seed mask:
    one over all its voxels): the volumes and waytotal equal the oracle's on the same arrays."""
    import os

    from fdt_b200 import nifti, probtrack

    th, ph, f, mask = synth.fibre_field((20, 16, 10), nsamples=12, seed=4)
    d = str(tmp_path)
    synth.write_bedpostx_dir(d, th, ph, f, mask)
    masks = _masks(mask, ("avoid", "stop", "waypoints"))
    for name, m in (("avoid", masks["avoid"]), ("stop", masks["stop"]), ("w1", masks["waypoints"][0]),
                    ("w2", masks["waypoints"][1])):
        nifti.write(os.path.join(d, name + ".nii.gz"), np.transpose(m, (2, 1, 0)))
    with open(os.path.join(d, "ways.txt"), "w") as fh:
        fh.write("w1.nii.gz\nw2.nii.gz\n")
    common = ["-P", "150", "-S", "300", "--seed", "23", "--avoid", os.path.join(d, "avoid.nii.gz"), "--stop",
              os.path.join(d, "stop.nii.gz"), "--waypoints", os.path.join(d, "ways.txt")]
    # simple mode
    seeds = np.array([[5.0, 8.0, 5.0], [14.0, 7.0, 4.5]], np.float32)
    np.savetxt(os.path.join(d, "seeds.txt"), seeds)
    out = os.path.join(d, "simple")
    probtrack.main([d, "--seeds", os.path.join(d, "seeds.txt"), "--out", out] + common)
    o = TrackOptions.make(nparticles=150, nsteps=300, seed=23, per_seed=1)
    # the directory's NIfTI files carry unit voxels
    want_p, want_w = O.probtrack(o, th, ph, f, mask, seeds, voxel_size=(1.0, 1.0, 1.0), **masks)
    assert int(open(os.path.join(out, "waytotal")).read()) == want_w > 0
    for i, name in enumerate(("fdt_paths_5_8_5", "fdt_paths_14_7_4.5")):
        got, _ = nifti.read(os.path.join(out, name + ".nii.gz"))
        assert np.array_equal(np.transpose(got, (2, 1, 0)), want_p[i]), name
    # seedmask mode
    sm = np.zeros_like(mask)
    sm[5, 8, 5] = sm[4, 7, 14] = sm[5, 3, 10] = 1.0
    nifti.write(os.path.join(d, "seedmask.nii.gz"), np.transpose(sm, (2, 1, 0)))
    out = os.path.join(d, "seedmask")
    probtrack.main([d, "--seeds", os.path.join(d, "seedmask.nii.gz"), "--out", out, "--targetmasks",
                    os.path.join(d, "ways.txt"), "--os2t"] + common)
    pts = np.argwhere(sm > 0)[:, ::-1].astype(np.float32)  # z, y, x order of the voxels, as x y z
    o.per_seed = 0
    want_p, want_w, want_s = O.probtrack(o, th, ph, f, mask, pts, voxel_size=(1.0, 1.0, 1.0),
                                         targets=masks["waypoints"], **masks)
    got, _ = nifti.read(os.path.join(out, "fdt_paths.nii.gz"))
    assert int(open(os.path.join(out, "waytotal")).read()) == want_w > 0
    assert np.array_equal(np.transpose(got, (2, 1, 0)), want_p)
    # seeds_to_<target>: each seed voxel's count
    for t, name in enumerate(("w1", "w2")):
        vol, _ = nifti.read(os.path.join(out, f"seeds_to_{name}.nii.gz"))
        at = vol[pts[:, 0].astype(int), pts[:, 1].astype(int), pts[:, 2].astype(int)]
        assert np.array_equal(at, want_s[t]) and vol.sum() == want_s[t].sum(), name
    assert want_s.sum() > 0
    # --omatrix2 --lrmask: a tract-space mask of 2 mm voxels (the directory's voxels are 1 mm)
    lr = np.zeros((5, 8, 10), np.float32)
    lr[1:4, 2:6, 1:9] = 1.0
    lr_x = np.transpose(lr, (2, 1, 0))
    nifti.write(os.path.join(d, "lr.nii.gz"), lr_x, like=nifti.Header(dim=lr_x.shape, pixdim=(1.0, 2.0, 2.0, 2.0) + (1.0,) * 4))
    out = os.path.join(d, "matrix2")
    probtrack.main([d, "--seeds", os.path.join(d, "seedmask.nii.gz"), "--out", out, "--omatrix2", "--lrmask",
                    os.path.join(d, "lr.nii.gz")] + common)
    _, lr_hdr = nifti.read(os.path.join(d, "lr.nii.gz"))
    lr_vs = tuple(float(x) for x in lr_hdr.pixdim[1:4])
    _, _, want_m2 = O.probtrack(o, th, ph, f, mask, pts, voxel_size=(1.0, 1.0, 1.0), matrix2=(lr, lr_vs), **masks)
    got, _ = nifti.read(os.path.join(out, "fdt_matrix2.nii.gz"))
    assert got.shape[:2] == want_m2.shape and np.array_equal(got.reshape(want_m2.shape), want_m2)
    assert want_m2.sum() > 0
    lut, _ = nifti.read(os.path.join(out, "lookup_tractspace_fdt_matrix2.nii.gz"))
    tc, _ = nifti.read(os.path.join(out, "tract_space_coords_for_fdt_matrix2.nii.gz"))
    tc = tc.reshape(-1, 3)
    assert tc.shape[0] == want_m2.shape[1] and np.array_equal(lut[tc[:, 0], tc[:, 1], tc[:, 2]], np.arange(tc.shape[0]))
    sc, _ = nifti.read(os.path.join(out, "coords_for_fdt_matrix2.nii.gz"))
    assert np.array_equal(sc.reshape(-1, 3), pts.astype(int))
    # --omatrix1 (with --omatrix2 beside it): seeds x seed voxels
    out = os.path.join(d, "matrix1")
    probtrack.main([d, "--seeds", os.path.join(d, "seedmask.nii.gz"), "--out", out, "--omatrix1", "--omatrix2",
                    "--lrmask", os.path.join(d, "lr.nii.gz")] + common)
    _, _, want_m2b, want_m1 = O.probtrack(o, th, ph, f, mask, pts, voxel_size=(1.0, 1.0, 1.0), matrix2=(lr, lr_vs),
                                          matrix1=sm, **masks)
    got, _ = nifti.read(os.path.join(out, "fdt_matrix1.nii.gz"))
    assert got.shape[:2] == (3, 3) and np.array_equal(got.reshape(3, 3), want_m1) and want_m1.sum() > 0
    got, _ = nifti.read(os.path.join(out, "fdt_matrix2.nii.gz"))
    assert np.array_equal(got.reshape(want_m2b.shape), want_m2b)
    sc, _ = nifti.read(os.path.join(out, "coords_for_fdt_matrix1.nii.gz"))
    assert np.array_equal(sc.reshape(-1, 3), pts.astype(int))


@pytest.mark.parametrize("kw", [dict(), dict(distthresh=6.0), dict(modeuler=1, per_seed=1)], ids=["plain", "distthresh",
                                                                                           "modeuler_per_seed"])
def test_seeds_to_targets_equal_oracle(torch, kw):
    from fdt_b200 import lib

    lib.load()
    th, ph, f, mask = synth.fibre_field((20, 16, 10), nsamples=12, seed=4)
    seeds = np.array([[5.0, 8.0, 5.0], [14.0, 7.0, 4.6], [10.3, 3.2, 5.5]], np.float32)
    targets = _masks(mask, ("waypoints",))["waypoints"] + [_masks(mask, ("avoid",))["avoid"]]
    o = TrackOptions.make(nparticles=200, nsteps=300, seed=31, **kw)
    want_p, want_w, want_s = O.probtrack(o, th, ph, f, mask, seeds, targets=targets)
    got_p, got_w, got_s = lib.probtrack(o, *(lib.to_device(a) for a in (th, ph, f, mask)), seeds, targets=targets)
    torch.cuda.synchronize()
    assert got_w == want_w and np.array_equal(got_p.cpu().numpy(), want_p)
    assert np.array_equal(got_s, want_s) and want_s.sum() > 0, (got_s, want_s)


M2_CASES = [
    ("plain", dict()),
    ("pathdist", dict(pathdist=1)),
    ("masks_distthresh", dict(masks=("avoid", "stop", "waypoints"), distthresh=3.0)),
    ("modeuler_loopcheck_per_seed", dict(modeuler=1, loopcheck=1, per_seed=1)),
    ("with_targets", dict(targets=True, randfib=2)),
]


@pytest.mark.parametrize("name,kw", M2_CASES, ids=[c[0] for c in M2_CASES])
def test_matrix2_equals_oracle(torch, name, kw):
    """--omatrix2 on a tract-space grid of 3 mm voxels over a field of 2 x 2 x 2.5 mm voxels (the
    tract-space voxel changes inside diffusion voxels), a mask of about 70% of it."""
    from fdt_b200 import lib

    lib.load()
    th, ph, f, mask = synth.fibre_field((20, 16, 10), nsamples=12, seed=4)
    seeds = np.array([[5.0, 8.0, 5.0], [14.0, 7.0, 4.6], [10.3, 3.2, 5.5]], np.float32)
    lr = (np.random.default_rng(3).random((9, 11, 14)) < 0.7).astype(np.float32)
    kw = dict(kw)
    extra = _masks(mask, kw.pop("masks", ()))
    if kw.pop("targets", False):
        extra["targets"] = _masks(mask, ("waypoints",))["waypoints"]
    o = TrackOptions.make(nparticles=200, nsteps=300, seed=41, **kw)
    m2 = (lr, (3.0, 3.0, 3.0))
    want = O.probtrack(o, th, ph, f, mask, seeds, voxel_size=(2.0, 2.0, 2.5), matrix2=m2, **extra)
    dev = [lib.to_device(a) for a in (th, ph, f, mask)]
    dextra = {k: (lib.to_device(v) if k in ("avoid", "stop") else v) for k, v in extra.items()}
    got = lib.probtrack(o, *dev, seeds, voxel_size=(2.0, 2.0, 2.5), matrix2=m2, **dextra)
    torch.cuda.synchronize()
    assert got[1] == want[1] and np.array_equal(got[0].cpu().numpy(), want[0])
    for g, w in zip(got[2:], want[2:]):
        assert np.array_equal(g, w), (name, np.argwhere(g != w)[:5])
    assert want[-1].sum() > 0 and want[-1].shape == (3, int(lr.sum()))


M1_CASES = [
    ("plain", dict()),
    ("pathdist", dict(pathdist=1)),
    ("masks_distthresh", dict(masks=("avoid", "stop", "waypoints"), distthresh=3.0)),
    ("modeuler_loopcheck", dict(modeuler=1, loopcheck=1)),
    ("with_matrix2", dict(matrix2=True)),
]


@pytest.mark.parametrize("name,kw", M1_CASES, ids=[c[0] for c in M1_CASES])
def test_matrix1_equals_oracle(torch, name, kw):
    """--omatrix1 in seedmask mode: every voxel of a seed mask seeds, and each seed's row counts its
    kept streamlines through every seed-mask voxel (bit for bit against the oracle)."""
    from fdt_b200 import lib

    lib.load()
    th, ph, f, mask = synth.fibre_field((20, 16, 10), nsamples=12, seed=4)
    seedmask = np.zeros_like(mask)
    seedmask[4:6, 6:10, 6:13] = mask[4:6, 6:10, 6:13]
    seeds = np.argwhere(seedmask != 0)[:, ::-1].astype(np.float32)
    kw = dict(kw)
    extra = _masks(mask, kw.pop("masks", ()))
    if kw.pop("matrix2", False):
        extra["matrix2"] = ((np.random.default_rng(5).random((9, 11, 14)) < 0.7).astype(np.float32), (3.0, 3.0, 3.0))
    o = TrackOptions.make(nparticles=50, nsteps=300, seed=43, **kw)
    want = O.probtrack(o, th, ph, f, mask, seeds, voxel_size=(2.0, 2.0, 2.5), matrix1=seedmask, **extra)
    dev = [lib.to_device(a) for a in (th, ph, f, mask)]
    dextra = {k: (lib.to_device(v) if k in ("avoid", "stop") else v) for k, v in extra.items()}
    got = lib.probtrack(o, *dev, seeds, voxel_size=(2.0, 2.0, 2.5), matrix1=seedmask, **dextra)
    torch.cuda.synchronize()
    assert got[1] == want[1] and np.array_equal(got[0].cpu().numpy(), want[0])
    for g, w in zip(got[2:], want[2:]):
        assert np.array_equal(g, w), (name, np.argwhere(g != w)[:5])
    assert want[-1].sum() > 0 and want[-1].shape == (len(seeds), len(seeds))


PREF_CASES = [
    ("plain", dict()),
    ("modeuler", dict(modeuler=1)),
    ("loopcheck_pathdist", dict(loopcheck=1, pathdist=1)),
    ("randfib_usef_masks", dict(randfib=2, usef=1, masks=("avoid", "waypoints"))),
    ("with_matrix1", dict(matrix1=True)),
]


@pytest.mark.parametrize("name,kw", PREF_CASES, ids=[c[0] for c in PREF_CASES])
def test_prefdir_equals_oracle(torch, name, kw):
    """--prefdir on the crossing field: a preferred direction per voxel (unit vectors, zero in a
    third of the voxels, where the current direction decides); bit for bit against the oracle."""
    from fdt_b200 import lib

    lib.load()
    th, ph, f, mask = synth.fibre_field((20, 16, 10), nsamples=12, seed=4)
    rng = np.random.default_rng(9)
    pref = rng.normal(size=(3,) + mask.shape).astype(np.float32)
    pref /= np.linalg.norm(pref, axis=0, keepdims=True)
    pref[:, rng.random(mask.shape) < 1 / 3] = 0.0
    seeds = np.array([[5.0, 8.0, 5.0], [14.0, 7.0, 4.6], [10.3, 3.2, 5.5]], np.float32)
    kw = dict(kw)
    extra = _masks(mask, kw.pop("masks", ()))
    if kw.pop("matrix1", False):
        sm = np.zeros_like(mask)
        sm[4:6, 6:10, 6:13] = mask[4:6, 6:10, 6:13]
        seeds = np.argwhere(sm != 0)[:, ::-1].astype(np.float32)
        extra["matrix1"] = sm
    o = TrackOptions.make(nparticles=100, nsteps=300, seed=47, **kw)
    want = O.probtrack(o, th, ph, f, mask, seeds, prefdir=pref, **extra)
    dev = [lib.to_device(a) for a in (th, ph, f, mask)]
    dextra = {k: (lib.to_device(v) if k in ("avoid", "stop") else v) for k, v in extra.items()}
    got = lib.probtrack(o, *dev, seeds, prefdir=pref, **dextra)
    torch.cuda.synchronize()
    assert got[1] == want[1] > 0 and np.array_equal(got[0].cpu().numpy(), want[0]), name
    for g, w in zip(got[2:], want[2:]):
        assert np.array_equal(g, w), name
    # the preferred directions change the paths
    plain = O.probtrack(o, th, ph, f, mask, seeds, **extra)
    assert not np.array_equal(plain[0], want[0])


@pytest.mark.parametrize("modeuler", [0, 1])
def test_loopcheck_on_circling_tracts_equals_oracle(torch, modeuler):
    from fdt_b200 import lib

    lib.load()
    th, ph, f, mask = synth.circle_field()
    seeds = np.array([[13.5, 11.5, 3.0], [17.5, 11.5, 2.0], [11.5, 14.2, 4.0]], np.float32)
    o = TrackOptions.make(nparticles=300, nsteps=1000, seed=21, loopcheck=1, modeuler=modeuler)
    want_p, want_w = O.probtrack(o, th, ph, f, mask, seeds)
    got_p, got_w = lib.probtrack(o, *(lib.to_device(a) for a in (th, ph, f, mask)), seeds)
    torch.cuda.synchronize()
    assert got_w == want_w and np.array_equal(got_p.cpu().numpy(), want_p)
    o.loopcheck = 0
    free, _ = O.probtrack(o, th, ph, f, mask, seeds)
    assert want_p.sum() < free.sum()  # the check acted


def test_probtrack_network_mode_equals_oracle(torch, tmp_path):
    """--network: each mask seeds in turn, keeping streamlines that reach another mask; the summed
    fdt_paths and the per-mask waytotal equal the oracle run mask by mask."""
    import os

    from fdt_b200 import nifti, probtrack

    th, ph, f, mask = synth.fibre_field((20, 16, 10), nsamples=12, seed=4)
    d = str(tmp_path)
    synth.write_bedpostx_dir(d, th, ph, f, mask)
    masks = []
    for i, (z, y, x) in enumerate([(5, 8, 4), (5, 8, 10), (4, 7, 15)]):
        mk = np.zeros_like(mask)
        mk[z - 1:z + 1, y - 1:y + 1, x] = 1.0
        masks.append(mk)
        nifti.write(os.path.join(d, f"m{i}.nii.gz"), np.transpose(mk, (2, 1, 0)))
    with open(os.path.join(d, "masks.txt"), "w") as fh:
        fh.write("m0.nii.gz\nm1.nii.gz\nm2.nii.gz\n")
    out = os.path.join(d, "net")
    probtrack.main([d, "--seeds", os.path.join(d, "masks.txt"), "--network", "--out", out, "-P", "100", "-S", "300",
                    "--seed", "41"])
    o = TrackOptions.make(nparticles=100, nsteps=300, seed=41)
    total = np.zeros(mask.shape, np.int64)
    ways = []
    for i, mi in enumerate(masks):
        others = sum(mj for j, mj in enumerate(masks) if j != i)
        pts = np.argwhere(mi > 0)[:, ::-1].astype(np.float32)
        p, w = O.probtrack(o, th, ph, f, mask, pts, voxel_size=(1.0, 1.0, 1.0), waypoints=[others])
        total += p
        ways.append(w)
    got, _ = nifti.read(os.path.join(out, "fdt_paths.nii.gz"))
    assert [int(x) for x in open(os.path.join(out, "waytotal")).read().split()] == ways and sum(ways) > 0
    assert np.array_equal(np.transpose(got, (2, 1, 0)), total)


def test_probtrack_twomasks_mode_is_network_mode_of_two(torch, tmp_path):
    import os

    from fdt_b200 import nifti, probtrack

    th, ph, f, mask = synth.fibre_field((20, 16, 10), nsamples=12, seed=4)
    d = str(tmp_path)
    synth.write_bedpostx_dir(d, th, ph, f, mask)
    for i, x in enumerate((4, 12)):
        mk = np.zeros_like(mask)
        mk[4:6, 7:9, x] = 1.0
        nifti.write(os.path.join(d, f"m{i}.nii.gz"), np.transpose(mk, (2, 1, 0)))
    with open(os.path.join(d, "two.txt"), "w") as fh:
        fh.write("m0.nii.gz\nm1.nii.gz\n")
    common = ["-P", "80", "-S", "300", "--seed", "5"]
    probtrack.main([d, "--seeds", os.path.join(d, "m0.nii.gz"), "--mask2", os.path.join(d, "m1.nii.gz"), "--out",
                    os.path.join(d, "two")] + common)
    probtrack.main([d, "--seeds", os.path.join(d, "two.txt"), "--network", "--out", os.path.join(d, "net")] + common)
    a, _ = nifti.read(os.path.join(d, "two", "fdt_paths.nii.gz"))
    b, _ = nifti.read(os.path.join(d, "net", "fdt_paths.nii.gz"))
    wa = open(os.path.join(d, "two", "waytotal")).read().split()
    assert np.array_equal(a, b) and a.sum() > 0 and wa == open(os.path.join(d, "net", "waytotal")).read().split()
    assert len(wa) == 2
