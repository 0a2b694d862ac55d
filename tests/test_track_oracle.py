"""CPU checks of the probtrackx oracle (oracle/track_oracle.c): its sine/cosine is the GPU path's
(same literals, single-precision accuracy), and tracking follows the reference's rules on fields
whose answer is known: a straight tract is followed to the mask boundary in both directions and
every voxel on it is counted once per streamline; the curvature threshold stops a streamline at a
right-angle turn; the distance threshold drops short streamlines; the avoid, stop and waypoint
masks reject, end and select halves as Seedmanager::run and Streamliner::streamline do; --pd
weights voxels by their order on the path; --loopcheck stops paths that circle back on themselves;
--modeuler follows a straight tract as the plain steps do; --omatrix2 counts every tract-space voxel
once per streamline (column 0 never, as the reference's "column != 0" test has it); --omatrix1 is
each seed's path distribution read at the seed mask."""
import os
import re

import numpy as np

from fdt_b200 import synth
from fdt_b200.abi import TrackOptions
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_sincos_literals_match_the_gpu_header():
    hdr = open(os.path.join(ROOT, "fdt_b200", "csrc", "bpx_device.cuh")).read()
    src = open(os.path.join(ROOT, "oracle", "track_oracle.c")).read()
    for name in ("kSinQ", "kCosQ"):
        h = re.search(name + r"\(int i\) \{ return (.*?); \}", hdr).group(1)
        lits_h = [float(x.rstrip("f")) for x in re.findall(r"(-?[0-9.]+e?-?[0-9]*f)", h)]
        c = re.search(r"static const float " + name + r"\[3\] = \{(.*?)\};", src).group(1)
        lits_c = [float(x.strip().rstrip("f")) for x in c.split(",")]
        assert np.array_equal(np.float32(lits_h), np.float32(lits_c)), name


def test_sincos_fast_accuracy():
    xs = np.concatenate([np.linspace(-50, 50, 2001), [0.0, np.pi / 2, np.pi, -np.pi / 4]]).astype(np.float32)
    for x in xs:
        s, c = O.sincos_fast(float(x))
        assert abs(s - np.sin(np.float64(x))) < 3e-7 and abs(c - np.cos(np.float64(x))) < 3e-7, x


def _straight_box(n=(30, 9, 9)):
    nx, ny, nz = n
    K, ns = 1, 10
    th = np.full((K, ns, nz, ny, nx), np.pi / 2, np.float32)
    # phi slightly off 0: the reference takes no step for a sample with theta or phi exactly 0
    ph = np.full_like(th, 1e-4)
    f = np.full_like(th, 0.6)
    mask = np.zeros((nz, ny, nx), np.float32)
    mask[2:7, 2:7, 3:27] = 1.0
    return th, ph, f, mask


def test_straight_tract_is_followed_both_ways_and_counted_once_per_streamline():
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=50, nsteps=400, steplength=0.5, seed=3)
    paths, way = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]], voxel_size=(2.0, 2.0, 2.0))
    assert way == 50
    line = paths[4, 4, :]
    assert np.all(line[3:27] == 50) and np.all(line[:3] == 0) and np.all(line[27:] == 0)
    assert paths.sum() == line.sum()  # a straight path through voxel centres stays on its line


def test_pathdist_weights_the_dth_distinct_voxel_by_d():
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=20, nsteps=400, seed=3, pathdist=1)
    paths, way = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]])
    # 24 distinct voxels per streamline, the seed's first: weights 1..24 whichever half runs first
    assert way == 20 and paths.dtype == np.int32
    assert paths[4, 4, 15] == 20 and paths.sum() == 20 * (24 * 25 // 2)
    # k particles ran +x first (voxel 16 got 2, voxel 14 got 13), the others -x first (14, 2)
    k, r = divmod(20 * 14 - int(paths[4, 4, 16]), 12)
    assert r == 0 and 0 < k < 20 and paths[4, 4, 14] == 13 * k + 2 * (20 - k)


def test_per_seed_volumes_sum_to_the_volume_over_all_seeds():
    th, ph, f, mask = synth.fibre_field((16, 14, 8), nsamples=8, seed=2)
    seeds = [[4.0, 7.0, 4.0], [11.0, 6.0, 3.5], [8.0, 8.0, 4.0]]
    o = TrackOptions.make(nparticles=40, nsteps=200, seed=13)
    total, way = O.probtrack(o, th, ph, f, mask, seeds)
    o.per_seed = 1
    each, way_each = O.probtrack(o, th, ph, f, mask, seeds)
    assert each.shape == (3,) + mask.shape and way_each == way
    assert np.array_equal(each.sum(axis=0), total) and all(e.sum() > 0 for e in each)
    assert np.all(each[:, mask == 0] == 0)


def test_seeds_to_targets_count_streamlines_entering_each_target():
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=40, nsteps=400, seed=3)
    far = np.zeros_like(mask)
    far[0, 0, :] = 1.0  # outside the brain mask: never reached
    paths, way, s2t = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0], [10.0, 4.0, 4.0]],
                                  targets=[_plane(mask, 20), _plane(mask, 5), far])
    assert way == 80 and s2t.shape == (3, 2) and s2t.dtype == np.int32
    assert np.array_equal(s2t, [[40, 40], [40, 40], [0, 0]])
    # with distthresh 20 mm the x = 20 plane counts only where the counted path (first kept half,
    # then the second) is that long on arrival: after the -x half (24 mm), not straight from the seed
    o.distthresh = 20.0
    _, way, s2t = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]], targets=[_plane(mask, 20)])
    assert way == 40 and 0 < s2t[0, 0] < 40


def test_loopcheck_stops_paths_that_circle_back():
    th, ph, f, mask = synth.circle_field()
    seed = [[13.5, 11.5, 3.0]]  # two voxels from the axis: a circle fits in one coarse cell
    o = TrackOptions.make(nparticles=40, nsteps=1000, seed=3)
    free, way0 = O.probtrack(o, th, ph, f, mask, seed)
    o.loopcheck = 1
    checked, way1 = O.probtrack(o, th, ph, f, mask, seed)
    assert way0 == way1 == 40 and checked.sum() < 0.4 * free.sum() and np.all(checked <= free)
    # a straight tract never runs against itself
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=20, nsteps=400, seed=3)
    plain, _ = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]])
    o.loopcheck = 1
    assert np.array_equal(O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]])[0], plain)


def test_modeuler_follows_a_straight_tract_as_the_plain_steps_do():
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=20, nsteps=400, seed=3)
    plain, _ = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]])
    o.modeuler = 1
    euler, way = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]])
    assert way == 20 and np.array_equal(euler, plain)
    # on the circles the mean of the direction here and a step ahead differs from the plain step
    th, ph, f, mask = synth.circle_field()
    o = TrackOptions.make(nparticles=20, nsteps=300, seed=3)
    a, _ = O.probtrack(o, th, ph, f, mask, [[17.5, 11.5, 3.0]])
    o.modeuler = 1
    b, _ = O.probtrack(o, th, ph, f, mask, [[17.5, 11.5, 3.0]])
    assert not np.array_equal(a, b) and a.sum() > 0 and b.sum() > 0


def test_curvature_threshold_stops_at_a_right_angle_turn():
    th, ph, f, mask = _straight_box()
    ph[:, :, :, :, 20:] = np.pi / 2  # fibres turn to y at x = 20
    mask[2:7, 2:7, 3:27] = 1.0
    o = TrackOptions.make(nparticles=20, nsteps=400, c_thr=0.2, seed=5)
    paths, way = O.probtrack(o, th, ph, f, mask, [[10.0, 4.0, 4.0]])
    assert way == 20
    # positions in [19.5, 20) round to the first turned voxel but may still draw their sample from
    # voxel 19; no particle gets past x = 20, where both neighbours have turned
    assert paths[4, 4, 19] == 20 and 0 < paths[4, 4, 20] <= 20 and paths[4, 4, 21:].sum() == 0
    assert paths[4, 4, 3] == 20  # the other half reaches the boundary


def test_distance_threshold_drops_short_halves():
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=10, nsteps=400, distthresh=1000.0, seed=7)
    paths, way = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]])
    assert way == 0 and paths.sum() == 0


def test_crossing_field_options_run_and_conserve_counts():
    th, ph, f, mask = synth.fibre_field((16, 14, 8), nsamples=8, seed=2)
    seeds = [[4.0, 7.0, 4.0], [11.0, 6.0, 3.5]]
    for kw in (dict(), dict(randfib=1), dict(randfib=2), dict(randfib=3), dict(usef=1), dict(sampvox=1),
               dict(fibst=2)):
        o = TrackOptions.make(nparticles=30, nsteps=200, seed=11, **kw)
        paths, way = O.probtrack(o, th, ph, f, mask, seeds)
        assert 0 < way <= 60, kw
        assert paths.max() <= way and np.all(paths[mask == 0] == 0), kw
    # masks only ever remove streamlines or shorten them
    o = TrackOptions.make(nparticles=30, nsteps=200, seed=11)
    free, way0 = O.probtrack(o, th, ph, f, mask, seeds)
    slab = np.zeros_like(mask)
    slab[:, :, 8] = 1.0
    for kw in (dict(avoid=slab), dict(stop=slab), dict(waypoints=[slab])):
        paths, way = O.probtrack(o, th, ph, f, mask, seeds, **kw)
        assert way <= way0 and np.all(paths <= free), list(kw)


def _plane(mask, x):
    m = np.zeros_like(mask)
    m[:, :, x] = 1.0
    return m


def test_matrix2_on_the_diffusion_grid_is_the_per_seed_path_counts_inside_the_mask():
    # with the tract space equal to the diffusion grid every path position maps to its own voxel, so
    # a seed's matrix2 row is its path distribution read at the tract-space mask's voxels (z, y, x
    # order), column 0 excepted
    th, ph, f, mask = synth.fibre_field((16, 14, 8), nsamples=8, seed=2)
    seeds = [[4.0, 7.0, 4.0], [11.0, 6.0, 3.5], [8.0, 8.0, 4.0]]
    o = TrackOptions.make(nparticles=40, nsteps=200, seed=13, per_seed=1)
    lr = mask.copy()
    each, way, m2 = O.probtrack(o, th, ph, f, mask, seeds, matrix2=(lr, (2.0, 2.0, 2.0)))
    want = each[:, lr != 0]
    want[:, 0] = 0
    assert m2.shape == (3, int((lr != 0).sum())) and m2.dtype == np.int32
    assert np.array_equal(m2, want) and m2.sum() > 0
    # a tract-space mask of part of the grid keeps only its own columns
    lr2 = np.zeros_like(mask)
    lr2[:, 4:10, :] = mask[:, 4:10, :]
    _, _, m2b = O.probtrack(o, th, ph, f, mask, seeds, matrix2=(lr2, (2.0, 2.0, 2.0)))
    want = each[:, lr2 != 0]
    want[:, 0] = 0
    assert np.array_equal(m2b, want)


def test_matrix1_is_the_per_seed_path_counts_at_the_seed_mask():
    # Counter::update_matrix1 copies the seed's path distribution at every seed-mask voxel (z, y, x
    # order) into the seed's row, column 0 included; with --pd the same weighted counts
    th, ph, f, mask = synth.fibre_field((16, 14, 8), nsamples=8, seed=2)
    seedmask = np.zeros_like(mask)
    seedmask[3:6, 5:9, 4:12] = mask[3:6, 5:9, 4:12]
    zyx = np.argwhere(seedmask != 0)
    seeds = zyx[:, ::-1].astype(np.float32)  # seedmask mode's seeds: x y z, in z, y, x order
    for pd in (0, 1):
        o = TrackOptions.make(nparticles=20, nsteps=200, seed=17, per_seed=1, pathdist=pd)
        each, way, m1 = O.probtrack(o, th, ph, f, mask, seeds, matrix1=seedmask)
        assert m1.shape == (len(seeds), len(seeds)) and m1.dtype == np.int32
        assert np.array_equal(m1, each[:, seedmask != 0]) and m1.sum() > 0, pd
        assert np.all(np.diag(m1) > 0)  # every seed's streamlines start in its own voxel
        # the summed volume: the same matrix
        o.per_seed = 0
        paths, way2, m1b = O.probtrack(o, th, ph, f, mask, seeds, matrix1=seedmask)
        assert way2 == way and np.array_equal(m1b, m1) and np.array_equal(paths, each.sum(0))


def test_prefdir_chooses_the_fibre_closest_to_the_preferred_direction():
    # two fibres everywhere, along x (fibre 1) and along y (fibre 2); the first step follows fibre 1
    th, ph, f, mask = _straight_box()
    th = np.concatenate([th, th])
    ph = np.concatenate([ph, np.full_like(ph, np.pi / 2)])
    f = np.concatenate([f, f]) * np.float32(0.6)
    o = TrackOptions.make(nparticles=40, nsteps=400, seed=5)
    seed = [[15.0, 4.0, 4.0]]
    free, way = O.probtrack(o, th, ph, f, mask, seed)
    assert way == 40 and np.all(free[4, 4, 3:27] == 40)  # the current direction keeps it along x
    pref = np.zeros((3,) + mask.shape, np.float32)
    same, way0 = O.probtrack(o, th, ph, f, mask, seed, prefdir=pref)  # zero vectors: the current direction
    assert way0 == way and np.array_equal(same, free)
    pref[0] = 1.0  # along x: the same choice at every step
    alongx, _ = O.probtrack(o, th, ph, f, mask, seed, prefdir=pref)
    assert np.array_equal(alongx, free)
    pref[0], pref[1] = 0.0, 1.0  # along y: the second step turns by 90 degrees and the curvature test stops it
    alongy, wy = O.probtrack(o, th, ph, f, mask, seed, prefdir=pref)
    assert wy == 40 and alongy[4, 4, 3:13].sum() == 0 and alongy[4, 4, 18:27].sum() == 0
    assert 0 < alongy.sum() <= 40 * 4
    # with a curvature threshold that lets it turn, it follows y instead and leaves the x line
    o.c_thr = 0.0
    turned, _ = O.probtrack(o, th, ph, f, mask, seed, prefdir=pref)
    assert turned[4, 4, 3:13].sum() == 0 and turned[:, 2:7, 15].sum() > turned[4, 4, 15]


def test_matrix2_on_a_coarser_grid_counts_each_tract_space_voxel_once_per_streamline():
    th, ph, f, mask = _straight_box()  # 30 x 9 x 9 voxels of 2 mm, the tract along x at y = z = 4
    # tract space of 4 mm voxels: positions 2.5 <= x < 26.5 map to x_lr = round(x / 2) = 1 .. 13 at
    # y_lr = z_lr = 2; the mask holds x_lr = 1 .. 14 there, so x_lr = 1 is column 0 and never counted
    lr = np.zeros((5, 5, 15), np.float32)
    lr[2, 2, 1:15] = 1.0
    o = TrackOptions.make(nparticles=50, nsteps=400, seed=3)
    paths, way, m2 = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]], matrix2=(lr, (4.0, 4.0, 4.0)))
    assert way == 50 and m2.shape == (1, 14)
    assert m2[0, 0] == 0 and np.all(m2[0, 1:13] == 50) and m2[0, 13] == 0
    # --pd: the d-th tract-space voxel counted on a streamline adds d (12 counted columns)
    o.pathdist = 1
    _, _, m2 = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]], matrix2=(lr, (4.0, 4.0, 4.0)))
    assert m2.sum() == 50 * (12 * 13 // 2) and m2[0, 0] == 0


def test_avoid_mask_rejects_the_half_that_enters_it():
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=40, nsteps=400, seed=3)
    paths, way = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]], avoid=_plane(mask, 20))
    line = paths[4, 4, :]
    # one half of every particle runs into x = 20 and is dropped; the other reaches x = 3
    assert way == 40 and np.all(line[3:16] == 40) and line[16:].sum() == 0 and line[:3].sum() == 0


def test_stop_mask_ends_the_half_inside_it():
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=40, nsteps=400, seed=3)
    paths, way = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]], stop=_plane(mask, 20))
    line = paths[4, 4, :]
    assert way == 40 and np.all(line[3:21] == 40) and line[21:].sum() == 0


def test_one_waypoint_keeps_the_other_half_only_when_it_ran_second():
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=60, nsteps=400, seed=9)
    paths, way = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]], waypoints=[_plane(mask, 20)])
    line = paths[4, 4, :]
    # the half towards the waypoint is always kept; the other only when it ran second, after the
    # first had passed the waypoint (a first half that passed nothing gets reject flag 1 and is
    # dropped, although the second half then passes the waypoint)
    assert way == 60 and np.all(line[15:27] == 60)
    assert 0 < line[3] < 60 and np.all(line[3:15] == line[3])


def test_waypoints_passed_by_both_halves_together():
    th, ph, f, mask = _straight_box()
    o = TrackOptions.make(nparticles=30, nsteps=400, seed=9)
    both = [_plane(mask, 8), _plane(mask, 22)]
    paths, way = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]], waypoints=both)
    assert way == 30 and np.all(paths[4, 4, 3:27] == 30)
    unreachable = np.zeros_like(mask)
    unreachable[0, 0, :] = 1.0  # outside the brain mask
    paths, way = O.probtrack(o, th, ph, f, mask, [[15.0, 4.0, 4.0]], waypoints=[both[0], unreachable])
    assert way == 0 and paths.sum() == 0


def test_probtrack_cli_reads_samples_masks_and_waypoint_lists(tmp_path):
    from fdt_b200 import nifti, probtrack

    th, ph, f, mask = synth.fibre_field((12, 10, 6), nsamples=4, seed=1)
    synth.write_bedpostx_dir(str(tmp_path), th, ph, f, mask)
    rth, rph, rf, rm, _, vs = probtrack.read_samples(str(tmp_path))
    assert np.array_equal(rth, th) and np.array_equal(rph, ph) and np.array_equal(rf, f)
    assert np.array_equal(rm, mask) and vs == (1.0, 1.0, 1.0)
    w = np.zeros_like(mask)
    w[:, :, 5] = 1.0
    for name in ("w1.nii.gz", "w2.nii.gz"):
        nifti.write(os.path.join(str(tmp_path), name), np.transpose(w, (2, 1, 0)))
    lst = os.path.join(str(tmp_path), "waypoints.txt")
    with open(lst, "w") as fh:
        fh.write("w1.nii.gz\n\n" + os.path.join(str(tmp_path), "w2.nii.gz") + "\n")
    files = probtrack.waypoint_files(lst)
    assert [os.path.basename(p) for p in files] == ["w1.nii.gz", "w2.nii.gz"] and all(map(os.path.exists, files))
    assert probtrack.waypoint_files(files[0]) == [files[0]]
    assert np.array_equal(probtrack.read_mask(files[0], mask.shape[::-1]), w)
    # seeds: a text file of points (simple mode), or a mask's voxels in z, y, x order (seedmask mode)
    np.savetxt(os.path.join(str(tmp_path), "pts.txt"), [[1.0, 2.0, 3.0], [4.5, 5.0, 1.0]])
    pts, per_seed = probtrack.seed_points(os.path.join(str(tmp_path), "pts.txt"), mask.shape[::-1])
    assert per_seed and np.array_equal(pts, [[1, 2, 3], [4.5, 5, 1]])
    sm = np.zeros_like(mask)
    sm[1, 2, 3] = sm[0, 4, 5] = -2.0
    nifti.write(os.path.join(str(tmp_path), "sm.nii.gz"), np.transpose(sm, (2, 1, 0)))
    pts, per_seed = probtrack.seed_points(os.path.join(str(tmp_path), "sm.nii.gz"), mask.shape[::-1])
    assert not per_seed and np.array_equal(pts, [[5, 4, 0], [3, 2, 1]])


def test_probtrack_cli_reads_prefdir_and_checks_matrix1_arguments(tmp_path):
    import pytest

    from fdt_b200 import nifti, probtrack

    th, ph, f, mask = synth.fibre_field((12, 10, 6), nsamples=4, seed=1)
    synth.write_bedpostx_dir(str(tmp_path), th, ph, f, mask)
    grid = mask.shape[::-1]
    # --prefdir: a 4D [x][y][z][3] volume becomes [3][z][y][x]
    pref = np.random.default_rng(0).normal(size=(3,) + mask.shape).astype(np.float32)
    path = os.path.join(str(tmp_path), "pref.nii.gz")
    nifti.write(path, np.transpose(pref, (3, 2, 1, 0)))
    assert np.array_equal(probtrack.read_prefdir(path, grid), pref)
    bad = os.path.join(str(tmp_path), "pref2.nii.gz")
    nifti.write(bad, np.transpose(pref[:2], (3, 2, 1, 0)))  # two components
    with pytest.raises(ValueError):
        probtrack.read_prefdir(bad, grid)
    # --omatrix1 needs seedmask mode; matrix1 and matrix2 are not for multiple seed tractography
    np.savetxt(os.path.join(str(tmp_path), "pts.txt"), [[1.0, 2.0, 3.0]])
    with pytest.raises(SystemExit):
        probtrack.main([str(tmp_path), "--seeds", os.path.join(str(tmp_path), "pts.txt"), "--out",
                        os.path.join(str(tmp_path), "o"), "--omatrix1"])
    with pytest.raises(SystemExit):
        probtrack.main([str(tmp_path), "--seeds", os.path.join(str(tmp_path), "pts.txt"), "--out",
                        os.path.join(str(tmp_path), "o"), "--network", "--omatrix1"])
