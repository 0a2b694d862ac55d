"""Host logic of the posterior-agreement statistics (fdt_b200/agreement.py), on synthetic chains."""
import numpy as np

from fdt_b200 import agreement


def _records(rng, nvox, R, K, ns, f_true, shift=0.0, rho=0.9):
    """AR(1) chains around per-voxel means (autocorrelated, as MCMC samples are)."""
    n = nvox * R
    rec = np.zeros((6 + 3 * K, ns, n))
    mu = np.concatenate([f_true] * R, axis=1) + shift  # [K][n]
    x = np.zeros((K, n))
    for s in range(ns):
        x = rho * x + np.sqrt(1 - rho * rho) * rng.normal(0, 0.02, (K, n))
        for k in range(K):
            rec[8 + 3 * k, s] = mu[k] + x[k]
            rec[6 + 3 * k, s] = 0.5 + 0.01 * rng.normal(size=n)
            rec[7 + 3 * k, s] = 1.0 + k + 0.01 * rng.normal(size=n)
        rec[0, s] = 1e-3 + 1e-5 * rng.normal(size=n)
        rec[5, s] = 1000 + rng.normal(size=n)
    return rec


def test_two_sets_of_one_distribution_agree_at_the_nominal_rate():
    rng = np.random.default_rng(0)
    nvox, K, ns = 2000, 2, 50
    f_true = np.stack([rng.uniform(0.4, 0.6, nvox), rng.uniform(0.1, 0.25, nvox)])
    a = agreement.ChainSet(_records(rng, nvox, 16, K, ns, f_true), K, 16)
    b = agreement.ChainSet(_records(rng, nvox, 16, K, ns, f_true), K, 16)
    c = agreement.compare(a, b)
    for k in range(K):
        assert 0.92 <= c["f_within_2se"][k] <= 0.97, c  # t with ~30 dof: about 0.945
    assert c["dyad_median_deg_supported"] < 1.0
    # a shift of 3 standard errors is caught in most voxels
    se = 0.02 * np.sqrt((1 + 0.9) / (1 - 0.9) / ns) / 4  # AR(1) SE of a 16-chain mean
    d = agreement.ChainSet(_records(rng, nvox, 16, K, ns, f_true, shift=3 * np.sqrt(2) * se), K, 16)
    c2 = agreement.compare(d, a)
    assert max(c2["f_within_2se"]) < 0.5, c2


def test_fibres_are_sorted_per_chain_and_subsets_keep_voxels():
    rng = np.random.default_rng(1)
    nvox, K, ns, R = 50, 3, 20, 4
    f_true = np.stack([np.full(nvox, 0.1), np.full(nvox, 0.5), np.full(nvox, 0.2)])
    s = agreement.ChainSet(_records(rng, nvox, R, K, ns, f_true), K, R)
    p = s.pooled()
    assert np.all(p["f"][0] > p["f"][1]) and np.all(p["f"][1] > p["f"][2])
    assert np.allclose(p["f"][0], 0.5, atol=0.02)
    sub = s.subset(slice(0, 2))
    assert sub.R == 2 and sub.nvox == nvox and sub.pooled()["f"].shape == (K, nvox)


def test_replicate_orders_chains_by_block():
    x = np.arange(6).reshape(3, 2)
    r = agreement.replicate(x, 2)
    assert r.shape == (6, 2) and np.array_equal(r[3:], x) and np.array_equal(r[:3], x)


def test_truth_errors_rank_fibres_and_measure_angles():
    rng = np.random.default_rng(2)
    nvox, K, ns, R = 400, 2, 30, 4
    f_true = np.stack([rng.uniform(0.1, 0.25, nvox), rng.uniform(0.4, 0.6, nvox)])  # second fibre the larger
    rec = _records(rng, nvox, R, K, ns, f_true)
    s = agreement.ChainSet(rec, K, R)
    # true directions: the larger fibre (record fibre 1) at (th, ph) = (0.5, 2.0), the smaller at (0.5, 1.0)
    d2 = lambda th, ph: np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    v = np.zeros((nvox, K, 3))
    v[:, 0], v[:, 1] = d2(0.5, 1.0), d2(0.5, 2.0)
    e = agreement.truth_errors(s, f_true.T, v, np.full(nvox, 1e-3))
    assert e["f_abs_median"][0] < 0.01 and e["f_abs_median"][1] < 0.01, e
    assert e["dyad_deg_median"][0] < 1.0 and e["dyad_deg_median"][1] < 1.0, e
    assert e["d_rel_median"] < 0.01 and e["dyad_voxels"] == [nvox, nvox]
    # directions swapped between the ranks: the angle between them (~27 degrees) shows up
    e2 = agreement.truth_errors(s, f_true.T, v[:, ::-1], np.full(nvox, 1e-3))
    assert min(e2["dyad_deg_median"]) > 20.0, e2
