"""Posterior agreement between two sets of MCMC chains over the same voxels.

Criterion (c) of the path asks that two runs' posterior means of f, d and the fibre directions
(dyads) agree per voxel within two Monte-Carlo standard errors (MC SE), with a median dyad angle
difference below 1 degree.  The MC SE of a posterior mean is estimated here from R independent
chains per voxel (different random streams, same start): the chain means of a voxel are independent
draws, so SE = sd(chain means) / sqrt(R) holds whatever the autocorrelation inside each chain.
(One chain's 50 thinned samples give no reliable SE when the samples are strongly autocorrelated,
which is the case for the small fractions under ARD.)

A run is stored as records [6+3K][nsamples][R*nvox] (the record rows of the library: d, f0, tau,
d_std, R, S0, then th, ph, f per fibre), chain r of voxel v in column r*nvox + v.  Each chain is
finished as the reference finishes one (CUDA/samples.cu:299-330): fibres sorted by the sum of their
f over the samples, largest first; the dyad of a fibre is the principal eigenvector of its mean
dyadic tensor (CUDA/samples.cu:134-229).

For a perfect match with a known SE, |difference| <= 2 SE holds in 95.4% of voxels; with the SE
estimated from R chains per side the expected fraction is lower (about 94.5% at R = 16, 93% at
R = 8), which is why every comparison here is reported beside the same statistic for two
independent chain sets of one implementation (the yardstick).
"""
from __future__ import annotations

import numpy as np

REC_D, REC_F0, REC_TAU, REC_DSTD, REC_R, REC_S0 = 0, 1, 2, 3, 4, 5


def _dirs(th: np.ndarray, ph: np.ndarray) -> np.ndarray:
    st = np.sin(th)
    return np.stack([st * np.cos(ph), st * np.sin(ph), np.cos(th)], -1)


class ChainSet:
    """Per-chain summaries of R chains per voxel."""

    def __init__(self, rec: np.ndarray, nfib: int, R: int):
        rec = np.asarray(rec, np.float64)
        nrec, ns, n = rec.shape
        assert nrec == 6 + 3 * nfib and n % R == 0, (rec.shape, nfib, R)
        self.K, self.R, self.nvox = nfib, R, n // R
        r = rec.reshape(nrec, ns, R, self.nvox)  # [row][sample][chain][voxel]
        th = np.stack([r[6 + 3 * k] for k in range(nfib)])  # [K][ns][R][nvox]
        ph = np.stack([r[7 + 3 * k] for k in range(nfib)])
        f = np.stack([r[8 + 3 * k] for k in range(nfib)])
        order = np.argsort(-f.sum(1), axis=0, kind="stable")  # [K][R][nvox], per chain
        take = lambda a: np.take_along_axis(a, order[:, None], axis=0)
        th, ph, f = take(th), take(ph), take(f)
        self.f = f.mean(1)  # [K][R][nvox] chain means
        self.d = r[REC_D].mean(0)  # [R][nvox]
        self.S0 = r[REC_S0].mean(0)
        v = _dirs(th, ph)  # [K][ns][R][nvox][3]
        self.T = np.einsum("ksrvi,ksrvj->krvij", v, v) / ns  # mean dyadic tensor per chain

    def pooled(self):
        """Pooled posterior means over the R chains and their MC standard errors."""
        R = self.R
        se = lambda a: a.std(axis=-2, ddof=1) / np.sqrt(R) if R > 1 else np.full(a.shape[:-2] + a.shape[-1:], np.nan)
        f_m, f_se = self.f.mean(-2), se(self.f)
        d_m, d_se = self.d.mean(0), se(self.d)
        T = self.T.mean(1)  # [K][nvox][3][3]
        w, V = np.linalg.eigh(T)
        dyad = V[..., :, -1]  # eigenvector of the largest eigenvalue, [K][nvox][3]
        return dict(f=f_m, f_se=f_se, d=d_m, d_se=d_se, dyad=dyad)

    def subset(self, chains: slice | np.ndarray) -> "ChainSet":
        """The same voxels with a subset of the chains."""
        c = object.__new__(ChainSet)
        c.K, c.nvox = self.K, self.nvox
        c.f, c.d, c.S0, c.T = self.f[:, chains], self.d[chains], self.S0[chains], self.T[:, chains]
        c.R = c.d.shape[0]
        return c


def compare(a: ChainSet, b: ChainSet, fmin: float = 0.05) -> dict:
    """Agreement of two chain sets over the same voxels.

    f_within_2se[k], d_within_2se: fraction of voxels with |mean_a - mean_b| <= 2 sqrt(se_a^2 + se_b^2);
    dyad_median_deg[k]: median angle between the pooled dyads of fibre k;
    dyad_median_deg_supported: the median over fibres and voxels where both sets' mean f_k >= fmin
    (the bedpostx post-processing threshold below which a fibre's dyad is masked out, maskdyads).
    """
    pa, pb = a.pooled(), b.pooled()
    z = lambda ma, mb, sa, sb: np.abs(ma - mb) / np.maximum(np.sqrt(sa * sa + sb * sb), 1e-30)
    zf = z(pa["f"], pb["f"], pa["f_se"], pb["f_se"])  # [K][nvox]
    zd = z(pa["d"], pb["d"], pa["d_se"], pb["d_se"])
    cosang = np.clip(np.abs(np.sum(pa["dyad"] * pb["dyad"], -1)), 0.0, 1.0)
    ang = np.degrees(np.arccos(cosang))  # [K][nvox]
    sup = (pa["f"] >= fmin) & (pb["f"] >= fmin)
    return {
        "voxels": int(a.nvox),
        "chains": [int(a.R), int(b.R)],
        "f_within_2se": [round(float(np.mean(zf[k] <= 2.0)), 4) for k in range(a.K)],
        "d_within_2se": round(float(np.mean(zd <= 2.0)), 4),
        "dyad_median_deg": [round(float(np.median(ang[k])), 3) for k in range(a.K)],
        "dyad_median_deg_supported": round(float(np.median(ang[sup])), 3) if sup.any() else None,
        "supported_fraction": [round(float(np.mean(sup[k])), 4) for k in range(a.K)],
    }


def replicate(x: np.ndarray, R: int) -> np.ndarray:
    """Stack R copies of per-voxel rows (axis 0): chain r of voxel v becomes row r*nvox + v."""
    return np.ascontiguousarray(np.concatenate([x] * R, axis=0))


def truth_errors(s: ChainSet, f_true: np.ndarray, v_true: np.ndarray, d_true: np.ndarray,
                 fmin: float = 0.05) -> dict:
    """Errors of a chain set's pooled posterior means against the ground truth of synthetic voxels.

    f_true [nvox][K], v_true [nvox][K][3] (unit vectors), d_true [nvox].  True fibres are ranked by
    their fraction (largest first), as the finished outputs rank the estimated ones, and compared
    rank by rank:
      f_abs_median[k]: median |mean f_k - true f_k|;
      dyad_deg_median[k]: median angle between the pooled dyad and the true direction of rank k,
        over voxels whose true f_k >= fmin (a fibre below the post-processing threshold has no
        direction to recover);
      d_rel_median: median |mean d - true d| / true d.
    """
    p = s.pooled()
    K = s.K
    order = np.argsort(-f_true, axis=1, kind="stable")  # [nvox][K]
    ft = np.take_along_axis(f_true, order, axis=1).T  # [K][nvox]
    vt = np.take_along_axis(v_true, order[:, :, None], axis=1).transpose(1, 0, 2)  # [K][nvox][3]
    fe = np.abs(p["f"] - ft)
    cosang = np.clip(np.abs(np.sum(p["dyad"] * vt, -1)), 0.0, 1.0)
    ang = np.degrees(np.arccos(cosang))
    return {
        "voxels": int(s.nvox),
        "f_abs_median": [round(float(np.median(fe[k])), 4) for k in range(K)],
        "dyad_deg_median": [round(float(np.median(ang[k][ft[k] >= fmin])), 3) if np.any(ft[k] >= fmin) else None
                            for k in range(K)],
        "dyad_voxels": [int(np.sum(ft[k] >= fmin)) for k in range(K)],
        "d_rel_median": round(float(np.median(np.abs(p["d"] - d_true) / d_true)), 4),
    }
