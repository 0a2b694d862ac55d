"""Seeded synthetic diffusion data for the benchmark configurations.

The reference measures on no public dataset, so volumes are generated from the ball-and-stick
forward models themselves (the same models bedpostx fits; the reference's own generators
basgen.cc:115-145 and xfibres_pred.cc predict signals through PVM_single/PVM_multi the same way)
with Rician noise.  Protocols:

* ``single_shell_64``: 4 b=0 + 60 directions at b=1000 s/mm^2 (Fibonacci sphere).
* ``three_shell(nb0)``: ``nb0`` b=0 + 90 directions at each of b=1000/2000/3000.

Fibre orientations are uniform on the sphere, ``d ~ U(0.5e-3, 2e-3)`` mm^2/s, ``f1 ~ U(0.3, 0.7)``,
``f2 ~ U(0, min(0.3, 1-f1))``, ``f3 ~ U(0, 0.15)`` (clipped so that the fractions sum below 1),
``d_std ~ U(0.1, 0.5)*d`` for the Gamma-diffusivity model, S0 = 1000, and Rician noise
``|S + sigma*(n1 + i*n2)|`` with ``sigma = S0/SNR``.
"""
from __future__ import annotations

import dataclasses

import numpy as np

GOLDEN_ANGLE = np.pi * (3.0 - np.sqrt(5.0))


def fibonacci_sphere(n: int) -> np.ndarray:
    """``n`` near-uniform unit vectors, shape [3][n]."""
    i = np.arange(n, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = i * GOLDEN_ANGLE
    return np.stack([r * np.cos(phi), r * np.sin(phi), z])


@dataclasses.dataclass
class Protocol:
    bvecs: np.ndarray  # [3][ndir] float32, unit (zero rows for b=0)
    bvals: np.ndarray  # [ndir] float32

    @property
    def ndir(self) -> int:
        return int(self.bvals.shape[0])


def single_shell_64() -> Protocol:
    """4 b=0 + 60 directions at b=1000 (the CPU-runnable configuration)."""
    g = fibonacci_sphere(60)
    bvecs = np.concatenate([np.zeros((3, 4)), g], axis=1)
    bvals = np.concatenate([np.zeros(4), np.full(60, 1000.0)])
    return Protocol(bvecs.astype(np.float32), bvals.astype(np.float32))


def three_shell(nb0: int = 9, ndir_shell: int = 90) -> Protocol:
    """``nb0`` b=0 + ``ndir_shell`` directions at each of b=1000/2000/3000.

    b=0 volumes are spread through the acquisition (one every len/nb0 volumes), as scanners do.
    """
    g = fibonacci_sphere(ndir_shell)
    dw_vecs, dw_vals = [], []
    for s, b in enumerate((1000.0, 2000.0, 3000.0)):
        # rotate each shell's set about z so shells do not share directions
        ang = s * GOLDEN_ANGLE / 3.0
        c, sn = np.cos(ang), np.sin(ang)
        rot = np.array([[c, -sn, 0.0], [sn, c, 0.0], [0.0, 0.0, 1.0]])
        dw_vecs.append(rot @ g)
        dw_vals.append(np.full(ndir_shell, b))
    dw_vecs = np.concatenate(dw_vecs, axis=1)
    dw_vals = np.concatenate(dw_vals)
    # interleave the three shells so that any prefix samples all of them
    order = np.arange(3 * ndir_shell).reshape(3, ndir_shell).T.reshape(-1)
    dw_vecs, dw_vals = dw_vecs[:, order], dw_vals[order]
    n = nb0 + dw_vals.shape[0]
    b0_pos = set(np.linspace(0, n - 1, nb0).round().astype(int).tolist())
    bvecs = np.zeros((3, n))
    bvals = np.zeros(n)
    j = 0
    for i in range(n):
        if i in b0_pos:
            continue
        bvecs[:, i] = dw_vecs[:, j]
        bvals[i] = dw_vals[j]
        j += 1
    return Protocol(bvecs.astype(np.float32), bvals.astype(np.float32))


def truncated_three_shell(ndir: int) -> Protocol:
    """The first ``ndir`` volumes of the 279-volume three-shell scheme (mixed-batch sizes)."""
    full = three_shell(9, 90)
    if ndir > full.ndir:
        raise ValueError("ndir > 279")
    p = Protocol(full.bvecs[:, :ndir].copy(), full.bvals[:ndir].copy())
    if not np.any(p.bvals == 0):
        p.bvals[0] = 0.0
        p.bvecs[:, 0] = 0.0
    return p


def random_unit(rng: np.random.Generator, n: int) -> np.ndarray:
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


@dataclasses.dataclass
class Truth:
    S0: np.ndarray
    d: np.ndarray
    dstd: np.ndarray | None
    f: np.ndarray  # [nvox][nfib]
    v: np.ndarray  # [nvox][nfib][3]


def sample_truth(rng: np.random.Generator, nvox: int, nfib: int, gamma: bool) -> Truth:
    S0 = np.full(nvox, 1000.0)
    d = rng.uniform(0.5e-3, 2e-3, nvox)
    f = np.zeros((nvox, nfib))
    f[:, 0] = rng.uniform(0.3, 0.7, nvox)
    if nfib > 1:
        f[:, 1] = rng.uniform(0.0, 1.0, nvox) * np.minimum(0.3, 1.0 - f[:, 0])
    if nfib > 2:
        room = np.maximum(0.0, 0.99 - f[:, 0] - f[:, 1])
        f[:, 2] = rng.uniform(0.0, 1.0, nvox) * np.minimum(0.15, room)
    v = random_unit(rng, nvox * nfib).reshape(nvox, nfib, 3)
    dstd = rng.uniform(0.1, 0.5, nvox) * d if gamma else None
    return Truth(S0, d, dstd, f, v)


def predict(truth: Truth, prot: Protocol, gamma: bool) -> np.ndarray:
    """Noise-free signal [nvox][ndir] (float64)."""
    g = prot.bvecs.astype(np.float64)  # [3][ndir]
    b = prot.bvals.astype(np.float64)[None, :]
    d = truth.d[:, None]
    fsum = truth.f.sum(axis=1)[:, None]
    if gamma:
        s2 = (truth.dstd**2)[:, None]
        alpha = d * d / s2
        beta = s2 / d
        iso = np.exp(-alpha * np.log1p(beta * b))
    else:
        iso = np.exp(-b * d)
    sig = (1.0 - fsum) * iso
    for k in range(truth.f.shape[1]):
        c = (truth.v[:, k, :] @ g) ** 2
        if gamma:
            an = np.exp(-alpha * np.log1p(beta * b * c))
        else:
            an = np.exp(-b * d * c)
        sig = sig + truth.f[:, k : k + 1] * an
    return truth.S0[:, None] * sig


def add_rician(rng: np.random.Generator, s: np.ndarray, sigma: np.ndarray | float) -> np.ndarray:
    sigma = np.asarray(sigma, dtype=np.float64)
    if sigma.ndim == 1:
        sigma = sigma[:, None]
    n1 = rng.normal(size=s.shape)
    n2 = rng.normal(size=s.shape)
    return np.sqrt((s + sigma * n1) ** 2 + (sigma * n2) ** 2)


def ellipsoid_mask(shape: tuple[int, int, int], target: int) -> np.ndarray:
    """Boolean mask of a centred ellipsoid with about ``target`` voxels inside ``shape``."""
    nx, ny, nz = shape
    x, y, z = np.meshgrid(
        np.arange(nx) - (nx - 1) / 2.0,
        np.arange(ny) - (ny - 1) / 2.0,
        np.arange(nz) - (nz - 1) / 2.0,
        indexing="ij",
    )
    lo, hi = 0.05, 1.0
    for _ in range(60):
        s = 0.5 * (lo + hi)
        r = (x / (s * nx / 2.0)) ** 2 + (y / (s * ny / 2.0)) ** 2 + (z / (s * nz / 2.0)) ** 2
        cnt = int((r <= 1.0).sum())
        if cnt > target:
            hi = s
        else:
            lo = s
    r = (x / (lo * nx / 2.0)) ** 2 + (y / (lo * ny / 2.0)) ** 2 + (z / (lo * nz / 2.0)) ** 2
    return r <= 1.0


@dataclasses.dataclass
class Volume:
    data: np.ndarray  # [nvox][ndir] float32
    prot: Protocol
    truth: Truth
    model: int
    nfib: int
    shape: tuple[int, int, int] | None = None
    mask: np.ndarray | None = None

    @property
    def nvox(self) -> int:
        return int(self.data.shape[0])


def make_volume(
    nvox: int,
    prot: Protocol,
    nfib: int,
    gamma: bool,
    snr: float | np.ndarray,
    seed: int,
    chunk: int = 65536,
) -> tuple[np.ndarray, Truth]:
    rng = np.random.default_rng(seed)
    truth = sample_truth(rng, nvox, nfib, gamma)
    out = np.empty((nvox, prot.ndir), dtype=np.float32)
    snr = np.broadcast_to(np.asarray(snr, dtype=np.float64), (nvox,))
    for s in range(0, nvox, chunk):
        e = min(nvox, s + chunk)
        part = Truth(
            truth.S0[s:e],
            truth.d[s:e],
            None if truth.dstd is None else truth.dstd[s:e],
            truth.f[s:e],
            truth.v[s:e],
        )
        sig = predict(part, prot, gamma)
        out[s:e] = add_rician(rng, sig, truth.S0[s:e] / snr[s:e]).astype(np.float32)
    return out, truth


def config_small_model1(seed: int = 1, nvox: int = 500) -> Volume:
    """Model 1, 2 fibres, 10x10x5 = 500 voxels, 64 measurements, SNR 20."""
    prot = single_shell_64()
    data, truth = make_volume(nvox, prot, 2, False, 20.0, seed)
    return Volume(data, prot, truth, 1, 2, (10, 10, 5))


def config_multishell_model2(seed: int = 2, nvox: int | None = None) -> Volume:
    """Model 2, 3 fibres, 279 measurements, 96x96x60 ellipsoid of ~200k voxels, SNR 25."""
    prot = three_shell(9, 90)
    shape = (96, 96, 60)
    mask = None
    if nvox is None:
        mask = ellipsoid_mask(shape, 200_000)
        nvox = int(mask.sum())
    data, truth = make_volume(nvox, prot, 3, True, 25.0, seed)
    return Volume(data, prot, truth, 2, 3, shape, mask)


def config_whole_brain(seed: int = 4, nvox: int | None = None) -> Volume:
    """Model 2, 3 fibres, 288 measurements, 145x174x145 ellipsoid of ~900k voxels, SNR 25."""
    prot = three_shell(18, 90)
    shape = (145, 174, 145)
    mask = None
    if nvox is None:
        mask = ellipsoid_mask(shape, 900_000)
        nvox = int(mask.sum())
    data, truth = make_volume(nvox, prot, 3, True, 25.0, seed)
    return Volume(data, prot, truth, 2, 3, shape, mask)


def fibre_field(shape=(24, 20, 12), nsamples: int = 20, jitter: float = 0.08, seed: int = 0):
    """Posterior samples of a synthetic fibre field for tracking (the bedpostx outputs probtrackx
    reads): an ellipsoidal mask; fibre 1 runs along x everywhere, fibre 2 along y in the
    half-space x >= nx/2 (a crossing region), fibre 3 has f below the usual threshold.  Angles are
    jittered per sample by N(0, jitter) rad.  Returns th, ph, f [3][nsamples][nz][ny][nx] and
    mask [nz][ny][nx] (float32)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = [(nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2]
    r = ((xx - c[0]) / (0.48 * nx)) ** 2 + ((yy - c[1]) / (0.48 * ny)) ** 2 + ((zz - c[2]) / (0.48 * nz)) ** 2
    mask = (r <= 1.0).astype(np.float32)
    K = 3
    th = np.zeros((K, nsamples, nz, ny, nx), np.float32)
    ph = np.zeros_like(th)
    f = np.zeros_like(th)
    g = lambda: rng.normal(0.0, jitter, (nsamples, nz, ny, nx))  # noqa: E731
    th[0] = np.pi / 2 + g()
    ph[0] = 0.0 + g()
    f[0] = 0.5 + 0.05 * rng.standard_normal((nsamples, nz, ny, nx))
    cross = (xx >= nx // 2)[None]
    th[1] = np.pi / 2 + g()
    ph[1] = np.pi / 2 + g()
    f[1] = np.where(cross, 0.3, 0.005) + 0.02 * rng.standard_normal((nsamples, nz, ny, nx))
    th[2] = rng.uniform(0.1, np.pi - 0.1, (nsamples, nz, ny, nx))
    ph[2] = rng.uniform(-np.pi, np.pi, (nsamples, nz, ny, nx))
    f[2] = 0.004
    f = np.clip(f, 0.0, 1.0)
    return th, ph, f.astype(np.float32), mask


def write_bedpostx_dir(d: str, th, ph, f, mask) -> None:
    """Writes th/ph/f [K][nsamples][nz][ny][nx] and mask [nz][ny][nx] as a bedpostX directory holds
    them: merged_{th,ph,f}{k}samples ([x][y][z][nsamples]) and nodif_brain_mask, unit voxels."""
    import os

    from . import nifti

    os.makedirs(d, exist_ok=True)
    for q, a in (("th", th), ("ph", ph), ("f", f)):
        for k in range(a.shape[0]):
            nifti.write(os.path.join(d, f"merged_{q}{k + 1}samples.nii.gz"), np.transpose(a[k], (3, 2, 1, 0)))
    nifti.write(os.path.join(d, "nodif_brain_mask.nii.gz"), np.transpose(mask, (2, 1, 0)))


def circle_field(n: int = 24, nz: int = 6, nsamples: int = 8):
    """Fibres along circles about the grid's central z axis (th, ph, f [1][nsamples][nz][n][n] and a
    full mask): streamlines from a seed near the axis circle back through their own path."""
    c = (n - 1) / 2.0
    x = np.arange(n)[None, :]
    y = np.arange(n)[:, None]
    phi = (np.arctan2(y - c, x - c) + np.pi / 2).astype(np.float32)
    th = np.full((1, nsamples, nz, n, n), np.pi / 2, np.float32)
    ph = np.ascontiguousarray(np.broadcast_to(phi, th.shape))
    f = np.full_like(th, 0.8)
    return th, ph, f, np.ones((nz, n, n), np.float32)
