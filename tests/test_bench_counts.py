"""The roofline accounting of bench.py: the canonical per-term operation counts reproduce the
published per-voxel figures of the whole-brain (C4), multi-shell (C1) and CPU-runnable (C0)
configurations, and the kernel's own formulation differs only where it hoists or merges work."""
import pytest

import bench
from fdt_b200.abi import Options


def test_whole_brain_counts():
    plain = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=1000, njumps=1250)
    learned = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=200, njumps=1250)
    mufu_p, fma_p = bench.mcmc_work_canonical(plain, 288)
    mufu_l, _ = bench.mcmc_work_canonical(learned, 288)
    assert mufu_p / 2250 == 4032 * 3 + 14 * 288 * 2 == 20160   # per iteration
    assert mufu_p == pytest.approx(45.36e6) and mufu_l == pytest.approx(29.232e6)
    assert fma_p / 2250 == 4032 * 6 + 14 * 288 * (3 + 4 + 12)


def test_multishell_and_small_counts():
    c1 = Options.make(model=2, nfibres=3, nburn=1000, njumps=1250)
    mufu, _ = bench.mcmc_work_canonical(c1, 279)
    assert mufu / 2250 == 3906 * 3 and mufu == pytest.approx(26.37e6, rel=1e-3)
    c0 = Options.make(model=1, nfibres=2, nburn=1000, njumps=1250)
    mufu0, _ = bench.mcmc_work_canonical(c0, 64)
    assert mufu0 / 2250 == 448


def test_kernel_formulation_hoists_and_merges():
    o = Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=200, njumps=1250)
    mufu_c, fma_c = bench.mcmc_work_canonical(o, 288)
    mufu_k, fp32_k = bench.mcmc_work_per_voxel(o, 288)
    # Gamma scale hoisted (2 instead of 3 per model-2 signal term), one log2 per five Rician terms
    assert mufu_k / 1450 == 4032 * 2 + 14 * 288 * 1.2
    # the log I0 polynomials are counted: 19 operations per Rician term instead of 12
    assert fp32_k - fma_c == 1450 * 14 * 288 * 7
