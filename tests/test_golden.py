"""The oracle reproduces its committed golden fixtures (tests/golden/, made by make_golden.py):
fits, a short chain on the shared Philox stream and the finished outputs of a longer chain."""
import glob
import os

import numpy as np
import pytest

from fdt_b200.abi import Options

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

import importlib.util  # noqa: E402

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
def test_oracle_reproduces_golden(oracle, name):
    c = make_golden.CASES[name]
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    o = Options.make(**c["opts"])
    y, bv, bl = g["y"], g["bvecs"], g["bvals"]
    params, tau, status = oracle.fit(o, y, bv, bl)
    np.testing.assert_allclose(params, g["params"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(tau, g["tau"], rtol=1e-9, atol=1e-12)
    assert np.array_equal(status, g["status"])
    rec = oracle.mcmc(Options.make(**c["opts"], **make_golden.SHORT), y, bv, bl, g["params"], g["tau"])
    np.testing.assert_allclose(rec, g["rec_short"], rtol=1e-9, atol=1e-12)
    of = Options.make(**c["opts"], **make_golden.FULL)
    fin = oracle.finish(of, oracle.mcmc(of, y, bv, bl, g["params"], g["tau"]))
    for k, v in fin.items():
        np.testing.assert_allclose(v, g["fin_" + k], rtol=1e-9, atol=1e-12, err_msg=k)


def test_every_fixture_has_a_case():
    names = {os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))}
    assert names == set(make_golden.CASES)
