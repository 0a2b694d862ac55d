"""The C-ABI from C: tests/c_host/xfibres_host_example.c, a host program that includes
include/bpx.h and links libbpx.so and nothing else (no Python, no torch), runs bpx_xfibres_host on
a subpart written to raw files; its outputs equal the Python mirror's call of the same entry, bit
for bit.  The program is compiled here with gcc, as a reference-side host would build against the
library."""
import os
import subprocess

import numpy as np
import pytest

from fdt_b200 import build, synth
from fdt_b200.abi import Options

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_c_host_program_matches_the_python_mirror(torch, tmp_path):
    from fdt_b200 import lib

    d = str(tmp_path)
    exe = os.path.join(d, "xfibres_host_example")
    libdir = os.path.dirname(build.LIB)
    subprocess.run(["gcc", "-O2", "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c_host",
                                                                                          "xfibres_host_example.c"),
                    "-L" + libdir, "-lbpx", "-Wl,-rpath," + libdir, "-o", exe], check=True)
    prot = synth.three_shell(9, 90)
    y, _ = synth.make_volume(300, prot, 3, True, 25.0, seed=71)
    nvox, ndir = y.shape
    np.ascontiguousarray(y, np.float32).tofile(os.path.join(d, "data.f32"))
    np.ascontiguousarray(prot.bvecs, np.float32).tofile(os.path.join(d, "bvecs.f32"))
    np.ascontiguousarray(prot.bvals, np.float32).tofile(os.path.join(d, "bvals.f32"))
    args = dict(model=2, nfibres=3, nburn=100, njumps=200, sampleevery=10, rician=1, f0=1, seed=12345)
    r = subprocess.run([exe, d, str(nvox), str(ndir)] + [str(args[k]) for k in ("model", "nfibres", "nburn", "njumps",
                                                                                 "sampleevery", "rician", "f0", "seed")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    want = lib.xfibres_host(Options.make(**args), y, prot.bvecs, prot.bvals)
    ns = args["njumps"] // args["sampleevery"]
    for k, shape in (("th", (3, ns, nvox)), ("ph", (3, ns, nvox)), ("f", (3, ns, nvox)), ("mean_d", (nvox,)),
                     ("mean_S0", (nvox,))):
        got = np.fromfile(os.path.join(d, k + ".f32"), np.float32).reshape(shape)
        assert np.array_equal(got, want[k].numpy()), k
