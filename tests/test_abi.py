"""CPU tests of the C-ABI boundary: libbpx.so loads, exports every function include/bpx.h
declares, the ctypes mirror matches the C struct layout, and host-side argument checks reject
bad input without touching a device."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from fdt_b200 import abi, build
from fdt_b200.abi import Options, Outputs, Volume

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bpx.h")


@pytest.fixture(scope="module")
def libbpx():
    path = build.build()  # incremental: a no-op when the library is current
    return C.CDLL(path)


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bpx_[a-z0-9_]+)\s*\(", txt)))


def test_exports_every_declared_symbol(libbpx):
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(libbpx, n)]
    assert not missing, missing


def test_ctypes_structs_match_c_layout():
    src = r"""
#include <stddef.h>
#include <stdio.h>
#include "bpx.h"
#define F(T, m) printf(#T " " #m " %zu\n", offsetof(T, m));
int main(void) {
  printf("bpx_options size %zu\n", sizeof(bpx_options));
  printf("bpx_volume size %zu\n", sizeof(bpx_volume));
  printf("bpx_outputs size %zu\n", sizeof(bpx_outputs));
  printf("bpx_track_options size %zu\n", sizeof(bpx_track_options));
  printf("bpx_track_volume size %zu\n", sizeof(bpx_track_volume));
  F(bpx_options, seed) F(bpx_options, gradnonlin) F(bpx_options, mcmc_tpv) F(bpx_options, R_prior_fudge)
  F(bpx_volume, data) F(bpx_volume, voxel_offset) F(bpx_outputs, dyads) F(bpx_outputs, status)
  F(bpx_track_options, seed) F(bpx_track_options, pathdist) F(bpx_track_options, modeuler)
  F(bpx_track_volume, mask) F(bpx_track_volume, waypoints) F(bpx_track_volume, nwaypoints)
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            t, m, v = line.split()
            got[(t, m)] = int(v)
    assert got[("bpx_options", "size")] == C.sizeof(Options)
    assert got[("bpx_volume", "size")] == C.sizeof(Volume)
    assert got[("bpx_outputs", "size")] == C.sizeof(Outputs)
    assert got[("bpx_track_options", "size")] == C.sizeof(abi.TrackOptions)
    assert got[("bpx_track_volume", "size")] == C.sizeof(abi.TrackVolume)
    for (t, m), v in got.items():
        if m == "size":
            continue
        cls = {"bpx_options": Options, "bpx_volume": Volume, "bpx_outputs": Outputs,
               "bpx_track_options": abi.TrackOptions, "bpx_track_volume": abi.TrackVolume}[t]
        assert getattr(cls, m).offset == v, (t, m)


def test_defaults_and_counts(libbpx):
    o = Options()
    libbpx.bpx_options_default(C.byref(o))
    ref = Options.make()
    for name, _ in Options._fields_:
        if name == "reserved":
            continue
        assert getattr(o, name) == pytest.approx(getattr(ref, name)), name
    assert o.seed == 8665904 and o.njumps == 1250 and o.nburn == 1000 and o.sampleevery == 25
    assert libbpx.bpx_abi_version() == 1
    for model, nf, f0, want in [(1, 1, 0, 5), (1, 2, 1, 9), (2, 3, 0, 12), (2, 3, 1, 13), (3, 2, 1, 10)]:
        q = Options.make(model=model, nfibres=nf, f0=f0)
        assert libbpx.bpx_nparams_fit(C.byref(q)) == want == q.nparams_fit
    assert libbpx.bpx_nsamples(C.byref(Options.make())) == 50
    assert libbpx.bpx_max_ndir() >= 288


def test_host_argument_checks_reject_bad_input(libbpx):
    """Validation runs before any device call, so these need no GPU."""
    libbpx.bpx_last_error.restype = C.c_char_p
    vol = Volume()
    vol.nvox, vol.ndir = 10, 64
    bad = Options.make(model=5)
    assert libbpx.bpx_fit_dev(C.byref(bad), C.byref(vol), None, None, None, None) == abi.BPX_ERR_INVALID_ARG
    assert b"model" in libbpx.bpx_last_error()
    bad = Options.make(nfibres=4)
    assert libbpx.bpx_mcmc_dev(C.byref(bad), C.byref(vol), None, None, None, None, None) == abi.BPX_ERR_INVALID_ARG
    ok = Options.make()
    vol.ndir = 4000
    assert libbpx.bpx_fit_dev(C.byref(ok), C.byref(vol), None, None, None, None) == abi.BPX_ERR_UNSUPPORTED
    vol.ndir = 64
    assert libbpx.bpx_fit_dev(C.byref(ok), C.byref(vol), None, None, None, None) == abi.BPX_ERR_INVALID_ARG  # NULL data
    bad = Options.make(sampleevery=0)
    assert libbpx.bpx_finish_dev(C.byref(bad), 3, None, None, None) == abi.BPX_ERR_INVALID_ARG
    assert libbpx.bpx_prepare_data_dev(-1, 64, None, None) == abi.BPX_ERR_INVALID_ARG
    # stretches of the chain: the iteration range, and a state when not starting at iteration 0
    ok_s = Options.make(nburn=10, njumps=20)
    st = libbpx.bpx_mcmc_stretch_dev
    assert st(C.byref(ok_s), C.byref(vol), None, None, None, None, None, 0, 31, 0, None, None, None, None, None,
              None) == abi.BPX_ERR_INVALID_ARG
    assert b"it_begin" in libbpx.bpx_last_error()
    assert st(C.byref(ok_s), C.byref(vol), None, None, None, None, None, 5, 5, 0, None, None, None, None, None,
              None) == abi.BPX_ERR_INVALID_ARG
    assert st(C.byref(ok_s), C.byref(vol), None, None, None, None, None, 5, 30, 0, None, None, None, None, None,
              None) == abi.BPX_ERR_INVALID_ARG
    assert b"state_in" in libbpx.bpx_last_error()
    # tracking: options, grid and buffers are checked first
    t = abi.TrackOptions.make()
    tv = abi.TrackVolume()
    tv.nx, tv.ny, tv.nz, tv.dx, tv.dy, tv.dz, tv.nfib, tv.nsamples = 8, 8, 8, 2.0, 2.0, 2.0, 3, 50
    pt = libbpx.bpx_probtrack_dev
    assert pt(C.byref(t), C.byref(tv), 1, None, None, None, None) == abi.BPX_ERR_INVALID_ARG  # NULL buffers
    assert b"NULL" in libbpx.bpx_last_error()
    tv.nwaypoints = 33
    assert pt(C.byref(t), C.byref(tv), 1, None, None, None, None) == abi.BPX_ERR_INVALID_ARG
    assert b"nwaypoints" in libbpx.bpx_last_error()
    tv.nwaypoints, tv.nsamples = 0, (1 << 20) + 1
    assert pt(C.byref(t), C.byref(tv), 1, None, None, None, None) == abi.BPX_ERR_UNSUPPORTED
    tv.nsamples, tv.nfib = 50, 4
    assert pt(C.byref(t), C.byref(tv), 1, None, None, None, None) == abi.BPX_ERR_INVALID_ARG
    tv.nfib = 3
    assert pt(C.byref(abi.TrackOptions.make(nsteps=1)), C.byref(tv), 1, None, None, None, None) == abi.BPX_ERR_INVALID_ARG
    assert pt(C.byref(t), C.byref(tv), 0, None, None, None, None) == abi.BPX_OK  # no seeds: nothing to do
    # empty volumes are valid and do nothing
    vol.nvox = 0
    assert libbpx.bpx_fit_dev(C.byref(ok), C.byref(vol), None, None, None, None) == abi.BPX_OK


def test_layout_table(libbpx):
    n = libbpx.bpx_mcmc_layouts(None, None, 0)
    tpv = (C.c_int32 * n)()
    mpl = (C.c_int32 * n)()
    libbpx.bpx_mcmc_layouts(tpv, mpl, n)
    caps = [t * m for t, m in zip(tpv, mpl)]
    assert all(t in (4, 8, 16, 32) for t in tpv)
    assert max(caps) >= libbpx.bpx_max_ndir()
