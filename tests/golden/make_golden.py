"""Golden fixtures of the FP64 oracle (oracle/, test infrastructure) on seeded synthetic voxels.

    python tests/golden/make_golden.py        # rewrites tests/golden/*.npz

For each case: the data (float32 [nvox][M], stored so that the fixtures do not depend on the
synthetic generator), the protocol, the oracle's LM fits, tau and status, a short chain on the
Philox stream the GPU kernel shares (records of every iteration) and the finished outputs of a
standard-length chain.  The reference ships no golden vectors for this path; the oracle is pinned
analytically (tests/test_oracle.py), and these files freeze its outputs so that any change to it
shows up as a diff (tests/test_golden.py) and the CUDA path is checked against committed numbers
(tests/test_gpu_golden.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fdt_b200 import synth  # noqa: E402
from fdt_b200.abi import Options  # noqa: E402

CASES = {
    "m1_k2": dict(opts=dict(model=1, nfibres=2), prot=("single_shell_64",), nvox=32, snr=20.0, seed=701),
    "m2_k3_rician_f0": dict(opts=dict(model=2, nfibres=3, rician=1, f0=1, ardf0=1), prot=("three_shell", 18, 90),
                            nvox=16, snr=25.0, seed=702),
    "m3_k2_rician": dict(opts=dict(model=3, nfibres=2, rician=1), prot=("three_shell", 9, 90), nvox=16, snr=25.0,
                         seed=703),
}
SHORT = dict(nburn=0, njumps=30, sampleevery=1)      # chain compared step by step
FULL = dict(nburn=100, njumps=200, sampleevery=10)   # chain whose finished outputs are stored


def protocol(spec):
    return synth.single_shell_64() if spec[0] == "single_shell_64" else synth.three_shell(spec[1], spec[2])


def make(name, c, O):
    prot = protocol(c["prot"])
    o = Options.make(**c["opts"])
    gamma = o.model >= 2
    y, _ = synth.make_volume(c["nvox"], prot, o.nfibres, gamma, c["snr"], seed=c["seed"])
    if o.rician:
        y = O.prepare_data(y)
    y = np.ascontiguousarray(y, np.float32)
    params, tau, status = O.fit(o, y, prot.bvecs, prot.bvals, nthreads=1)
    os_ = Options.make(**c["opts"], **SHORT)
    rec_short = O.mcmc(os_, y, prot.bvecs, prot.bvals, params, tau, nthreads=1)
    of = Options.make(**c["opts"], **FULL)
    rec_full = O.mcmc(of, y, prot.bvecs, prot.bvals, params, tau, nthreads=1)
    fin = O.finish(of, rec_full)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), y=y, bvecs=prot.bvecs, bvals=prot.bvals,
                        params=params, tau=tau, status=status, rec_short=rec_short,
                        **{"fin_" + k: v for k, v in fin.items()})


def main():
    from oracle import oracle as O

    O.build()
    for name, c in CASES.items():
        make(name, c, O)
        print("wrote", name)


if __name__ == "__main__":
    main()
