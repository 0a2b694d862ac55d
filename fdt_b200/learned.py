"""The learned form: training the initialiser network on the GPU and running the learned pipeline.

Training data are voxels the forward model generates on the GPU (bpx_synth_dev), labelled with
their LM fits (bpx_fit_dev) and with the proposal widths a plain chain adapts to by the end of its
burn-in (bpx_mcmc_ex_dev).  Every step of training -- forward, loss, backward, Adam -- runs in the
library's own kernels (tcgen05 GEMMs with fused epilogues); PyTorch only holds device memory and
gathers the mini-batches.

The trained network replaces the LM initialiser and sets per-voxel proposal widths (which the
chain then adapts, or keeps frozen), so the chain needs a shorter burn-in; the plain LM-initialised
chain with the full burn-in stays the fallback and the comparator for its accuracy (posterior_study and
study_report measure both against it and against a long chain).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
import os

import numpy as np

from . import lib
from .abi import Options

WIDTH, HIDDEN, NOUT = 256, 4, 32
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")


def nin(ndir: int) -> int:
    return (ndir + 7) // 8 * 8


def geometry(ndir: int):
    k = [nin(ndir)] + [WIDTH] * HIDDEN
    n = [WIDTH] * HIDDEN + [NOUT]
    woff, boff, o = [], [], 0
    for l in range(HIDDEN + 1):
        woff.append(o)
        o += k[l] * n[l]
        boff.append(o)
        o += n[l]
    return k, n, woff, boff, o


def init_params(ndir: int, seed: int = 0) -> np.ndarray:
    """He-normal hidden weights, small output weights, zero biases (FP32 flat vector)."""
    rng = np.random.default_rng(seed)
    k, n, woff, boff, total = geometry(ndir)
    p = np.zeros(total, np.float32)
    for l in range(HIDDEN + 1):
        std = math.sqrt(2.0 / k[l]) if l < HIDDEN else 0.1 * math.sqrt(1.0 / k[l])
        p[woff[l] : woff[l] + n[l] * k[l]] = rng.normal(0.0, std, n[l] * k[l])
    return p


@dataclasses.dataclass
class TrainingSet:
    x: object  # [n][nin] bf16 device tensor
    targets: object  # [n][32] float32 device tensor
    tweights: object  # [n][32] float32 device tensor
    ndir: int

    @property
    def n(self) -> int:
        return int(self.x.shape[0])


MEAN_LABEL_SAMPLES = 10


def label_options(opts: Options, samples: int = 1, burnin: int | None = None, every: int | None = None) -> Options:
    """Options of the labelling chain: the plain chain's burn-in (or `burnin` iterations), then
    `samples` samples recorded every sampleevery (or `every`) iterations."""
    o = Options.make(**{f: getattr(opts, f) for f, _ in Options._fields_ if f != "reserved"})
    if burnin is not None:
        o.nburn = burnin
    if every is not None:
        o.sampleevery = every
    o.njumps = o.sampleevery * samples
    return o


def state_mean_from_records(opts: Options, rec):
    """(params [n][P] in the fit layout, tau [n]) of the posterior mean over the recorded samples:
    means of the scalars and fractions; for each fibre the principal eigenvector of the mean dyadic
    tensor (v v^T over samples, so the sign of v does not matter), as angles with theta in [0, pi]."""
    import torch

    r = rec.double()
    m = r.mean(1)  # [rows][n]
    K = opts.nfibres
    cols = [m[5], m[0]] + ([m[3]] if opts.model >= 2 else [])
    for k in range(K):
        th, ph = r[6 + 3 * k], r[7 + 3 * k]  # [ns][n]
        v = torch.stack([torch.sin(th) * torch.cos(ph), torch.sin(th) * torch.sin(ph), torch.cos(th)], -1)
        dyad = torch.nan_to_num(torch.einsum("sni,snj->nij", v, v) / v.shape[0], nan=0.0, posinf=0.0, neginf=0.0)
        _, vecs = torch.linalg.eigh(dyad.cpu())  # host LAPACK: the batched device solver rejects large batches
        e = vecs[..., 2].to(dyad.device)  # largest eigenvalue's vector
        e = torch.where((e[:, 2:3] < 0), -e, e)
        cols += [m[8 + 3 * k], torch.arccos(e[:, 2].clamp(-1.0, 1.0)), torch.atan2(e[:, 1], e[:, 0])]
    if opts.f0:
        cols.append(m[1])
    return torch.stack(cols, 1).float().contiguous(), m[2].float().contiguous()


def state_from_record(opts: Options, rec, sample: int = 0):
    """(params [n][P] in the fit layout, tau [n]) of one recorded chain state."""
    import torch

    r = rec[:, sample, :]
    K = opts.nfibres
    cols = [r[5], r[0]] + ([r[3]] if opts.model >= 2 else [])
    for k in range(K):
        cols += [r[8 + 3 * k], r[6 + 3 * k], r[7 + 3 * k]]
    if opts.f0:
        cols.append(r[1])
    return torch.stack(cols, 1).contiguous(), r[2].contiguous()


def make_training_set(opts: Options, bvecs: np.ndarray, bvals: np.ndarray, n: int, seed: int = 1,
                      snr=(10.0, 40.0), chunk: int = 131072, widths: bool = True,
                      state_labels: str = "mean", label_samples: int = MEAN_LABEL_SAMPLES,
                      label_burnin: int | None = None, label_every: int | None = None) -> TrainingSet:
    """n forward-model voxels (SNR ~ U(snr)) with their labels.  The plain chain is run from each
    voxel's LM fit through its full burn-in; its proposal widths at that point are the width
    labels, and the state labels are either that chain state (state_labels="chain": the state the
    LM-initialised chain reaches, which is where a chain with frozen widths must start), the
    posterior mean over `label_samples` samples recorded after the burn-in ("mean"; with the plain
    chain's 50 samples, the plain form's own posterior means; widths then
    taken at the end of that recording) or the LM fit itself ("lm").  label_burnin / label_every
    replace the labelling chain's burn-in and sample spacing (default: the plain chain's)."""
    import torch

    L = lib.load()
    ndir = bvals.shape[0]
    bv, bl = lib.to_device(bvecs), lib.to_device(bvals)
    x = torch.empty((n, nin(ndir)), device="cuda", dtype=torch.bfloat16)
    t = torch.empty((n, NOUT), device="cuda", dtype=torch.float32)
    w = torch.empty((n, NOUT), device="cuda", dtype=torch.float32)
    lo = label_options(opts, label_samples if state_labels == "mean" else 1, label_burnin, label_every)
    stream = lib._stream(torch)
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        data, _ = lib.synth(opts.model, opts.nfibres, m, bv, bl, seed, snr, voxel_offset=s)
        if opts.rician:
            lib.prepare_data(data)
        params, tau, status = lib.fit(opts, data, bv, bl)
        s0hat = torch.empty(m, device="cuda", dtype=torch.float32)
        vol = lib.make_volume(data, bv, bl)
        lib._check(L.bpx_mlp_features_dev(C.byref(vol), 0, lib._ptr(x[s : s + m]), lib._ptr(s0hat), stream),
                   "bpx_mlp_features_dev")
        props = None
        if widths or state_labels in ("chain", "mean"):
            rec, props = lib.mcmc_ex(lo, data, bv, bl, params, tau if opts.rician else None, want_props=True,
                                     voxel_offset=s, status=status)
            if state_labels == "chain":
                params, tau = state_from_record(opts, rec)
            elif state_labels == "mean":
                params, tau = state_mean_from_records(opts, rec)
            if not widths:
                props = None
        lib._check(L.bpx_mlp_targets_dev(C.byref(opts), m, lib._ptr(params), lib._ptr(tau if opts.rician else None),
                                         lib._ptr(props), lib._ptr(s0hat), lib._ptr(t[s : s + m]),
                                         lib._ptr(w[s : s + m]), stream), "bpx_mlp_targets_dev")
        bad = (status & 5) != 0  # non-finite data, or a chain that met a non-finite energy: no targets
        if bool(bad.any()):
            w[s : s + m][bad] = 0.0
    torch.cuda.synchronize()
    return TrainingSet(x, t, w, ndir)


def output_bias_from_targets(ts: TrainingSet, params: np.ndarray) -> np.ndarray:
    """Set the output layer's bias to the weighted mean target (a better start than zero)."""
    k, n, woff, boff, total = geometry(ts.ndir)
    t, w = ts.targets, ts.tweights
    mean = ((t * w).sum(0) / w.sum(0).clamp_min(1e-12)).cpu().numpy()
    mean[3:12] = 0.0
    p = params.copy()
    p[boff[HIDDEN] : boff[HIDDEN] + NOUT] = mean
    return p


def train(ts: TrainingSet, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0,
          params: np.ndarray | None = None, log_every: int = 0):
    """Adam with a cosine learning-rate decay over `steps` mini-batches.  Returns (params, losses)."""
    import torch

    L = lib.load()
    stream = lib._stream(torch)
    p0 = params if params is not None else output_bias_from_targets(ts, init_params(ts.ndir, seed))
    p = torch.from_numpy(np.ascontiguousarray(p0, np.float32)).cuda()
    g = torch.zeros_like(p)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    loss = torch.zeros(1, device="cuda", dtype=torch.float32)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    perm = torch.randperm(ts.n, device="cuda", generator=gen)
    pos = 0
    losses = []
    for step in range(1, steps + 1):
        if pos + batch > ts.n:
            perm = torch.randperm(ts.n, device="cuda", generator=gen)
            pos = 0
        idx = perm[pos : pos + batch]
        pos += batch
        xb, tb, wb = ts.x[idx].contiguous(), ts.targets[idx].contiguous(), ts.tweights[idx].contiguous()
        bs = int(xb.shape[0])
        lib._check(L.bpx_mlp_train_step_dev(ts.ndir, lib._ptr(p), lib._ptr(g), bs, lib._ptr(xb), lib._ptr(tb),
                                            lib._ptr(wb), lib._ptr(loss), stream), "bpx_mlp_train_step_dev")
        lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * (step - 1) / max(1, steps)))
        lib._check(L.bpx_mlp_adam_dev(p.numel(), lib._ptr(p), lib._ptr(g), lib._ptr(m), lib._ptr(v), lr_t, 0.9, 0.999,
                                      1e-8, step, stream), "bpx_mlp_adam_dev")
        if log_every and (step % log_every == 0 or step == 1 or step == steps):
            losses.append((step, float(loss.item())))
    torch.cuda.synchronize()
    if lib.poll_error() != 0:
        raise lib.BpxError("a tensor-core kernel gave up waiting during training")
    return p.cpu().numpy(), losses


def forward(params, ndir: int, x):
    """Network outputs [n][32] (device) for bf16 inputs x [n][nin] (device)."""
    import torch

    n = int(x.shape[0])
    out = torch.empty((n, NOUT), device="cuda", dtype=torch.float32)
    p = params if hasattr(params, "data_ptr") else torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda()
    lib._check(lib.load().bpx_mlp_forward_dev(ndir, lib._ptr(p), n, lib._ptr(x), lib._ptr(out), lib._stream(torch)),
               "bpx_mlp_forward_dev")
    return out


def features(data, bvecs, bvals):
    """(x [n][nin] bf16, s0hat [n]) on the device."""
    import torch

    n, ndir = int(data.shape[0]), int(data.shape[1])
    x = torch.empty((n, nin(ndir)), device="cuda", dtype=torch.bfloat16)
    s0 = torch.empty(n, device="cuda", dtype=torch.float32)
    vol = lib.make_volume(data, bvecs, bvals)
    lib._check(lib.load().bpx_mlp_features_dev(C.byref(vol), 0, lib._ptr(x), lib._ptr(s0), lib._stream(torch)),
               "bpx_mlp_features_dev")
    return x, s0


def decode(opts: Options, out, s0hat):
    """(params [n][P], tau [n], props [6+3K][n], status [n]) starting state from network outputs."""
    import torch

    n = int(out.shape[0])
    params = torch.empty((n, opts.nparams_fit), device="cuda", dtype=torch.float32)
    tau = torch.empty(n, device="cuda", dtype=torch.float32)
    props = torch.empty((6 + 3 * opts.nfibres, n), device="cuda", dtype=torch.float32)
    status = torch.empty(n, device="cuda", dtype=torch.int32)
    lib._check(lib.load().bpx_mlp_decode_dev(C.byref(opts), n, lib._ptr(out), lib._ptr(s0hat), lib._ptr(params),
                                             lib._ptr(tau), lib._ptr(props), lib._ptr(status), lib._stream(torch)),
               "bpx_mlp_decode_dev")
    return params, tau, props, status


def xfibres_learned(opts: Options, data, bvecs, bvals, params, freeze: int = 2, out=None):
    """The learned pipeline on device tensors (bpx_xfibres_learned_dev); returns the output dict.
    freeze: 0 adapt the network's widths throughout, 1 never, 2 during the burn-in only."""
    import torch

    n = int(data.shape[0])
    t, o = out if out is not None else lib.alloc_outputs(opts, n)
    p = params if hasattr(params, "data_ptr") else torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda()
    vol = lib.make_volume(data, bvecs, bvals)
    lib._check(lib.load().bpx_xfibres_learned_dev(C.byref(opts), C.byref(vol), lib._ptr(p), int(freeze), C.byref(o),
                                                  lib._stream(torch)), "bpx_xfibres_learned_dev")
    return t


def save(path: str, params: np.ndarray, **meta) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez_compressed(path, params=np.asarray(params, np.float32), **{k: np.asarray(v) for k, v in meta.items()})


def load_weights(path: str):
    z = np.load(path)
    return z["params"], {k: z[k] for k in z.files if k != "params"}


def posterior_study(opts: Options, data, bvecs, bvals, mlp_params, R: int = 8, seed: int = 100,
                    gold: bool = True) -> dict:
    """Chain sets of the learned form and its comparators on the same voxels, R chains per voxel
    (independent random streams: the volume is replicated R times, so every copy of a voxel has its
    own RNG key), for agreement.compare:

      plain           LM start, the reference's widths, opts.nburn (1000): the comparator for the others
      plain_other_seed   the same with another seed (yardstick of plain-vs-plain agreement)
      learned         network start state and widths, burn-in 200, widths adapting (freeze 0)
      learned_frozen  the same, widths frozen after the burn-in (freeze 2)
      lm_burnin200    the method without the network at the learned form's burn-in: LM start,
                      the reference's widths, burn-in 200
      gold            LM start, burn-in 5000, 12500 jumps recorded every 125: a long chain whose
                      posterior means carry less start dependence and Monte-Carlo error

    data: [n][ndir] device tensor (cleaned under --rician); bvecs/bvals device tensors; mlp_params the
    network (host or device).  Returns {form: agreement.ChainSet}."""
    import torch

    from . import agreement

    n = int(data.shape[0])
    K = opts.nfibres
    dR = data.repeat(R, 1).contiguous()
    params, tau, _ = lib.fit(opts, data, bvecs, bvals)
    pR, tR = params.repeat(R, 1).contiguous(), tau.repeat(R).contiguous()
    tau_arg = tR if opts.rician else None
    x, s0 = features(data, bvecs, bvals)
    lo = Options.make(**{f: getattr(opts, f) for f, _ in Options._fields_ if f != "reserved"})
    lo.nburn = 200
    out = forward(mlp_params, int(data.shape[1]), x)
    pn, tn, props, _ = decode(lo, out, s0)
    pnR, tnR, propsR = pn.repeat(R, 1).contiguous(), tn.repeat(R).contiguous(), props.repeat(1, R).contiguous()

    def with_(**kw):
        o = Options.make(**{f: getattr(opts, f) for f, _ in Options._fields_ if f != "reserved"})
        for k, v in kw.items():
            setattr(o, k, v)
        return o

    def chains(o, p, t, pin=None, freeze=0):
        rec, _ = lib.mcmc_ex(o, dR, bvecs, bvals, p, t, props_in=pin, freeze=freeze)
        torch.cuda.synchronize()
        return agreement.ChainSet(rec.cpu().numpy(), K, R)

    sets = {
        "plain": chains(with_(seed=seed), pR, tau_arg),
        "plain_other_seed": chains(with_(seed=seed + 7), pR, tau_arg),
        "learned": chains(with_(seed=seed + 1, nburn=200), pnR, tnR if opts.rician else None, propsR, 0),
        "learned_frozen": chains(with_(seed=seed + 1, nburn=200), pnR, tnR if opts.rician else None, propsR, 2),
        "lm_burnin200": chains(with_(seed=seed + 2, nburn=200), pR, tau_arg),
    }
    if gold:
        sets["gold"] = chains(with_(seed=seed + 3, nburn=5000, njumps=12500, sampleevery=125), pR, tau_arg)
    return sets


def study_report(sets: dict, truth=None) -> dict:
    """Agreement of each form with the plain chain and with the long (gold) chain; with the ground
    truth of synthetic voxels (truth: synth.Truth of the same voxels), each form's errors against it."""
    from . import agreement

    rep = {"chains_per_voxel": int(sets["plain"].R), "voxels": int(sets["plain"].nvox),
           "vs_plain": {k: agreement.compare(sets[k], sets["plain"])
                        for k in ("plain_other_seed", "learned", "learned_frozen", "lm_burnin200") if k in sets}}
    if "gold" in sets:
        rep["vs_gold"] = {k: agreement.compare(sets[k], sets["gold"])
                          for k in ("plain", "learned", "learned_frozen", "lm_burnin200") if k in sets}
    if truth is not None:
        n = int(sets["plain"].nvox)
        rep["vs_truth"] = {k: agreement.truth_errors(v, truth.f[:n], truth.v[:n], truth.d[:n]) for k, v in sets.items()}
    return rep


# chain options of the configurations a network is trained for
OPTION_SETS = {
    "whole_brain": dict(model=2, nfibres=3, rician=1, f0=1, ardf0=1),  # the whole-brain configuration
    "c1": dict(model=2, nfibres=3),  # the multi-shell configuration: no Rician noise model, no f0
}
DEFAULT_OPTIONS = {"whole_brain": "whole_brain", "multishell": "c1"}

PROTOCOLS = {
    "whole_brain": lambda synth: synth.three_shell(18, 90),
    "multishell": lambda synth: synth.three_shell(9, 90),
}


def default_weights_path(protocol: str) -> str:
    return os.path.join(WEIGHTS_DIR, f"initialiser_model2_k3_{protocol}.npz")


def main(argv=None) -> None:
    """Train the initialiser for a protocol on the GPU and save it:

        python -m fdt_b200.learned --protocol whole_brain --n 10485760 --steps 40000
    """
    import argparse
    import time

    import torch

    from . import synth

    ap = argparse.ArgumentParser()
    ap.add_argument("--protocol", default="whole_brain", choices=sorted(PROTOCOLS))
    ap.add_argument("--options", default=None, choices=sorted(OPTION_SETS),
                    help="chain options the network is trained for (default: the protocol's configuration)")
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=None)
    ap.add_argument("--eval", type=int, default=8192, help="held-out voxels for the learned-vs-plain check")
    ap.add_argument("--labels", default="mean", choices=["chain", "mean", "lm"])
    ap.add_argument("--label-samples", type=int, default=MEAN_LABEL_SAMPLES,
                    help="--labels mean: samples (every sampleevery iterations) the labels average")
    ap.add_argument("--label-burnin", type=int, default=None,
                    help="burn-in of the labelling chain (default: the plain chain's)")
    ap.add_argument("--label-every", type=int, default=None,
                    help="sample spacing of the labelling chain (default: the plain chain's)")
    ap.add_argument("--weights", default=None, help="evaluate these weights instead of training")
    ap.add_argument("--time-forward", type=int, default=0, metavar="ROWS",
                    help="only time the network's forward pass on ROWS inputs (CUDA events) and exit")
    a = ap.parse_args(argv)
    prot = PROTOCOLS[a.protocol](synth)
    if a.time_forward:
        import json

        params, _ = load_weights(a.weights or default_weights_path(a.protocol))
        g = torch.Generator(device="cuda").manual_seed(a.seed)
        x = (1.2 * torch.rand((a.time_forward, nin(prot.ndir)), device="cuda", generator=g)).to(torch.bfloat16)
        p = torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda()
        for _ in range(3):
            forward(p, prot.ndir, x)
        ts = []
        for _ in range(20):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            forward(p, prot.ndir, x)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        if lib.poll_error() != 0:
            raise SystemExit("a tensor-core kernel reported a timed-out wait")
        print(json.dumps({"rows": a.time_forward, "layers": 5, "forward_ms_min": min(ts),
                          "forward_ms_median": float(np.median(ts))}))
        return
    oname = a.options or DEFAULT_OPTIONS[a.protocol]
    opts = Options.make(**OPTION_SETS[oname])
    if a.weights:
        params, _ = load_weights(a.weights)
    else:
        t0 = time.time()
        ts = make_training_set(opts, prot.bvecs, prot.bvals, a.n, seed=a.seed, state_labels=a.labels,
                               label_samples=a.label_samples, label_burnin=a.label_burnin,
                               label_every=a.label_every)
        t1 = time.time()
        params, losses = train(ts, a.steps, a.batch, a.lr, seed=a.seed, log_every=max(1, a.steps // 20))
        t2 = time.time()
        print(f"training set {a.n} voxels in {t1 - t0:.1f} s; {a.steps} steps in {t2 - t1:.1f} s")
        for s, l in losses:
            print(f"  step {s:6d} loss {l:.5f}")
        out = a.out or default_weights_path(a.protocol)
        save(out, params, ndir=prot.ndir, model=2, nfibres=3, protocol=a.protocol, n_train=a.n, steps=a.steps,
             seed=a.seed, labels=a.labels, label_samples=a.label_samples,
             label_burnin=opts.nburn if a.label_burnin is None else a.label_burnin,
             label_every=opts.sampleevery if a.label_every is None else a.label_every,
             bvals=prot.bvals, bvecs=prot.bvecs,
             options=oname,
             rician=opts.rician, f0=opts.f0, ardf0=opts.ardf0)
        print("saved", out)
        del ts
        torch.cuda.empty_cache()
    if a.eval:
        import json

        data, _ = synth.make_volume(a.eval, prot, 3, True, 25.0, seed=a.seed + 1000)
        bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
        d = lib.to_device(data)
        if opts.rician:
            lib.prepare_data(d)
        print(json.dumps(study_report(posterior_study(opts, d, bv, bl, params, R=8))))


if __name__ == "__main__":
    main()
