#!/usr/bin/env python
"""Benchmark of the bedpostx per-voxel path on B200 (and of the CPU baseline).

Workload (the whole-brain configuration): model 2 (Gamma-distributed diffusivity), 3 fibres,
--rician --f0 --ardf0, 288 measurements (18 b=0 + 90 directions at b=1000/2000/3000),
burn-in 1000, 1250 jumps, sample every 25, seeded synthetic voxels with SNR 25 generated from the
forward model (no dataset exists for this path).  One step = the whole path over one chunk of voxels already resident in HBM: for the plain form
Rician data clean-up, LM fits + tau, MCMC (burn-in 1000) and sample finishing; for the learned form
the data clean-up, the initialiser network (features, 5 tensor-core layers, decode), MCMC from the
network's state and widths (burn-in 200) and finishing.  The headline value is the learned form's
voxels/s; the plain form is timed beside it on the same chunks, and the accuracy block compares
their posteriors on the same voxels (with a second plain run at another seed as the yardstick).  The chunk (131072 voxels x 288 x 4 B = 151 MB) is larger than the 126 MB L2 and
the L2 is also flushed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank processes its own chunks (weak scaling, no data-path collective); the
step time is the max over ranks.  `--impl reference` times the CPU implementation of the path
(the FP64 oracle port, OpenMP over voxels, all host threads) on a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from fdt_b200 import synth  # noqa: E402
from fdt_b200.abi import Options  # noqa: E402

METRIC = "voxels/s, learned-init vs plain MCMC on 1 B200 at matched dyad error"
WORKLOAD = ("whole-brain: model 2, 3 fibres, rician+f0+ardf0, 288 measurements, burnin 1000, njumps 1250, "
            "sampleevery 25, plain LM-initialised chain")
WORKLOAD_LEARNED = ("whole-brain: model 2, 3 fibres, rician+f0+ardf0, 288 measurements, njumps 1250, sampleevery 25; "
                    "learned-init batched form (network start state and proposal widths, burnin 200, one CUDA-graph "
                    "launch per step) against the plain LM-initialised chain (burnin 1000)")


# DRAM bytes (read + write) of one mcmc_kernel launch on the whole-brain workload at this bench's
# launch size, from an ncu capture of a 131072-voxel launch (the learned chain: 1450 iterations,
# 50 samples): 278,176,512 B read + 420,939,776 B written, 5334 B per voxel against 4224 B of
# inputs, start state and samples.  The chain state stays on chip, so the traffic does not grow
# with iterations; per voxel it grows with the launch size (4465 B at 65536 voxels), since the
# one-word record stores of neighbouring voxels reach L2 further apart in time.
MCMC_DRAM_BYTES_LAUNCH = 278176512 + 420939776
MCMC_DRAM_LAUNCH_VOXELS = 131072


def whole_brain_options() -> Options:
    return Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=1000, njumps=1250, sampleevery=25)


def _mcmc_terms(o: Options, ndir: int) -> tuple[int, int, int, int, int]:
    """(J, L, T, K, M): iterations, likelihood evaluations and signal-term updates per iteration."""
    K, M = o.nfibres, ndir
    J = o.nburn + o.njumps
    L = (1 if o.f0 else 0) + (1 if o.rician else 0) + 1 + (1 if o.model >= 2 else 0) + (1 if o.model == 3 else 0) \
        + 1 + 3 * K
    T = (K + 1) * M + (K + 1) * M * (1 if o.model == 2 else 0) + M * (1 if o.model == 3 else 0) \
        + K * M * (1 if o.model == 3 else 0) + 2 * K * M
    return J, L, T, K, M


def mcmc_work_canonical(o: Options, ndir: int) -> tuple[float, float]:
    """Canonical algorithmic MUFU and FP32-FMA operations of one voxel's chain: the path's minimal
    formulation with the reference's operations (model-2 signal terms rcp + log2 + exp2, Rician
    likelihood terms log2 + rsqrt; FMA per signal term 6, per likelihood term K+4, +12 Rician)."""
    J, L, T, K, M = _mcmc_terms(o, ndir)
    c_sig = 3 if o.model == 2 else 1
    c_lik = 2 if o.rician else 0
    mufu = J * (T * c_sig + L * M * c_lik)
    fp32 = J * (T * 6 + L * M * (K + 4 + (12 if o.rician else 0)))
    return float(mufu), float(fp32)


def mcmc_work_per_voxel(o: Options, ndir: int) -> tuple[float, float]:
    """MUFU and FP32 operations of one voxel's chain as this kernel formulates it.

    MUFU per signal term: 1 (models 1/3: exp2) or 2 (model 2: log2 + exp2 with the per-proposal
    Gamma scale hoisted); per Rician likelihood term 1.2 (an rsqrt, and one log2 per product of five
    Bessel factors), Gaussian 0.  FP32 operations (an FMA counts as one) per signal term 6, per
    likelihood term K+4 (prediction, residual, weighted square) plus 19 when Rician (the two log I0
    polynomials of degrees 6 and 5, their arguments z, z^2, 1/z and the product/sum accumulations).
    """
    J, L, T, K, M = _mcmc_terms(o, ndir)
    c_sig = 2 if o.model == 2 else 1
    c_lik = 1.2 if o.rician else 0.0
    mufu = J * (T * c_sig + L * M * c_lik)
    fp32 = J * (T * 6 + L * M * (K + 4 + (19 if o.rician else 0)))
    return float(mufu), float(fp32)


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(p))
    except (OSError, ValueError):
        return {}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, world, rank):
    """CPU implementation of the path (the FP64 oracle port), all host threads, bounded samples."""
    if rank != 0:
        return
    from oracle import oracle as O

    o = whole_brain_options()
    prot = synth.three_shell(18, 90)
    cores = os.cpu_count() or 1
    per_step = args.ref_voxels or max(8, 2 * cores)
    times = []
    for step in range(args.warmup + args.steps):
        y, _ = synth.make_volume(per_step, prot, 3, True, 25.0, seed=1000 + step)
        t0 = time.perf_counter()
        y = O.prepare_data(y)
        p, tau, st = O.fit(o, y, prot.bvecs, prot.bvals, nthreads=cores)
        rec = O.mcmc(o, y, prot.bvecs, prot.bvals, p, tau, voxel_offset=step * per_step, nthreads=cores)
        O.finish(o, rec)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
    tot = sum(times)
    v = per_step * len(times) / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "voxels/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "voxels_per_step": per_step, "host_threads": cores},
        "cpu_baseline": {"value": v, "unit": "voxels/s", "cores": cores, "kind": "port",
                         "sample": f"{per_step} voxels per step of the whole-brain workload, full chain"},
        "e2e": {"value": v, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(seconds: float = 12.0) -> dict:
    from oracle import oracle as O

    o = whole_brain_options()
    prot = synth.three_shell(18, 90)
    cores = os.cpu_count() or 1
    n = max(4, cores)
    done, t_all, step = 0, 0.0, 0
    while t_all < seconds and step < 64:
        y, _ = synth.make_volume(n, prot, 3, True, 25.0, seed=5000 + step)
        t0 = time.perf_counter()
        y = O.prepare_data(y)
        p, tau, st = O.fit(o, y, prot.bvecs, prot.bvals, nthreads=cores)
        rec = O.mcmc(o, y, prot.bvecs, prot.bvals, p, tau, nthreads=cores)
        O.finish(o, rec)
        t_all += time.perf_counter() - t0
        done += n
        step += 1
    return {"value": done / t_all, "unit": "voxels/s", "cores": cores, "kind": "port",
            "sample": f"{done} voxels of the whole-brain workload (full chain), {t_all:.1f} s on {cores} threads"}


def batched_workload(scale: float, seed: int = 31):
    """Config C2: 16 volumes, voxel counts log-uniform in [5k, 300k] (times `scale`), measurement
    counts from {33, 65, 129, 279} (the 279-volume three-shell scheme truncated), models 1 and 2
    mixed across volumes, fibre count 1..3 per voxel, SNR ~ U(10, 40).  Returns a list of items
    (host arrays), one per (volume, fibre count)."""
    rng = np.random.default_rng(seed)
    items = []
    for v in range(16):
        n = int(round(np.exp(rng.uniform(np.log(5000), np.log(300000))) * scale))
        M = int(rng.choice([33, 65, 129, 279]))
        model = int(rng.choice([1, 2]))
        prot = synth.truncated_three_shell(M)
        ks = rng.integers(1, 4, size=n)
        off = 0
        for K in (1, 2, 3):
            m = int((ks == K).sum())
            if m == 0:
                continue
            snr = rng.uniform(10.0, 40.0, size=m)
            y, _ = synth.make_volume(m, prot, K, model == 2, snr, seed=seed * 1000 + 10 * v + K)
            items.append(dict(host=y, prot=prot, model=model, nfibres=K, volume=v, voxel_offset=off))
            off += m
    return items


def batched_record(scale: float, steps: int, warmup: int) -> dict:
    """Times the batched form (one graph launch over all volumes of config C2 at voxel-count scale
    `scale`) against the same items run one after another through bpx_xfibres_dev with the default
    layouts.  Returns the measurement as a dict (the --workload batched line, or the C2 sub-record
    of the default line)."""
    import torch

    from fdt_b200 import lib

    o = whole_brain_options()
    items = batched_workload(scale)
    protos = {}
    dev_items = []
    for it in items:
        M = it["prot"].ndir
        if M not in protos:
            protos[M] = (lib.to_device(it["prot"].bvecs), lib.to_device(it["prot"].bvals))
        bv, bl = protos[M]
        dev_items.append(dict(data=lib.to_device(it["host"]), bvecs=bv, bvals=bl, model=it["model"],
                              nfibres=it["nfibres"], voxel_offset=it["voxel_offset"]))
    nvox = sum(int(it["host"].shape[0]) for it in items)
    t0 = time.perf_counter()
    batch = lib.Batch(o, dev_items, autotune=True)
    t_create = time.perf_counter() - t0
    stream = torch.cuda.current_stream()

    def timed(fn, k):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for e0, e1 in evs:
            e0.record(stream)
            fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return sum(e0.elapsed_time(e1) for e0, e1 in evs) / 1e3 / k

    for _ in range(warmup):
        batch.run()
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    t_batch = timed(batch.run, steps)
    ck = clocks.stop()
    work = [torch.empty_like(d["data"]) for d in dev_items]
    outs = []
    for it in items:
        oi = Options.make(**{f: getattr(o, f) for f, _ in Options._fields_ if f != "reserved"})
        oi.model, oi.nfibres = it["model"], it["nfibres"]
        outs.append((oi, lib.alloc_outputs(oi, int(it["host"].shape[0]))))

    def sequential():
        for d, w, (oi, out) in zip(dev_items, work, outs):
            w.copy_(d["data"])
            lib.xfibres_dev(oi, w, d["bvecs"], d["bvals"], voxel_offset=d["voxel_offset"], out=out)

    sequential()
    torch.cuda.synchronize()
    t_seq = timed(sequential, 1)
    line = {
        "metric": "voxels/s, batched form (16 mixed volumes in one CUDA-graph launch)", "value": nvox / t_batch,
        "unit": "voxels/s", "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": 1e3 * t_batch,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": "C2 batch: 16 volumes, voxels log-uniform in [5k, 300k] x %g, ndir from "
                   "{33, 65, 129, 279}, models 1/2 per volume, 1..3 fibres per voxel, SNR U(10,40); "
                   "rician+f0+ardf0, burnin 1000, njumps 1250" % scale,
                   "scale": scale, "voxels": nvox, "items": len(items), "l2": "inputs larger than L2"},
        "sequential_per_item": {"value": nvox / t_seq, "unit": "voxels/s", "launches": 4 * len(items)},
        "batched_over_sequential": t_seq / t_batch,
        "buckets": batch.buckets(), "create_s": t_create,
        "gpu_launches": 1, "clocks": ck,
    }
    batch.close()
    return line


def run_batched(args):
    print(json.dumps(batched_record(args.batch_scale, args.steps, args.warmup)), flush=True)


def whole_volume_once(L, lo: Options, prot, mlp_h, freeze: int, seed: int = 4) -> dict:
    """The whole-brain volume (145x174x145 grid, ellipsoidal mask of ~900k voxels) through ONE call
    of bpx_xfibres_learned_host with pinned host buffers: data generated by the forward model on the
    device (bpx_synth_dev, SNR 25) and copied to the host first, outside the timed call."""
    import ctypes as C

    import torch

    from fdt_b200 import lib
    from fdt_b200.abi import Volume

    mask = synth.ellipsoid_mask((145, 174, 145), 900_000)
    n = int(mask.sum())
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    d, _ = lib.synth(2, 3, n, bv, bl, seed, (25.0, 25.0))
    hd = torch.empty(d.shape, dtype=torch.float32, pin_memory=True)
    hd.copy_(d)
    del d
    torch.cuda.empty_cache()
    hout = lib.alloc_outputs(lo, n, device="cpu", pin=True)
    bh = np.ascontiguousarray(prot.bvecs, np.float32)
    lh = np.ascontiguousarray(prot.bvals, np.float32)
    v = Volume()
    v.nvox, v.ndir = n, prot.ndir
    v.data, v.bvecs, v.bvals = hd.data_ptr(), bh.ctypes.data, lh.ctypes.data
    v.grad = None
    v.voxel_offset = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lib._check(L.bpx_xfibres_learned_host(C.byref(lo), C.byref(v), mlp_h.ctypes.data, freeze, C.byref(hout[1])),
               "xfibres_learned_host (whole volume)")
    dt = time.perf_counter() - t0
    ok = bool(torch.isfinite(hout[0]["mean_f"]).all())
    L.bpx_release_workspace()
    return {"voxels": n, "grid": [145, 174, 145], "calls": 1, "seconds": dt, "voxels_per_s": n / dt,
            "entry": "bpx_xfibres_learned_host", "outputs_finite": ok,
            "h2d_bytes": n * prot.ndir * 4, "d2h_bytes": sum(t.numel() * t.element_size() for t in hout[0].values())}


def run_c3(args):
    """Config C3: the initialiser network for the 279-measurement multi-shell protocol (9 b=0 + 90
    directions at b=1000/2000/3000; model 2, 3 fibres, the options of config C1), evaluated on a
    ~200k-voxel volume (96x96x60 grid, ellipsoidal mask; forward-model voxels, SNR 25): the learned
    form (burn-in 200) against the plain LM-initialised chain (burn-in 1000), each one call over the
    whole volume on device buffers, plus the multi-chain accuracy study on a subset."""
    import torch

    from fdt_b200 import learned, lib

    o = Options.make(**learned.OPTION_SETS["c1"])
    lo = learned_options(o)
    prot = synth.three_shell(9, 90)
    wpath = args.weights or learned.default_weights_path("multishell")
    mlp_h, meta = learned.load_weights(wpath)
    if int(meta["ndir"]) != prot.ndir:
        raise SystemExit(f"{wpath}: trained for {int(meta['ndir'])} measurements, the protocol has {prot.ndir}")
    mlp_d = torch.from_numpy(mlp_h).cuda()
    n = int(synth.ellipsoid_mask((96, 96, 60), 200_000).sum())
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    data, truth_d = lib.synth(2, 3, n, bv, bl, 2, (25.0, 25.0))
    stream = torch.cuda.current_stream()
    outs = {"plain": lib.alloc_outputs(o, n), "learned": lib.alloc_outputs(lo, n)}

    def run(form):
        if form == "plain":
            lib.xfibres_dev(o, data, bv, bl, out=outs["plain"])
        else:
            learned.xfibres_learned(lo, data, bv, bl, mlp_d, freeze=args.freeze, out=outs["learned"])

    t = {}
    clocks = ClockSampler(0)
    clocks.start()
    for form in ("plain", "learned"):
        for _ in range(max(1, min(args.warmup, 1))):
            run(form)
        k = max(1, min(args.steps, 2))
        e = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for e0, e1 in e:
            e0.record(stream)
            run(form)
            e1.record(stream)
        torch.cuda.synchronize()
        t[form] = sum(a.elapsed_time(b) for a, b in e) / 1e3 / k
    ck = clocks.stop()
    # ground truth of the study's voxels (state rows: S0, d, d_std, R, tau, f0, then th, ph, f per fibre)
    tr = truth_d[: args.acc_voxels].double().cpu().numpy()
    th, ph = tr[:, 6::3][:, :3], tr[:, 7::3][:, :3]
    v = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1)
    truth = synth.Truth(tr[:, 0], tr[:, 1], tr[:, 2], tr[:, 8::3][:, :3], v)
    acc = learned.study_report(learned.posterior_study(o, data[: args.acc_voxels].contiguous(), bv, bl, mlp_d,
                                                       R=args.acc_chains), truth)
    line = {
        "metric": "voxels/s, learned-init vs plain MCMC on 1 B200 (config C3)", "value": n / t["learned"],
        "unit": "voxels/s", "n_gpus": 1, "steps": k, "warmup": 1, "ms_per_step": 1e3 * t["learned"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": "C3: 279-measurement multi-shell protocol, model 2, 3 fibres (C1 options), "
                   "96x96x60 ellipsoid of %d voxels, SNR 25; learned burn-in 200 vs plain burn-in 1000, "
                   "njumps 1250, one call per volume" % n, "weights": os.path.relpath(wpath, ROOT),
                   "n_train": int(meta.get("n_train", 0)), "freeze_props": args.freeze},
        "forms": {f: {"voxels_per_s": n / t[f], "seconds_per_volume": t[f]} for f in t},
        "learned_over_plain": t["plain"] / t["learned"],
        "accuracy": acc, "clocks": ck, "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)


def run_plain_config(args, name: str):
    """The plain form (prepare, LM fits, MCMC burn-in 1000, finishing) on one whole volume of config
    C0 (model 1, 2 fibres, 500 voxels, 64 measurements, SNR 20) or C1 (model 2, 3 fibres, 96x96x60
    ellipsoid of ~200k voxels, 279 measurements, SNR 25), one call per step on device buffers, with
    the fit and chain phases timed separately and the chain's roofline fraction."""
    import ctypes as C

    import torch

    from fdt_b200 import lib

    if name == "c0":
        vol = synth.config_small_model1()
        o = Options.make(model=1, nfibres=2)
    else:
        vol = synth.config_multishell_model2()
        o = Options.make(model=2, nfibres=3)
    prot, n, M = vol.prot, vol.nvox, vol.prot.ndir
    L = lib.load()
    d = lib.to_device(vol.data)
    bv, bl = lib.to_device(prot.bvecs), lib.to_device(prot.bvals)
    params = torch.empty((n, o.nparams_fit), device="cuda")
    tau = torch.empty(n, device="cuda")
    status = torch.zeros(n, device="cuda", dtype=torch.int32)
    rec = torch.empty((6 + 3 * o.nfibres, o.nsamples, n), device="cuda")
    out = lib.alloc_outputs(o, n)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    vv = lib.make_volume(d, bv, bl)

    def step(ev=None):
        if ev:
            ev[0].record(stream)
        lib._check(L.bpx_fit_dev(C.byref(o), C.byref(vv), params.data_ptr(), tau.data_ptr(), status.data_ptr(), sp),
                   "fit")
        if ev:
            ev[1].record(stream)
        lib._check(L.bpx_mcmc_dev(C.byref(o), C.byref(vv), params.data_ptr(), tau.data_ptr(), rec.data_ptr(),
                                  status.data_ptr(), sp), "mcmc")
        if ev:
            ev[2].record(stream)
        lib._check(L.bpx_finish_dev(C.byref(o), n, rec.data_ptr(), C.byref(out[1]), sp), "finish")
        if ev:
            ev[3].record(stream)

    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    k = max(1, args.steps)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(k)]
    for e in evs:
        step(e)
    torch.cuda.synchronize()
    ck = clocks.stop()
    ph = [sum(e[a].elapsed_time(e[a + 1]) for e in evs) / 1e3 / k for a in range(3)]
    t = sum(ph)
    mufu_peak, fma_peak = lib.measure_pipes()
    mufu_v, fp32_v = mcmc_work_canonical(o, M)
    frac = max(mufu_v * n / mufu_peak, fp32_v * n / fma_peak) / ph[1]
    line = {
        "metric": f"voxels/s, plain form on config {name.upper()} (1 B200)", "value": n / t, "unit": "voxels/s",
        "n_gpus": 1, "steps": k, "warmup": max(1, args.warmup), "ms_per_step": 1e3 * t, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"config {name.upper()}: model {o.model}, {o.nfibres} fibres, {M} measurements, "
                   f"{n} voxels, burnin 1000, njumps 1250, sampleevery 25, one call per volume"},
        "phases_s": {"fit": ph[0], "mcmc": ph[1], "finish": ph[2]},
        "mcmc_roofline": {"frac": frac, "bound": "fp32" if fp32_v / fma_peak > mufu_v / mufu_peak else "sfu",
                          "counts": "canonical per-term counts, measured MUFU/FFMA peaks"},
        "clocks": ck, "gpu_launches": 7 * k,
    }
    print(json.dumps(line), flush=True)


def run_probtrack(args):
    """probtrackx on the GPU: streamlines/s on a synthetic crossing-fibre field with the
    whole-brain sample count (96x96x60 grid, ellipsoidal mask, 3 fibres x 50 samples; fibre 1 along
    x, fibre 2 along y in half the volume), 1024 seed points in the mask x 5000 particles, probtrackx
    defaults (2000 steps, 0.5 mm, cthr 0.2, fibthresh 0.01), 2 mm voxels.  The CPU oracle of the
    same tracking is timed on 4 seed points per host thread (all threads) as the CPU baseline."""
    import torch

    from fdt_b200 import lib
    from fdt_b200.abi import TrackOptions
    from oracle import oracle as O

    th, ph, f, mask = synth.fibre_field((96, 96, 60), nsamples=50, seed=1)
    rng = np.random.default_rng(2)
    inside = np.argwhere(mask > 0)  # [z, y, x]
    pick = inside[rng.choice(len(inside), args.track_seeds, replace=False)]
    seeds = np.ascontiguousarray(pick[:, ::-1].astype(np.float32))
    # --track-options: loopcheck, modeuler (options), targets (3 target planes across the x-running
    # tracts, seeds to targets), matrix2 (a tract space of 4 mm voxels over the whole grid), prefdir
    # (a preferred direction along x in every voxel of the mask's lower half, zero elsewhere)
    topts = [t for t in args.track_options.split(",") if t]
    for t in topts:
        if t not in ("loopcheck", "modeuler", "targets", "matrix2", "prefdir"):
            raise SystemExit(f"--track-options: unknown option {t}")
    o = TrackOptions.make(seed=9, loopcheck=int("loopcheck" in topts), modeuler=int("modeuler" in topts))
    extra = {}
    if "targets" in topts:
        planes = []
        for x in (20, 48, 70):
            pl = np.zeros_like(mask)
            pl[:, :, x] = 1.0
            planes.append(pl)
        extra["targets"] = planes
    if "matrix2" in topts:
        extra["matrix2"] = (np.ones((30, 48, 48), np.float32), (4.0, 4.0, 4.0))
    if "prefdir" in topts:
        pref = np.zeros((3,) + mask.shape, np.float32)
        pref[0, : mask.shape[0] // 2] = 1.0
        extra["prefdir"] = pref
    dev = [lib.to_device(a) for a in (th, ph, f, mask)]
    sd = lib.to_device(seeds)
    v = lib.track_volume(*dev)
    if "prefdir" in topts:
        pref_d = lib.to_device(extra["prefdir"])
        v.prefdir = pref_d.data_ptr()
    outs = []  # per-option outputs, zeroed every step
    if "targets" in topts:
        tb = torch.from_numpy(lib.waypoint_bits(extra["targets"])).cuda()
        s2t = torch.zeros((3, len(seeds)), device="cuda", dtype=torch.int32)
        v.ntargets, v.targets, v.seeds_to_targets = 3, tb.data_ptr(), s2t.data_ptr()
        outs.append(s2t)
    if "matrix2" in topts:
        lut = torch.from_numpy(lib.matrix2_lookup(extra["matrix2"][0])).cuda()
        m2 = torch.zeros((len(seeds), int(lut.numel())), device="cuda", dtype=torch.int32)
        v.m2_ncols, v.lr_nx, v.lr_ny, v.lr_nz = int(lut.numel()), 48, 48, 30
        v.lr_dx = v.lr_dy = v.lr_dz = 4.0
        v.m2_lookup, v.matrix2 = lut.data_ptr(), m2.data_ptr()
        outs.append(m2)
    paths = torch.zeros(mask.shape, device="cuda", dtype=torch.int32)
    way = torch.zeros(1, device="cuda", dtype=torch.int64)
    L = lib.load()
    import ctypes as C

    stream = torch.cuda.current_stream()

    def step():
        paths.zero_()
        way.zero_()
        for t in outs:
            t.zero_()
        lib._check(L.bpx_probtrack_dev(C.byref(o), C.byref(v), len(seeds), sd.data_ptr(), paths.data_ptr(),
                                       way.data_ptr(), C.c_void_p(stream.cuda_stream)), "probtrack")

    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    k = max(1, args.steps)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
    for e0, e1 in ev:
        e0.record(stream)
        step()
        e1.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    t = sum(a.elapsed_time(b) for a, b in ev) / 1e3 / k
    n_lines = len(seeds) * o.nparticles
    # the CPU oracle on all host threads (OpenMP over particles), 4 seed points per thread
    cores = os.cpu_count() or 1
    nb = min(len(seeds), 4 * cores)
    o_cpu = TrackOptions.make(seed=9, loopcheck=o.loopcheck, modeuler=o.modeuler)
    t0 = time.perf_counter()
    O.probtrack(o_cpu, th, ph, f, mask, seeds[:nb], **extra)
    t_cpu = time.perf_counter() - t0
    line = {
        "metric": "streamlines/s, probtrackx on bedpostx samples (1 B200)", "value": n_lines / t,
        "unit": "streamlines/s", "n_gpus": 1, "steps": k, "warmup": max(1, args.warmup), "ms_per_step": 1e3 * t,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": "probtrackx (one path distribution over all seeds, as seedmask mode): 96x96x60 "
                   "crossing-fibre field, 3 fibres x 50 samples, "
                   "%d seeds x 5000 particles, 2000 steps of 0.5 mm, cthr 0.2, fibthresh 0.01" % len(seeds)
                   + "".join(", " + t for t in topts),
                   "streamlines": n_lines, "waytotal": int(way.item()), "visits": int(paths.sum(dtype=torch.int64).item())},
        "cpu_baseline": {"value": nb * o.nparticles / t_cpu, "unit": "streamlines/s", "cores": cores, "kind": "port",
                         "sample": f"{nb} seed points x {o.nparticles} particles through the CPU oracle, "
                                   f"{t_cpu:.1f} s on {cores} threads"},
        "gpu_launches": k, "clocks": ck,
    }
    print(json.dumps(line), flush=True)


def learned_options(o: Options) -> Options:
    """Options of the learned form: the plain options with burn-in 200 and another RNG seed."""
    lo = Options.make(**{f: getattr(o, f) for f, _ in Options._fields_ if f != "reserved"})
    lo.nburn = 200
    lo.seed = o.seed + 1
    return lo


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--chunk", type=int, default=131072, help="voxels per step per GPU")
    ap.add_argument("--ref-voxels", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--form", default="all", choices=["all", "plain", "learned", "learned_batched"],
                    help="forms to time (the headline value is the learned, batched form's)")
    ap.add_argument("--freeze", type=int, default=0, choices=[0, 1, 2],
                    help="learned form: 0 network widths adapt, 1 frozen, 2 frozen after burn-in")
    ap.add_argument("--weights", default=None, help="initialiser weights (default: the committed whole-brain set)")
    ap.add_argument("--workload", default="whole_brain",
                    choices=["whole_brain", "batched", "c0", "c1", "c3", "probtrack"],
                    help="batched: the mixed 16-volume batch in one graph launch (one GPU); c3: the "
                         "279-measurement network on a 200k-voxel volume (one GPU)")
    ap.add_argument("--batch-scale", type=float, default=0.5,
                    help="batched: voxel-count scale (also the C2 sub-record of the default line)")
    ap.add_argument("--no-c2", action="store_true", help="skip the C2 (mixed batch) sub-record")
    ap.add_argument("--track-seeds", type=int, default=1024, help="probtrack: seed points")
    ap.add_argument("--track-options", default="",
                    help="probtrack: comma list of loopcheck, modeuler, targets, matrix2 (default: none)")
    ap.add_argument("--no-whole-volume", action="store_true",
                    help="skip the one-call run of the ~900k-voxel whole-brain volume")
    ap.add_argument("--acc-voxels", type=int, default=4096, help="accuracy study: voxels")
    ap.add_argument("--acc-chains", type=int, default=8, help="accuracy study: chains per voxel and form")
    ap.add_argument("--prof", action="store_true",
                    help="profiling case: run the steps only (no e2e, CPU baseline, accuracy or calibration)")
    ap.add_argument("--nburn", type=int, default=None, help="override burn-in (profiling cases)")
    ap.add_argument("--njumps", type=int, default=None, help="override jumps (profiling cases)")
    args = ap.parse_args()
    if args.prof:
        args.no_e2e = True
        args.no_cpu_baseline = True
        args.no_accuracy = True
        args.no_c2 = True
        args.no_whole_volume = True
    world, rank, local = dist_setup(args)

    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "batched":
        if rank == 0:
            run_batched(args)
        return
    if args.workload == "c3":
        if rank == 0:
            run_c3(args)
        return
    if args.workload == "probtrack":
        if rank == 0:
            run_probtrack(args)
        return
    if args.workload in ("c0", "c1"):
        if rank == 0:
            run_plain_config(args, args.workload)
        return

    import ctypes as C

    import torch

    from fdt_b200 import learned, lib

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    L = lib.load()
    o = whole_brain_options()
    if args.nburn is not None:
        o.nburn = args.nburn
    if args.njumps is not None:
        o.njumps = args.njumps
    lo = learned_options(o)
    prot = synth.three_shell(18, 90)
    M = prot.ndir
    chunk = args.chunk
    forms = ["plain", "learned", "learned_batched", "lm_burnin200"] if args.form == "all" else [args.form]
    # the ablation form (the method without the network at the learned form's burn-in) is timed on
    # fewer steps: it is a reported comparison, not the headline
    short_forms = {"lm_burnin200"}
    wpath = args.weights or learned.default_weights_path("whole_brain")
    uses_net = "learned" in forms or "learned_batched" in forms
    mlp_h, meta = learned.load_weights(wpath) if uses_net else (None, None)
    if mlp_h is not None and int(meta["ndir"]) != M:
        raise SystemExit(f"{wpath}: trained for {int(meta['ndir'])} measurements, the workload has {M}")
    mlp_d = torch.from_numpy(mlp_h).cuda() if mlp_h is not None else None
    # two distinct chunks per rank, alternated between steps
    chunks_h = []
    truth0 = None  # ground truth of the first chunk (the accuracy study's voxels)
    for c in range(2):
        y, tr = synth.make_volume(chunk, prot, 3, True, 25.0, seed=9000 + 17 * rank + c)
        chunks_h.append(y)
        truth0 = tr if c == 0 else truth0
    bvecs = lib.to_device(prot.bvecs)
    bvals = lib.to_device(prot.bvals)
    chunks_d = [lib.to_device(y) for y in chunks_h]
    work = torch.empty_like(chunks_d[0])
    nin = learned.nin(M)
    params = torch.empty((chunk, o.nparams_fit), device="cuda")
    tau = torch.empty(chunk, device="cuda")
    status = torch.zeros(chunk, device="cuda", dtype=torch.int32)
    rec = torch.empty((6 + 3 * o.nfibres, o.nsamples, chunk), device="cuda")
    x = torch.empty((chunk, nin), device="cuda", dtype=torch.bfloat16)
    s0hat = torch.empty(chunk, device="cuda")
    netout = torch.empty((chunk, 32), device="cuda")
    props = torch.empty((6 + 3 * o.nfibres, chunk), device="cuda")
    outs = {f: lib.alloc_outputs(o, chunk) for f in forms}
    flush = torch.empty(256 * 1024 * 1024 // 4, device="cuda")
    stream = torch.cuda.current_stream()
    sptr = C.c_void_p(stream.cuda_stream)

    def plain_step(i, ev=None, opts=o, out=None):
        work.copy_(chunks_d[i % 2])  # the path cleans the data in place under --rician
        vol = lib.make_volume(work, bvecs, bvals, voxel_offset=(rank * 1_000_000_000) + i * chunk)
        if ev:
            ev[0].record(stream)
        lib._check(L.bpx_prepare_data_dev(chunk, M, work.data_ptr(), sptr), "prepare")
        lib._check(L.bpx_fit_dev(C.byref(opts), C.byref(vol), params.data_ptr(), tau.data_ptr(), status.data_ptr(),
                                 sptr), "fit")
        if ev:
            ev[1].record(stream)
        lib._check(L.bpx_mcmc_dev(C.byref(opts), C.byref(vol), params.data_ptr(), tau.data_ptr(), rec.data_ptr(),
                                  status.data_ptr(), sptr), "mcmc")
        if ev:
            ev[2].record(stream)
        lib._check(L.bpx_finish_dev(C.byref(opts), chunk, rec.data_ptr(), C.byref((out or outs["plain"])[1]), sptr),
                   "finish")
        if ev:
            ev[3].record(stream)

    def learned_step(i, ev=None):
        work.copy_(chunks_d[i % 2])
        vol = lib.make_volume(work, bvecs, bvals, voxel_offset=(rank * 1_000_000_000) + i * chunk)
        if ev:
            ev[0].record(stream)
        lib._check(L.bpx_prepare_data_dev(chunk, M, work.data_ptr(), sptr), "prepare")
        lib._check(L.bpx_mlp_features_dev(C.byref(vol), 0, x.data_ptr(), s0hat.data_ptr(), sptr), "features")
        lib._check(L.bpx_mlp_forward_dev(M, mlp_d.data_ptr(), chunk, x.data_ptr(), netout.data_ptr(), sptr), "network")
        lib._check(L.bpx_mlp_decode_dev(C.byref(lo), chunk, netout.data_ptr(), s0hat.data_ptr(), params.data_ptr(),
                                        tau.data_ptr(), props.data_ptr(), status.data_ptr(), sptr), "decode")
        if ev:
            ev[1].record(stream)
        lib._check(L.bpx_mcmc_ex_dev(C.byref(lo), C.byref(vol), params.data_ptr(), tau.data_ptr(), props.data_ptr(),
                                     None, args.freeze, rec.data_ptr(), status.data_ptr(), sptr), "mcmc")
        if ev:
            ev[2].record(stream)
        lib._check(L.bpx_finish_dev(C.byref(lo), chunk, rec.data_ptr(), C.byref(outs["learned"][1]), sptr), "finish")
        if ev:
            ev[3].record(stream)

    lbatches = None
    if "learned_batched" in forms:
        # one batch (one captured graph) per input chunk; the chunk's voxels form one bucket
        lbatches = [lib.Batch(o, [dict(data=chunks_d[c], bvecs=bvecs, bvals=bvals, model=o.model, nfibres=o.nfibres,
                                       mlp=mlp_d, nburn=lo.nburn, freeze=args.freeze,
                                       voxel_offset=rank * 1_000_000_000 + (2 + c) * chunk)], autotune=False)
                    for c in range(2)]

    def learned_batched_step(i, ev=None):
        if ev:
            ev[0].record(stream)
        lbatches[i % 2].run()
        if ev:
            ev[1].record(stream)
            ev[2].record(stream)
            ev[3].record(stream)

    lm200 = Options.make(**{f: getattr(o, f) for f, _ in Options._fields_ if f != "reserved"})
    lm200.nburn = 200
    lm200.seed = o.seed + 2

    def lm200_step(i, ev=None):
        plain_step(i, ev, opts=lm200, out=outs["lm_burnin200"])

    steps_fn = {"plain": plain_step, "learned": learned_step, "learned_batched": learned_batched_step,
                "lm_burnin200": lm200_step}
    # learned: prepare, features, weight cast + 5 GEMMs per 32768 voxels, decode, mcmc, finish;
    # learned_batched: one CUDA-graph launch (gather, the same kernels, scatter)
    n_gemm = 5 * ((chunk + 32767) // 32768)
    # kernels per step: plain = Rician clean-up, 4 fit stages, MCMC, finishing; learned = clean-up,
    # features, weight cast, the GEMMs, decode, MCMC, finishing; the graph form launches once and its
    # graph holds gather, the learned form's kernels and scatter
    launches = {"plain": 7, "learned": 6 + n_gemm, "learned_batched": 8 + n_gemm, "lm_burnin200": 7}
    timing = {}
    clocks = ClockSampler(local)
    clocks.start()
    nsteps = {}
    for f in forms:
        ns_f, nw_f = (min(args.steps, 3), min(args.warmup, 1)) if f in short_forms else (args.steps, args.warmup)
        nsteps[f] = ns_f
        for i in range(nw_f):
            flush.zero_()
            steps_fn[f](i)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(ns_f)]
        for i in range(ns_f):
            flush.zero_()  # L2 flush (256 MB write), outside the timed events
            steps_fn[f](nw_f + i, evs[i])
        torch.cuda.synchronize()
        t = [sum(e[a].elapsed_time(e[a + 1]) for e in evs) / 1e3 for a in range(3)]
        tt = torch.tensor([sum(t)] + t, device="cuda", dtype=torch.float64)
        if pg:
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        timing[f] = tt.tolist()
    ck = clocks.stop()
    head = "learned_batched" if "learned_batched" in forms else ("learned" if "learned" in forms else "plain")
    t_step = timing[head][0]
    vox_total = chunk * args.steps * world
    value = vox_total / t_step
    # the MCMC kernel time for the roofline: from a form whose phases are timed separately
    rf = "learned" if "learned" in forms else ("plain" if "plain" in forms else head)
    t_mcmc = timing[rf][2] if rf != "learned_batched" else timing[rf][0]
    ho = o if rf == "plain" else lo

    # ---- accuracy of the learned form against the plain chain on the same voxels ----
    accuracy = None
    if not args.no_accuracy and uses_net and rank == 0:
        # R independent chains per voxel and form (the Monte-Carlo SE of a posterior mean is the
        # spread of the chain means), on the first voxels of the first chunk, cleaned as the path
        # cleans them; forms: plain (the comparator), plain at another seed (yardstick), learned
        # (adapting and frozen widths), LM start at the learned burn-in (the method without the
        # network), and a long LM-started chain (gold)
        d_acc = chunks_d[0][: args.acc_voxels].clone()
        lib.prepare_data(d_acc)
        sets = learned.posterior_study(o, d_acc, bvecs, bvals, mlp_d, R=args.acc_chains)
        accuracy = learned.study_report(sets, truth0)
        accuracy["se"] = ("Monte-Carlo SE of a posterior mean = sd of the chain means / sqrt(chains); "
                          "|difference| <= 2 sqrt(se_a^2 + se_b^2) counts as agreement")
        accuracy["dyads"] = "median angle between pooled dyads; 'supported' = fibres with mean f >= 0.05 in both"
        accuracy["truth"] = ("vs_truth: each form's pooled posterior means against the synthetic ground truth, "
                             "fibres ranked by fraction; dyad angles over fibres with true f >= 0.05")
        del sets

    # ---- end to end through the host-buffer public entries (pinned host memory) ----
    e2e = None
    if not args.no_e2e:
        hp = [torch.from_numpy(y).pin_memory() for y in chunks_h]
        hout = lib.alloc_outputs(o, chunk, device="cpu", pin=True)
        bh = np.ascontiguousarray(prot.bvecs, np.float32)
        lh = np.ascontiguousarray(prot.bvals, np.float32)
        from fdt_b200.abi import Volume

        def host_step(i):
            v = Volume()
            v.nvox, v.ndir = chunk, M
            v.data, v.bvecs, v.bvals = hp[i % 2].data_ptr(), bh.ctypes.data, lh.ctypes.data
            v.grad = None
            v.voxel_offset = rank * 1_000_000_000 + i * chunk
            if head != "plain":
                lib._check(L.bpx_xfibres_learned_host(C.byref(lo), C.byref(v), mlp_h.ctypes.data, args.freeze,
                                                      C.byref(hout[1])), "xfibres_learned_host")
            else:
                lib._check(L.bpx_xfibres_host(C.byref(o), C.byref(v), C.byref(hout[1])), "xfibres_host")

        host_step(0)
        if pg:
            pg.barrier()
        n_e2e = max(1, min(args.steps, 3))
        t0 = time.perf_counter()
        for i in range(n_e2e):
            host_step(i + 1)
        te = torch.tensor([time.perf_counter() - t0], device="cuda", dtype=torch.float64)
        if pg:
            pg.all_reduce(te, op=pg.ReduceOp.MAX)
        h2d = chunk * M * 4 + 4 * 4 * M + (mlp_h.nbytes if head != "plain" else 0)
        d2h = sum(t.numel() * t.element_size() for t in hout[0].values())
        e2e = {"value": chunk * n_e2e * world / te.item(), "unit": "voxels/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": n_e2e, "entry": "bpx_xfibres_learned_host" if head != "plain"
               else "bpx_xfibres_host"}
        del hp, hout
        if not args.no_whole_volume and head != "plain" and rank == 0:
            e2e["whole_volume_once"] = whole_volume_once(L, lo, prot, mlp_h, args.freeze)

    if args.prof:
        if rank == 0:
            print(json.dumps({"prof": True, "voxels": chunk, "timing": timing}), flush=True)
        return
    # ---- roofline of the dominant kernel (the MCMC chain) ----
    mufu_peak, fma_peak = lib.measure_pipes()
    mcmc_per_launch_s = t_mcmc / args.steps

    def pipe_fracs(mufu_v: float, fp32_v: float) -> dict:
        t_mufu, t_fp32 = mufu_v * chunk / mufu_peak, fp32_v * chunk / fma_peak
        sfu_a, fp32_a = mufu_v * chunk / mcmc_per_launch_s, fp32_v * chunk / mcmc_per_launch_s
        fp32_bound = t_fp32 >= t_mufu  # the pipe whose work takes longer at its measured peak
        return {"bound": "fp32" if fp32_bound else "sfu",
                "achieved": (fp32_a if fp32_bound else sfu_a) / 1e9,
                "peak": (fma_peak if fp32_bound else mufu_peak) / 1e9,
                "frac": max(t_mufu, t_fp32) / mcmc_per_launch_s,
                "sfu_achieved": sfu_a / 1e9, "sfu_frac": sfu_a / mufu_peak,
                "fp32_achieved": fp32_a / 1e9, "fp32_frac": fp32_a / fma_peak,
                "work_per_voxel": {"mufu": mufu_v, "fp32": fp32_v}}

    canon = pipe_fracs(*mcmc_work_canonical(ho, M))
    own = pipe_fracs(*mcmc_work_per_voxel(ho, M))
    roofline = {
        "bound": canon["bound"], "achieved": canon["achieved"], "peak": canon["peak"], "unit": "Gop/s",
        "frac": canon["frac"],
        "traffic": (MCMC_DRAM_BYTES_LAUNCH if chunk == MCMC_DRAM_LAUNCH_VOXELS else
                    MCMC_DRAM_BYTES_LAUNCH / MCMC_DRAM_LAUNCH_VOXELS * chunk)
        if (o.model, o.nfibres, M, o.nsamples) == (2, 3, 288, 50) else None,
        "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one 131072-voxel mcmc_kernel launch "
                           "on this workload's options" + ("" if chunk == MCMC_DRAM_LAUNCH_VOXELS else
                                                           ", per voxel, scaled by the voxels of this launch")),
        "kernel": f"mcmc_kernel (burn-in + recording), timed in the {rf} form's step",
        "counts": "canonical per-term counts (model-2 signal rcp+log2+exp2, Rician log2+rsqrt; FMA 6 per signal "
                  "term, K+4(+12 Rician) per likelihood term)",
        "sfu_peak": mufu_peak / 1e9, "fp32_peak": fma_peak / 1e9,
        "sfu_frac": canon["sfu_frac"], "fp32_frac": canon["fp32_frac"],
        "work_per_voxel": canon["work_per_voxel"],
        "kernel_formulation": {k: own[k] for k in ("bound", "frac", "sfu_frac", "fp32_frac", "work_per_voxel")},
        "peak_source": "measured on this GPU by bpx_measure_pipes (ex2.approx and FFMA issue-rate kernels)",
    }
    peaks = measured_peaks()
    forms_out = {}
    nb_form = {"plain": o.nburn, "learned": lo.nburn, "learned_batched": lo.nburn, "lm_burnin200": lm200.nburn}
    for f in forms:
        ts_, ti, tm, tf = timing[f]
        k = nsteps[f]
        forms_out[f] = {"voxels_per_s": chunk * k * world / ts_, "ms_per_step": 1e3 * ts_ / k, "steps": k,
                        "nburn": nb_form[f], "gpu_launches_per_step": launches[f]}
        if f != "learned_batched":
            forms_out[f]["phases_s_per_step"] = {"init": ti / k, "mcmc": tm / k, "finish": tf / k}
    if "lm_burnin200" in forms_out:
        forms_out["lm_burnin200"]["what"] = ("the method without the network at the learned form's burn-in: "
                                             "LM fits + tau, reference widths, burn-in 200")
    result = {
        "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_step / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": WORKLOAD_LEARNED if head != "plain" else WORKLOAD,
                   "voxels_per_step_per_gpu": chunk, "ndir": M,
                   "l2": "flushed between steps (256 MB write) and inputs (151 MB/step) larger than L2",
                   "form": head, "freeze_props": args.freeze if head != "plain" else None,
                   "weights": os.path.relpath(wpath, ROOT) if head != "plain" else None},
        "forms": forms_out,
        "learned_over_plain": (forms_out[head]["voxels_per_s"] / forms_out["plain"]["voxels_per_s"])
        if "plain" in forms and head != "plain" else None,
        "accuracy": accuracy,
        "roofline": roofline,
        "e2e": e2e,
        "gpu_launches": launches[head] * args.steps,
        "clocks": ck,
        "hbm_peak_gbs": peaks.get("hbm_gbs"),
    }
    if "lm_burnin200" in forms_out and head != "plain":
        result["learned_over_lm_burnin200"] = forms_out[head]["voxels_per_s"] / forms_out["lm_burnin200"]["voxels_per_s"]
    if rank == 0 and not args.no_c2 and world == 1:
        del outs, chunks_d, work, flush
        if lbatches:
            for b in lbatches:
                b.close()
        torch.cuda.empty_cache()
        c2 = batched_record(args.batch_scale, steps=2, warmup=1)
        result["c2_batched"] = {k: c2[k] for k in ("value", "unit", "ms_per_step", "steps", "warmup", "config",
                                                   "sequential_per_item", "batched_over_sequential", "create_s",
                                                   "buckets", "clocks")}
    if rank == 0 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(result), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
