#!/usr/bin/env python
"""Benchmark of the bedpostx per-voxel path on B200 (and of the CPU baseline).

Workload (the whole-brain configuration): model 2 (Gamma-distributed diffusivity), 3 fibres,
--rician --f0 --ardf0, 288 measurements (18 b=0 + 90 directions at b=1000/2000/3000),
burn-in 1000, 1250 jumps, sample every 25, seeded synthetic voxels with SNR 25 generated from the
forward model (no dataset exists for this path).  One step = the whole path (Rician data clean-up,
LM fits + tau, MCMC burn-in + recording, sample finishing) over one chunk of voxels already
resident in HBM.  The chunk (131072 voxels x 288 x 4 B = 151 MB) is larger than the 126 MB L2 and
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


def whole_brain_options() -> Options:
    return Options.make(model=2, nfibres=3, rician=1, f0=1, ardf0=1, nburn=1000, njumps=1250, sampleevery=25)


def mcmc_work_per_voxel(o: Options, ndir: int) -> tuple[float, float]:
    """Algorithmic MUFU and FP32 operations of one voxel's chain (minimal formulation).

    Per iteration: L likelihood evaluations over the M measurements and T signal-term updates.
    MUFU per signal term: 1 (models 1/3: exp2) or 2 (model 2: log2 + exp2 with the per-proposal
    Gamma scale hoisted); per Rician likelihood term 2 (rsqrt + log2), Gaussian 0.  FP32 ops per
    signal term 6, per likelihood term K+4 (+12 Rician).
    """
    K, M = o.nfibres, ndir
    J = o.nburn + o.njumps
    L = (1 if o.f0 else 0) + (1 if o.rician else 0) + 1 + (1 if o.model >= 2 else 0) + (1 if o.model == 3 else 0) \
        + 1 + 3 * K
    T = (K + 1) * M + (K + 1) * M * (1 if o.model == 2 else 0) + M * (1 if o.model == 3 else 0) \
        + K * M * (1 if o.model == 3 else 0) + 2 * K * M
    c_sig = 2 if o.model == 2 else 1
    c_lik = 2 if o.rician else 0
    mufu = J * (T * c_sig + L * M * c_lik)
    fp32 = J * (T * 6 + L * M * (K + 4 + (12 if o.rician else 0)))
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
    ap.add_argument("--prof", action="store_true",
                    help="profiling case: run the steps only (no e2e, CPU baseline or pipe calibration)")
    ap.add_argument("--nburn", type=int, default=None, help="override burn-in (profiling cases)")
    ap.add_argument("--njumps", type=int, default=None, help="override jumps (profiling cases)")
    args = ap.parse_args()
    if args.prof:
        args.no_e2e = True
        args.no_cpu_baseline = True
    world, rank, local = dist_setup(args)

    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch

    from fdt_b200 import lib

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
    prot = synth.three_shell(18, 90)
    M = prot.ndir
    chunk = args.chunk
    # two distinct chunks per rank, alternated between steps
    chunks_h = []
    for c in range(2):
        y, _ = synth.make_volume(chunk, prot, 3, True, 25.0, seed=9000 + 17 * rank + c)
        chunks_h.append(y)
    bvecs = lib.to_device(prot.bvecs)
    bvals = lib.to_device(prot.bvals)
    chunks_d = [lib.to_device(y) for y in chunks_h]
    work = [torch.empty_like(chunks_d[0]) for _ in range(2)]
    np_fit = o.nparams_fit
    ns = o.nsamples
    params = torch.empty((chunk, np_fit), device="cuda")
    tau = torch.empty(chunk, device="cuda")
    status = torch.zeros(chunk, device="cuda", dtype=torch.int32)
    rec = torch.empty((6 + 3 * o.nfibres, ns, chunk), device="cuda")
    outs = lib.alloc_outputs(o, chunk)
    flush = torch.empty(256 * 1024 * 1024 // 4, device="cuda")
    stream = torch.cuda.current_stream()
    sptr = lib.C.c_void_p(stream.cuda_stream)

    import ctypes as C

    def step(i, ev=None):
        src = chunks_d[i % 2]
        w = work[i % 2]
        w.copy_(src)  # the path cleans the data in place under --rician
        vol = lib.make_volume(w, bvecs, bvals, voxel_offset=(rank * 1_000_000_000) + i * chunk)
        if ev:
            ev[0].record(stream)
        lib._check(L.bpx_prepare_data_dev(chunk, M, w.data_ptr(), sptr), "prepare")
        lib._check(L.bpx_fit_dev(C.byref(o), C.byref(vol), params.data_ptr(), tau.data_ptr(), status.data_ptr(), sptr),
                   "fit")
        if ev:
            ev[1].record(stream)
        lib._check(L.bpx_mcmc_dev(C.byref(o), C.byref(vol), params.data_ptr(), tau.data_ptr(), rec.data_ptr(),
                                  status.data_ptr(), sptr), "mcmc")
        if ev:
            ev[2].record(stream)
        lib._check(L.bpx_finish_dev(C.byref(o), chunk, rec.data_ptr(), C.byref(outs[1]), sptr), "finish")
        if ev:
            ev[3].record(stream)

    for i in range(args.warmup):
        flush.zero_()
        step(i)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.zero_()  # L2 flush (256 MB write), outside the timed events
        step(args.warmup + i, evs[i])
    torch.cuda.synchronize()
    ck = clocks.stop()
    t_fit = sum(e[0].elapsed_time(e[1]) for e in evs) / 1e3
    t_mcmc = sum(e[1].elapsed_time(e[2]) for e in evs) / 1e3
    t_fin = sum(e[2].elapsed_time(e[3]) for e in evs) / 1e3
    t_step = t_fit + t_mcmc + t_fin
    times = torch.tensor([t_step, t_fit, t_mcmc, t_fin], device="cuda", dtype=torch.float64)
    if pg:
        pg.all_reduce(times, op=pg.ReduceOp.MAX)
    t_step, t_fit, t_mcmc, t_fin = times.tolist()
    vox_total = chunk * args.steps * world
    value = vox_total / t_step

    # ---- end to end through the host-buffer public entry (pinned host memory) ----
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
        h2d = chunk * M * 4 + 4 * 4 * M
        d2h = sum(t.numel() * t.element_size() for t in hout[0].values())
        e2e = {"value": chunk * n_e2e * world / te.item(), "unit": "voxels/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": n_e2e}

    if args.prof:
        if rank == 0:
            print(json.dumps({"prof": True, "voxels": chunk, "mcmc_s_per_step": t_mcmc / args.steps,
                              "fit_s_per_step": t_fit / args.steps}), flush=True)
        return
    # ---- roofline of the dominant kernel (the MCMC chain) ----
    mufu_peak, fma_peak = lib.measure_pipes()
    mufu_v, fp32_v = mcmc_work_per_voxel(o, M)
    mcmc_per_launch_s = t_mcmc / args.steps
    achieved = mufu_v * chunk / mcmc_per_launch_s
    fp32_achieved = fp32_v * chunk / mcmc_per_launch_s
    roof_time = max(mufu_v * chunk / mufu_peak, fp32_v * chunk / fma_peak)
    roofline = {
        "bound": "sfu", "achieved": achieved / 1e9, "peak": mufu_peak / 1e9, "unit": "Gop/s",
        "frac": achieved / mufu_peak, "traffic": None,
        "fp32_achieved": fp32_achieved / 1e9, "fp32_peak": fma_peak / 1e9,
        "frac_of_roofline_time": roof_time / mcmc_per_launch_s,
        "peak_source": "measured on this GPU by bpx_measure_pipes (ex2.approx and FFMA issue-rate kernels)",
        "work_per_voxel": {"mufu": mufu_v, "fp32": fp32_v},
    }
    peaks = measured_peaks()
    result = {
        "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_step / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "voxels_per_step_per_gpu": chunk, "ndir": M, "l2": "flushed between steps "
                   "(256 MB write) and inputs (151 MB/step) larger than L2", "form": "plain (LM init, burnin 1000)"},
        "phases_s_per_step": {"fit": t_fit / args.steps, "mcmc": t_mcmc / args.steps, "finish": t_fin / args.steps},
        "roofline": roofline,
        "e2e": e2e,
        "gpu_launches": 4 * args.steps,
        "clocks": ck,
        "hbm_peak_gbs": peaks.get("hbm_gbs"),
    }
    if rank == 0 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(result), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
