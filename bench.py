#!/usr/bin/env python3
"""Benchmark of the p2r hot path on B200: track-layer updates/s of the fused chained forward.

Workload (one "step"): the fused forward (propagateToR + KalmanUpdate for every layer of
every track, chained) over 9600 tracks x 100 events x 20 layers, bsize 32, Bz 3.8 T,
synthetic helices (p2r_gen_helix). Inputs (0.80 GB) exceed the 126 MB L2, so no flush is
needed between steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs its own events (weak scaling, no data-path
collective: tracks are independent); the timed region is bracketed by barriers and device
synchronisation and the max over ranks is taken. Rank 0 prints one JSON line.

--impl reference times the reference's own CPU path (src/propagate-tor-test_tbb.cpp,
compiled unmodified into oracle/_ref/) on all host threads, on the same metric and workload
(each step a bounded sample of its events).
"""
from __future__ import annotations

import argparse
import dataclasses
import datetime
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "track-layer updates/s at 960k trk×20 lyr FP32; fwd+adjoint time vs plain fwd"
FLOP_PER_UPDATE = 1272  # 958 propagateToR + 314 KalmanUpdate FP32 ops (FMA = 2)
FP64_OPS_PER_UPDATE = 4
NTRKS, NEVTS, NLAYER, BSIZE, BZ = 9600, 100, 20, 32, 3.8
NOMINAL_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 74.4 at the 1965 MHz max SM clock


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--bsize", type=int, default=BSIZE)
    ap.add_argument("--nevts", type=int, default=NEVTS)
    ap.add_argument("--mode", choices=["chained", "restart"], default="chained")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip timing the reference's CUDA kernels")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adj-steps", type=int, default=10)
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-uneven", action="store_true")
    ap.add_argument("--uneven-steps", type=int, default=10)
    ap.add_argument("--uneven-events", type=int, default=1000, help="events in the uneven-batch workload")
    ap.add_argument("--no-calib", action="store_true", help="skip the 40-layer calibration workload")
    ap.add_argument("--calib-steps", type=int, default=3)
    ap.add_argument("--calib-nevts", type=int, default=100)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline sample budget")
    ap.add_argument("--ref-budget", type=float, default=90.0, help="reference arm: total seconds")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ workload
def make_inputs(p2r, nevts, bsize, seed):
    cfg = p2r.Config(bsize=bsize, nlayer=NLAYER, nevts=nevts, nb=NTRKS // bsize, bz=BZ,
                     mode=p2r.MODE_CHAINED)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=BZ, seed=seed))
    return cfg, trk, hit


def traffic_from_profiles(mode: str):
    """Per-launch DRAM bytes of the fused kernel (chained or restart) from the committed ncu
    summary of that mode, if any."""
    f = ROOT / "profiles" / f"fwd_kernel_{mode}_9600x100x20.md"
    if not f.exists():
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", f.read_text())
    return float(m.group(1)) if m else None


def fp32_gradient_error(g64: dict, g32: dict, bsize: int) -> dict:
    """Error of the FP32 adjoint's gradients against the FP64 adjoint's on the same inputs:
    per-layer dr and Bz relative to the largest |FP64| value; the initial-parameter gradients
    per element relative to the largest |FP64| value of the same parameter over all tracks
    (quantiles over tracks and parameters)."""
    import torch
    dr64, dr32 = g64["grad_dr"].double(), g32["grad_dr"].double()
    bz64, bz32 = float(g64["grad_bz"][0]), float(g32["grad_bz"][0])
    p64 = g64["grad_trk_in"].view(-1, 28, bsize)[:, 0:6, :].permute(0, 2, 1).reshape(-1, 6).double()
    p32 = g32["grad_trk_in"].view(-1, 28, bsize)[:, 0:6, :].permute(0, 2, 1).reshape(-1, 6).double()
    ep = ((p32 - p64).abs() / p64.abs().amax(0).clamp_min(1e-300)).reshape(-1)
    q = torch.quantile(ep[torch.randperm(ep.numel(), device=ep.device)[:1 << 24]],
                       torch.tensor([0.5, 0.99], dtype=torch.float64, device=ep.device)).tolist()
    return {"grad_dr_max_rel": float(((dr32 - dr64).abs().max() / dr64.abs().max()).item()),
            "grad_bz_rel": abs(bz32 - bz64) / abs(bz64),
            "grad_initial_par_p50": q[0], "grad_initial_par_p99": q[1], "grad_initial_par_max": float(ep.max().item())}


def fp64_flop_per_update():
    """Executed FP64 FLOPs per track-layer of the stride-1 FP64 adjoint (forward with tape +
    reverse), from the committed ncu summary, if any."""
    f = ROOT / "profiles" / "tape_adjoint_fp64_ck1_9600x8x20.md"
    if not f.exists():
        return None
    m = re.search(r"fp64_flop_per_update:\s*([0-9.eE+]+)", f.read_text())
    return float(m.group(1)) if m else None


def measured_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    try:
        return json.loads(f.read_text())
    except (OSError, ValueError):
        return {}


# ------------------------------------------------------------------ CPU reference timing
def accuracy_vs_fp64(trk_ev, hit_ev, ours_ev, nb, bsize, bz, nthreads, ref_gpu_ev=None):
    """Error of this library's output and of the reference's own CPU output against the FP64
    oracle on one event of the bench workload (the oracle as the checker). Parameters:
    |a - f64| / max(|f64|, floor), floor (1, 1, 1, 0.01, 1, 1) for (x, y, z, 1/pT, phi, theta);
    covariance: |a - f64| / max(|f64|, sqrt(P_ii P_jj)), P the covariance entering the last
    update. Quantiles over all elements."""
    from oracle.oracle import Oracle, RefTBB, ref_available
    f64 = Oracle().run(trk_ev, hit_ev, bsize, NLAYER, 1, bz, "f64")
    floor = np.array([1.0, 1.0, 1.0, 0.01, 1.0, 1.0])
    diag = [i * (i + 1) // 2 + i for i in range(6)]
    d = np.sqrt(np.abs(f64["prior"][:, diag]))
    scale = np.concatenate([d[:, i:i + 1] * d[:, :i + 1] for i in range(6)], axis=1)  # packed (i, j <= i)

    def unpack(out):
        t = np.ascontiguousarray(out, np.float32).reshape(-1, 28, bsize)
        par = t[:, 0:6, :].transpose(0, 2, 1).reshape(-1, 6).astype(np.float64)
        cov = t[:, 6:27, :].transpose(0, 2, 1).reshape(-1, 21).astype(np.float64)
        return par, cov

    def errs(out, against=None, truth=None):
        """Quantiles of the relative errors of `out` against the FP64 oracle (or against another
        output), and the fractions of elements beyond the stated bars (1e-4 parameters, 1e-3
        covariance)."""
        par, cov = unpack(out)
        t64 = f64 if truth is None else truth
        tp, tc = (t64["par"], t64["cov"]) if against is None else unpack(against)
        ep = np.abs(par - tp) / np.maximum(np.abs(tp), floor)
        ec = np.abs(cov - tc) / np.maximum(np.abs(tc), scale)
        q = lambda e: {"p50": float(np.quantile(e, 0.5)), "p99": float(np.quantile(e, 0.99)), "max": float(e.max())}
        return {"par": q(ep), "cov": q(ec), "frac_par_beyond_1e-4": float((ep > 1e-4).mean()),
                "frac_cov_beyond_1e-3": float((ec > 1e-3).mean())}

    res = {"sample": f"event 0 of the bench workload ({nb * bsize} tracks x {NLAYER} layers, chained)",
           "oracle": "own FP64 restatement (oracle/), Bz as the workload", "this_library": errs(ours_ev),
           "bars": "fractions of elements beyond relative 1e-4 (parameters, floors 1 cm / 0.01 GeV^-1 / 1 rad) "
                   "and 1e-3 (covariance, scale max(|C_ij|, sqrt(P_ii P_jj)) with P the covariance entering the "
                   "last update)"}
    if ref_available(bsize, "kf"):
        ref = RefTBB(bsize, "kf")
        ref.set_bz(bz)
        ref_out = ref.run(trk_ev, hit_ev, 1, nb, NLAYER, True, 1, nthreads)
        res["reference_cpu"] = errs(ref_out)
        res["this_library_vs_reference_cpu"] = errs(ours_ev, against=ref_out)
    if ref_gpu_ev is not None:
        # the reference's GPU program has its field compiled in (kfact of 3.8112 T, TBB:654): its
        # output is compared with the FP64 oracle run at that field on the same inputs
        f64_ref_field = Oracle().run(trk_ev, hit_ev, bsize, NLAYER, 1, 3.8112, "f64")
        res["reference_gpu_cuda_v4"] = dict(errs(ref_gpu_ev, truth=f64_ref_field),
                                            oracle_field="3.8112 T, the program's compiled-in kfact")
    return res


def reference_gpu(p2r, torch, cfg, d_trk, d_hit, stream, steps, ours_chained_ms):
    """The reference's own CUDA kernels (compiled unmodified from its sources into oracle/_ref)
    timed with CUDA events on the same device-resident inputs as this library's fused kernel:
    GPUsequence (cuda_v4.cu:821-849, chained, against p2r_forward CHAINED) and launch_p2r_kernel
    (cuda_uvm.cu:887-915, restart, against p2r_forward RESTART). Returns the record and the
    chained kernel's output (for the accuracy comparison), or (None, None)."""
    from oracle.oracle import RefGPU, refgpu_available
    rec, out_v4 = {}, None
    for kind in ("v4", "uvm"):
        if not refgpu_available(kind):
            rec[kind] = {"unavailable": "oracle/_ref/libp2r_refgpu_" + kind + ".so missing"}
            continue
        r = RefGPU(kind)
        ne, nb, nl, bs = r.sizes()
        if (ne, nb, nl, bs) != (cfg.nevts, cfg.nb, cfg.nlayer, cfg.bsize):
            rec[kind] = {"unavailable": f"compiled for nevts={ne} nb={nb} nlayer={nl} bsize={bs}"}
            continue
        out = torch.empty_like(d_trk)
        ms = r.run(d_trk.data_ptr(), d_hit.data_ptr(), out.data_ptr(), 3, steps, stream.cuda_stream) / steps
        if r.chained:
            ours = ours_chained_ms
            out_v4 = out
            what = ("GPUsequence, src/propagate-tor-test_cuda_v4.cu:821-849: chained layer loop, one 32-thread "
                    "CTA per Matriplex block, scratch matrices in shared memory; against p2r_forward CHAINED")
            ups = cfg.ntracks * cfg.nlayer
        else:
            rcfg = dataclasses.replace(cfg, mode=p2r.MODE_RESTART)
            o2 = torch.empty_like(d_trk)
            for _ in range(3):
                p2r.forward(rcfg, d_trk, d_hit, o2, stream=stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                p2r.forward(rcfg, d_trk, d_hit, o2, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ours = e0.elapsed_time(e1) / steps
            torch.cuda.synchronize()
            same = torch.equal(torch.isfinite(out), torch.isfinite(o2))
            del o2
            what = ("launch_p2r_kernel, src/propagate-tor-test_cuda_uvm.cu:887-915: restart layer loop (every "
                    "layer starts from the input track, only the last result is stored, so the compiler may "
                    "drop the other layers), one thread per track; against p2r_forward RESTART (which computes "
                    "only the last layer)")
            ups = cfg.ntracks
        rec[kind] = {"kernel": what, "ms_per_pass": ms, "this_library_ms_per_pass": ours,
                     "speedup_of_this_library": ms / ours, "updates_per_s": ups / (ms / 1e3),
                     "steps": steps,
                     "build": "nvcc -gencode arch=compute_100a,code=sm_100a -std=c++17 -maxrregcount=64 -g -lineinfo "
                              "--expt-relaxed-constexpr (the reference's build.py:97 flags, sm_100a for sm_70), "
                              "-Dntrks=9600 -Dnevts=100 -Dnlayer=20 -Dbsize=32"}
        if not r.chained:
            rec[kind]["nonfinite_pattern_equal"] = bool(same)
        else:
            del out
    return rec, out_v4


def cpu_reference_rate(trk, hit, nevts, nb, bsize, budget_s, nthreads):
    """Times the reference's own driver loop (oracle/_ref) on a bounded sample of events.
    Returns (updates/s, sample description, kind, threads)."""
    from oracle.oracle import RefTBB, ref_available, host_isa
    kind = host_isa()
    if not ref_available(bsize, kind):
        raise RuntimeError("reference CPU build (oracle/_ref) is missing")
    ref = RefTBB(bsize, kind)
    tw = 28 * bsize * nb  # floats per event of tracks
    hw = 9 * bsize * nb * NLAYER
    # probe one event to size the sample
    t0 = time.perf_counter()
    ref.run_into(trk[:tw], hit[:hw], np.empty(tw, np.float32), 1, nb, NLAYER, True, 1, nthreads)
    t_ev = max(time.perf_counter() - t0, 1e-4)
    nev = int(min(nevts, max(1, budget_s / 3 / t_ev)))
    out = np.empty(nev * tw, np.float32)
    reps, done, t_tot = 0, 0, 0.0
    while t_tot < budget_s / 2 or reps == 0:
        t0 = time.perf_counter()
        ref.run_into(trk[: nev * tw], hit[: nev * hw], out, nev, nb, NLAYER, True, 1, nthreads)
        t_tot += time.perf_counter() - t0
        reps += 1
        done += nev * nb * bsize * NLAYER
        if reps >= 1000:
            break
    sample = (f"{reps} pass(es) of the chained reference loop over {nev} of {nevts} events "
              f"({nev * nb * bsize} tracks x {NLAYER} layers), {t_tot:.1f} s wall")
    return done / t_tot, sample, kind, nthreads


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # This arm maps no library of this package: the inputs come from the oracle's copy of the
    # workload generator (bit-identical to p2r_gen_helix), the timed loop is the reference's.
    nthreads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    from oracle.oracle import ref_available, host_isa, gen_helix
    if not ref_available(args.bsize, host_isa()):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref missing"}))
        return 0
    nb = NTRKS // args.bsize
    trk, hit = gen_helix(args.bsize, args.nevts, nb, NLAYER, seed=20240001, bz=BZ)
    trk, hit = trk.reshape(-1), hit.reshape(-1)
    from oracle.oracle import RefTBB
    ref = RefTBB(args.bsize, host_isa())
    tw, hw = 28 * args.bsize * nb, 9 * args.bsize * nb * NLAYER
    chained = args.mode == "chained"
    t0 = time.perf_counter()
    ref.run_into(trk[:tw], hit[:hw], np.empty(tw, np.float32), 1, nb, NLAYER, chained, 1, nthreads)
    t_ev = max(time.perf_counter() - t0, 1e-4)
    per_step = args.ref_budget / max(1, args.steps + args.warmup)
    nev = int(min(args.nevts, max(1, per_step / t_ev)))
    out = np.empty(nev * tw, np.float32)
    for _ in range(args.warmup):
        ref.run_into(trk[: nev * tw], hit[: nev * hw], out, nev, nb, NLAYER, chained, 1, nthreads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.run_into(trk[: nev * tw], hit[: nev * hw], out, nev, nb, NLAYER, chained, 1, nthreads)
        times.append(time.perf_counter() - t0)
    # restart: the reference's loop computes every layer but only the last reaches the output;
    # the metric counts the updates that reach it, as this library's restart arm does
    ups = nev * nb * args.bsize * (NLAYER if chained else 1)
    tot = sum(times)
    value = ups * len(times) / tot
    sample = f"{nev} of {args.nevts} events per step ({nev * nb * args.bsize} tracks x {NLAYER} layers, {args.mode})"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "track-layer updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "track-layer updates/s", "cores": nthreads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "track-layer updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "mapped_libraries": mapped_in_tree_libraries(),
    }
    print(json.dumps(line))
    return 0


def mapped_in_tree_libraries() -> list[str]:
    """Shared libraries under this directory mapped into the process (from /proc/self/maps)."""
    found = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and path.startswith(str(ROOT)):
                    found.add(os.path.relpath(path, ROOT))
    except OSError:
        return []
    return sorted(found)


def workload_config(args):
    what = ("propagateToR + KalmanUpdate per layer" if args.mode == "chained" else
            "the reference's restart loop: every layer restarts from the input track and rewrites the "
            "output, so only the last layer is computed, one propagateToR + KalmanUpdate per track")
    return {"workload": f"fused {args.mode} p2r forward ({what}), "
                        f"{NTRKS} tracks x {args.nevts} events x {NLAYER} layers per GPU",
            "ntrks": NTRKS, "nevts": args.nevts, "nlayer": NLAYER, "bsize": args.bsize, "bz_tesla": BZ,
            "mode": args.mode, "generator": "p2r_gen_helix defaults (seeded synthetic helices)",
            "l2": l2_note(args.nevts)}


def l2_note(nevts: int) -> str:
    """Whether one step's inputs exceed the 126 MB L2 (then no flush is needed between steps)."""
    gb = NTRKS * nevts * (28 * 4 + NLAYER * 9 * 4) / 1e9
    if gb * 1e3 > 126:
        return f"inputs ({gb:.2f} GB per GPU) larger than the 126 MB L2; no flush"
    return (f"inputs ({gb * 1e3:.0f} MB per GPU) fit in the 126 MB L2 and are not flushed: "
            "a profiling size, not a bench measurement")


# ------------------------------------------------------------------ our arm
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import torch.distributed as dist
    import p2r_tests_b200 as p2r

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    cfg, trk, hit = make_inputs(p2r, args.nevts, args.bsize, 20240001 + rank)
    cfg.mode = p2r.MODE_CHAINED if args.mode == "chained" else p2r.MODE_RESTART
    d_trk = torch.from_numpy(trk.reshape(-1)).to(dev)
    d_hit = torch.from_numpy(hit.reshape(-1)).to(dev)
    d_out = torch.empty_like(d_trk)
    stream = torch.cuda.current_stream(dev)
    # track-layer updates computed per step per GPU. Restart: the reference's restart loop
    # rewrites the output at every layer from the same input track (TBB:870-926), so only the
    # last layer reaches the output and only that one is computed: one update per track.
    restart = cfg.mode == p2r.MODE_RESTART
    updates = cfg.ntracks * (1 if restart else NLAYER)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # warm-up
    for _ in range(max(3, args.warmup)):
        p2r.forward(cfg, d_trk, d_hit, d_out, stream=stream)
    torch.cuda.synchronize()

    # timed region: exactly K steps of the fused kernel
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.2)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        p2r.forward(cfg, d_trk, d_hit, d_out, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    t_ms = max_over_ranks(e0.elapsed_time(e1))
    ms_per_step = t_ms / args.steps
    value = world * updates * args.steps / (t_ms / 1e3)
    nonfinite = p2r.count_nonfinite(d_out, cfg.nblocks, cfg.bsize)

    # roofline of the fused kernel (the only kernel of a step): FP32 compute
    t_launch = ms_per_step / 1e3
    flops = FLOP_PER_UPDATE * updates
    achieved_tflops = flops / t_launch / 1e12
    probe_out = torch.empty(148 * 8 * 256, dtype=torch.float32, device=dev)
    probe_peaks = {}
    for packed in (False, True):  # scalar FFMA and packed f32x2 FMA; the larger is the peak
        p2r.fp32_fma_probe(probe_out, 2000, 148 * 8, 256, stream=stream, packed=packed)
        torch.cuda.synchronize()
        pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        pe0.record(stream)
        pflops = 0
        for _ in range(5):
            pflops += p2r.fp32_fma_probe(probe_out, 20000, 148 * 8, 256, stream=stream, packed=packed)
        pe1.record(stream)
        torch.cuda.synchronize()
        probe_peaks["f32x2" if packed else "f32"] = pflops / (pe0.elapsed_time(pe1) / 1e3) / 1e12
    fp32_peak = max(probe_peaks.values())
    # the FP64 FMA peak: the denominator of the FP64 adjoint's roofline
    probe64 = torch.empty(148 * 8 * 256, dtype=torch.float64, device=dev)
    p2r.fp64_fma_probe(probe64, 200, 148 * 8, 256, stream=stream)
    torch.cuda.synchronize()
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record(stream)
    pflops = sum(p2r.fp64_fma_probe(probe64, 2000, 148 * 8, 256, stream=stream) for _ in range(5))
    pe1.record(stream)
    torch.cuda.synchronize()
    fp64_peak = pflops / (pe0.elapsed_time(pe1) / 1e3) / 1e12
    del probe64
    alg_bytes = cfg.ntracks * (36 * (1 if restart else NLAYER) + 224)
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs")
    traffic = traffic_from_profiles(args.mode)

    # forward + adjoint (p2r_forward_backward: fused chained forward with checkpoints and
    # the hand-written reverse sweep, plus the deterministic reduction of the shared
    # gradients) against the plain fused forward, on the same workload
    adjoint = None
    if not args.no_adjoint and not restart:  # the adjoint is of the chained loop
        g_trk = torch.randn(d_trk.numel(), dtype=torch.float32, device=dev, generator=torch.Generator(dev).manual_seed(1))
        g_chi2 = torch.ones(cfg.ntracks, dtype=torch.float32, device=dev)
        d_dr = torch.zeros(NLAYER, dtype=torch.float32, device=dev)
        adjoint = {"ckpt_stride": {}, "steps": args.adj_steps}
        ws = {}
        for ck in (1, 5, 10):
            for _ in range(2):
                p2r.forward_backward(cfg, d_trk, d_hit, dr=d_dr, grad_trk_out=g_trk, grad_chi2=g_chi2,
                                     ckpt_stride=ck, stream=stream, out=ws)
            torch.cuda.synchronize()
            barrier()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(args.adj_steps):
                p2r.forward_backward(cfg, d_trk, d_hit, dr=d_dr, grad_trk_out=g_trk, grad_chi2=g_chi2,
                                     ckpt_stride=ck, stream=stream, out=ws)
            a1.record(stream)
            torch.cuda.synchronize()
            barrier()
            ams = max_over_ranks(a0.elapsed_time(a1)) / args.adj_steps
            adjoint["ckpt_stride"][str(ck)] = {"ms_per_step": ams, "ratio_vs_forward": ams / ms_per_step}
        # the same kernels instantiated in FP32 (P2R_FLAG_ADJ_FP32): the cost of the structure
        # without FP64 arithmetic; its gradients do not meet the 1e-3 bar (reported, not the result)
        cfg32 = dataclasses.replace(cfg, flags=cfg.flags | p2r.FLAG_ADJ_FP32)
        ws32, fp32 = {}, {}
        for ck in (1, 5):
            for _ in range(2):
                p2r.forward_backward(cfg32, d_trk, d_hit, dr=d_dr, grad_trk_out=g_trk, grad_chi2=g_chi2,
                                     ckpt_stride=ck, stream=stream, out=ws32)
            torch.cuda.synchronize()
            barrier()
            a0.record(stream)
            for _ in range(args.adj_steps):
                p2r.forward_backward(cfg32, d_trk, d_hit, dr=d_dr, grad_trk_out=g_trk, grad_chi2=g_chi2,
                                     ckpt_stride=ck, stream=stream, out=ws32)
            a1.record(stream)
            torch.cuda.synchronize()
            barrier()
            ams = max_over_ranks(a0.elapsed_time(a1)) / args.adj_steps
            fp32[str(ck)] = {"ms_per_step": ams, "ratio_vs_forward": ams / ms_per_step}
        # thread-local checkpoints (the smallest workspace; the path of the allocation-free
        # entry point)
        tl, wstl = {}, {}
        for ck in (5, 10):
            for _ in range(2):
                p2r.forward_backward(cfg, d_trk, d_hit, dr=d_dr, grad_trk_out=g_trk, grad_chi2=g_chi2,
                                     ckpt_stride=ck, stream=stream, out=wstl, tape=False)
            torch.cuda.synchronize()
            barrier()
            a0.record(stream)
            for _ in range(args.adj_steps):
                p2r.forward_backward(cfg, d_trk, d_hit, dr=d_dr, grad_trk_out=g_trk, grad_chi2=g_chi2,
                                     ckpt_stride=ck, stream=stream, out=wstl, tape=False)
            a1.record(stream)
            torch.cuda.synchronize()
            barrier()
            ams = max_over_ranks(a0.elapsed_time(a1)) / args.adj_steps
            tl[str(ck)] = {"ms_per_step": ams, "ratio_vs_forward": ams / ms_per_step}
        adjoint["thread_local_checkpoints"] = {"ckpt_stride": tl, "workspace_bytes": p2r.workspace_size(cfg)}
        del wstl
        adjoint["fp32_instance"] = {"ckpt_stride": fp32,
                                    "gradient_error_vs_fp64": fp32_gradient_error(ws, ws32, cfg.bsize),
                                    "note": "P2R_FLAG_ADJ_FP32, same tape kernels in float: the gradient error "
                                            "against the FP64 instance (which matches FP64 finite differences "
                                            "to ~1e-8) is above the 1e-3 bar"}
        del ws, ws32
        best = min(adjoint["ckpt_stride"], key=lambda k: adjoint["ckpt_stride"][k]["ms_per_step"])
        adjoint["ratio_vs_forward"] = adjoint["ckpt_stride"][best]["ratio_vs_forward"]
        f64u = fp64_flop_per_update()
        if f64u and best == "1":  # the executed FP64 work is counted for the stride-1 tape kernels
            a64 = f64u * updates / (adjoint["ckpt_stride"]["1"]["ms_per_step"] / 1e3) / 1e12
            adjoint["roofline_fp64"] = {
                "bound": "fp64", "achieved": a64, "peak": fp64_peak, "unit": "TFLOP/s", "frac": a64 / fp64_peak,
                "fp64_flop_per_update": f64u,
                "peak_source": "measured in this run: p2r_fp64_fma_probe (DFMA), full occupancy",
                "flop_source": "executed DADD + DMUL + 2 DFMA per track-layer of fwd_tape_kernel + "
                               "rev_tape_kernel<double, 1>, ncu counters (profiles/tape_adjoint_fp64_ck1_9600x8x20.md)"}
        adjoint["best_ckpt_stride"] = int(best)
        adjoint["definition"] = ("time of p2r_forward_backward in FP64 (forward outputs + gradients w.r.t. initial "
                                 "parameters/covariance, hits, per-layer dr and Bz of sum(g.out) + sum(chi2)), "
                                 "checkpoint tape in device memory, divided by the plain FP32 p2r_forward time")

    # bsize sweep of the fused forward (same tracks re-laid out; autotuned launch shape)
    sweep = None
    if not args.no_sweep and world == 1:
        from p2r_tests_b200 import autotune
        r = autotune.tune_forward(cfg, trk, hit, bsizes=(32, 64, 128), threads=(64, 96, 128), stages=(2, 4),
                                  reps=20, use_cache=False)
        sweep = {}
        for t in r["tried"]:
            k = str(t["bsize"])
            ups = updates / (t["ms"] / 1e3)
            if k not in sweep or ups > sweep[k]["updates_per_s"]:
                sweep[k] = {"updates_per_s": ups, "ms": t["ms"], "block_threads": t["block_threads"],
                            "stages": t["stages"]}

    # uneven batch: 1000 events by default (--uneven-events), log-normal track counts, 10-25 layers per track, one
    # persistent queue launch captured in a CUDA graph, launch shape picked by the autotuner
    uneven = None
    if not args.no_uneven and world == 1:
        from p2r_tests_b200 import autotune
        counts = p2r.lognormal_counts(args.uneven_events, median=2000, sigma=1.0, lo=50, hi=20000, seed=7)
        wl = {bs: p2r.uneven_workload(counts, bsize=bs, nlayer_max=25) for bs in (32, 64)}
        tq = autotune.tune_queue(counts, bsizes=(32, 64), granularity=(1, 4, 8, 16), threads=(64, 128),
                                 stages=(4,), reps=3, use_cache=False, workloads=wl)
        w = wl[tq["bsize"]]
        qflags = p2r.FLAG_ORDER_BY_LAYERS if tq.get("order") else 0
        q = p2r.Queue(w, blocks_per_item=tq["blocks_per_item"], block_threads=tq["block_threads"],
                      stages=tq["stages"], flags=qflags)
        qt = torch.from_numpy(w["trk"].reshape(-1)).to(dev)
        qh = torch.from_numpy(w["hit"].reshape(-1)).to(dev)
        qo = torch.empty_like(qt)
        q.capture(qt, qh, qo)
        for _ in range(3):
            q.replay(stream)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(args.uneven_steps):
            q.replay(stream)
        g1.record(stream)
        torch.cuda.synchronize()
        gms = g0.elapsed_time(g1) / args.uneven_steps
        lat = q.event_latency_ns() / 1e6
        qref = qo.cpu().numpy()
        q.release()
        # the same tracks ordered by layer count within each event (p2r.sort_by_layers): warps
        # of tracks with similar lengths idle less; per-track results are bit-identical
        ws_, perm = p2r.sort_by_layers(w)
        qs = p2r.Queue(ws_, blocks_per_item=tq["blocks_per_item"], block_threads=tq["block_threads"],
                       stages=tq["stages"], flags=qflags)
        st_, sh_ = torch.from_numpy(ws_["trk"].reshape(-1)).to(dev), torch.from_numpy(ws_["hit"].reshape(-1)).to(dev)
        so_ = torch.empty_like(st_)
        qs.capture(st_, sh_, so_)
        for _ in range(3):
            qs.replay(stream)
        torch.cuda.synchronize()
        g0.record(stream)
        for _ in range(args.uneven_steps):
            qs.replay(stream)
        g1.record(stream)
        torch.cuda.synchronize()
        sms = g0.elapsed_time(g1) / args.uneven_steps
        back = p2r.permute_tracks(so_.cpu().numpy(), p2r.inverse(perm), tq["bsize"], 28)
        same = bool(np.array_equal(back.view(np.uint32).reshape(-1), qref.view(np.uint32).reshape(-1)))
        qs.release()
        del st_, sh_, so_, ws_
        uneven = {"workload": f"{args.uneven_events} events, tracks/event log-normal (median 2000, sigma 1.0) clipped to "
                              "[50, 20000], layers/track uniform 10..25, chained",
                  "tracks": int(counts.sum()), "updates": w["updates"], "bsize": tq["bsize"],
                  "blocks_per_item": tq["blocks_per_item"], "block_threads": tq["block_threads"],
                  "stages": tq["stages"], "ordered_in_launch": bool(qflags),
                  "best_unordered": min(({"ms": x["ms"], "updates_per_s": x["updates_per_s"], "bsize": x["bsize"],
                                          "blocks_per_item": x["blocks_per_item"], "block_threads": x["block_threads"]}
                                         for x in tq["tried"] if not x.get("order")), key=lambda x: x["ms"],
                                        default=None),
                  "ms_per_step": gms, "updates_per_s": w["updates"] / (gms / 1e3),
                  "p50_event_ms": float(np.percentile(lat, 50)), "p99_event_ms": float(np.percentile(lat, 99)),
                  "launch": "CUDA graph (queue init + one persistent kernel" +
                            (", each CTA ordering its tracks by layer count in the launch)" if qflags else ")"),
                  "steps": args.uneven_steps,
                  "autotune_candidates": len(tq["tried"]),
                  "sorted_by_layer_count": {"ms_per_step": sms, "updates_per_s": w["updates"] / (sms / 1e3),
                                            "outputs_identical_per_track": same,
                                            "how": "each event's tracks ordered by layer count (p2r.sort_by_layers)"}}
        del qt, qh, qo, wl

    # calibration workload: 1e5 tracks x 100 events x 40 layers (r = 4..110 cm), generated on
    # the device, 20-40 layers per track, radius offsets of +-100 um; the forward alone
    # (masked fused forward) and forward + adjoint with per-event chi2 gradients w.r.t. the 40
    # offsets and Bz, captured once in a CUDA graph and replayed
    calib = None
    if not args.no_calib and world == 1:
        c4 = p2r.Config(bsize=32, nlayer=40, nevts=args.calib_nevts, nb=3125, bz=BZ)
        gp4 = p2r.gen_params(bz=BZ, seed=20240004, r_first=4.0, r_last=110.0)
        gen0, gen1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        gen0.record(stream)
        t4, h4 = p2r.generate_helix_device(c4, gp4, stream=stream)
        gen1.record(stream)
        g4 = torch.Generator(dev).manual_seed(4)
        nl4 = torch.randint(20, 41, (c4.ntracks,), dtype=torch.int32, device=dev, generator=g4)
        dr4 = (torch.rand(c4.nlayer, device=dev, generator=g4) * 0.02 - 0.01).contiguous()
        upd4 = int(nl4.sum().item())
        o4 = torch.empty_like(t4)
        for _ in range(2):
            p2r.forward(c4, t4, h4, o4, dr=dr4, nlay_lane=nl4, stream=stream)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.calib_steps):
            p2r.forward(c4, t4, h4, o4, dr=dr4, nlay_lane=nl4, stream=stream)
        f1.record(stream)
        torch.cuda.synchronize()
        fms = f0.elapsed_time(f1) / args.calib_steps
        # the same tracks ordered by layer count within each event (fewer idle lanes per warp)
        t4s, h4s, nl4s, _ = p2r.sort_by_layers_device(c4, t4, h4, nl4)
        for _ in range(2):
            p2r.forward(c4, t4s, h4s, o4, dr=dr4, nlay_lane=nl4s, stream=stream)
        torch.cuda.synchronize()
        f0.record(stream)
        for _ in range(args.calib_steps):
            p2r.forward(c4, t4s, h4s, o4, dr=dr4, nlay_lane=nl4s, stream=stream)
        f1.record(stream)
        torch.cuda.synchronize()
        fms_sorted = f0.elapsed_time(f1) / args.calib_steps
        # the masked forward with each CTA's tracks ordered by layer count inside the launch
        c4f = dataclasses.replace(c4, flags=c4.flags | p2r.FLAG_ORDER_BY_LAYERS)
        for _ in range(2):
            p2r.forward(c4f, t4, h4, o4, dr=dr4, nlay_lane=nl4, stream=stream)
        torch.cuda.synchronize()
        f0.record(stream)
        for _ in range(args.calib_steps):
            p2r.forward(c4f, t4, h4, o4, dr=dr4, nlay_lane=nl4, stream=stream)
        f1.record(stream)
        torch.cuda.synchronize()
        fms_ordered = f0.elapsed_time(f1) / args.calib_steps
        del o4
        gc4 = torch.ones(c4.ntracks, dtype=torch.float32, device=dev)
        out4 = {"grad_trk_in": None, "grad_hits": None}
        # checkpoint stride: 1 (the whole state tape, the fastest reverse) when its workspace fits
        # in 70 % of the free device memory, else 5
        torch.cuda.empty_cache()
        free4, _ = torch.cuda.mem_get_info(dev)
        ck4 = 1 if p2r.workspace_size(c4, 1) <= 0.7 * free4 else 5
        p2r.forward_backward(c4, t4, h4, dr=dr4, nlay_lane=nl4, grad_chi2=gc4, per_event=True, out=out4,
                             ckpt_stride=ck4, stream=stream)
        torch.cuda.synchronize()
        graph4 = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(device=dev)  # capture needs a non-default stream; replays run on the current one
        with torch.cuda.graph(graph4, stream=cap):
            p2r.forward_backward(c4, t4, h4, dr=dr4, nlay_lane=nl4, grad_chi2=gc4, per_event=True, out=out4,
                                 ckpt_stride=ck4, stream=cap)
        graph4.replay()
        torch.cuda.synchronize()
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for _ in range(args.calib_steps):
            graph4.replay()
        b1.record(stream)
        torch.cuda.synchronize()
        bms = b0.elapsed_time(b1) / args.calib_steps
        # the same forward + adjoint on the tracks ordered by layer count (same workspace)
        out4s = {"grad_trk_in": None, "grad_hits": None, "workspace": out4["workspace"]}
        p2r.forward_backward(c4, t4s, h4s, dr=dr4, nlay_lane=nl4s, grad_chi2=gc4, per_event=True, out=out4s,
                             ckpt_stride=ck4, stream=stream)
        torch.cuda.synchronize()
        b0.record(stream)
        for _ in range(args.calib_steps):
            p2r.forward_backward(c4, t4s, h4s, dr=dr4, nlay_lane=nl4s, grad_chi2=gc4, per_event=True, out=out4s,
                                 ckpt_stride=ck4, stream=stream)
        b1.record(stream)
        torch.cuda.synchronize()
        bms_sorted = b0.elapsed_time(b1) / args.calib_steps
        dr_rel = float(((out4s["grad_dr"] - out4["grad_dr"]).abs().max() / out4["grad_dr"].abs().max()).item())
        del out4s, t4s, h4s, nl4s
        # the grid path with the ordering inside the call (P2R_FLAG_ORDER_BY_LAYERS: the order is
        # computed on the device and the kernels read each position's track through it), in a graph
        ref_dr, ref_ev, ref_bz = (out4["grad_dr"].clone(), out4["grad_dr_event"].clone(),
                                  out4["grad_bz_event"].clone())
        ev_ok = bool(torch.allclose(out4["grad_dr_event"].sum(0), out4["grad_dr"], rtol=1e-10, atol=0))
        del graph4
        out4["workspace"] = None  # the ordered call's workspace is 4 bytes per track larger
        torch.cuda.empty_cache()
        c4o = dataclasses.replace(c4, flags=c4.flags | p2r.FLAG_ORDER_BY_LAYERS)
        out4o = {"grad_trk_in": None, "grad_hits": None}
        p2r.forward_backward(c4o, t4, h4, dr=dr4, nlay_lane=nl4, grad_chi2=gc4, per_event=True, out=out4o,
                             ckpt_stride=ck4, stream=stream)
        torch.cuda.synchronize()
        graph4o = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph4o, stream=cap):
            p2r.forward_backward(c4o, t4, h4, dr=dr4, nlay_lane=nl4, grad_chi2=gc4, per_event=True, out=out4o,
                                 ckpt_stride=ck4, stream=cap)
        graph4o.replay()
        torch.cuda.synchronize()
        b0.record(stream)
        for _ in range(args.calib_steps):
            graph4o.replay()
        b1.record(stream)
        torch.cuda.synchronize()
        bms_ord = b0.elapsed_time(b1) / args.calib_steps
        ord_rel = float(((out4o["grad_dr_event"] - ref_ev).abs().max() / ref_ev.abs().max()).item())
        ws_ord = int(out4o["workspace"].numel())
        del graph4o, out4o, out4
        torch.cuda.empty_cache()
        # the same forward + adjoint in ONE persistent launch over the work queue (per-warp tapes,
        # the workspace bounded by the resident warps), captured in a CUDA graph; plain and with
        # each event's tracks ordered by layer count inside the launch
        wq = {"event_block_offset": np.arange(c4.nevts + 1, dtype=np.int64) * c4.nb,
              "nlay_lane": nl4.cpu().numpy(), "nblocks": c4.nblocks, "bsize": c4.bsize, "nlayer": c4.nlayer,
              "bz": c4.bz}
        qadj = {}
        for name, fl in (("plain", 0), ("ordered_by_layers", p2r.FLAG_ORDER_BY_LAYERS)):
            qa = p2r.Queue(wq, blocks_per_item=4, flags=fl)
            oq = qa.capture_adjoint(t4, h4, dr=dr4, grad_chi2=gc4, out={"grad_trk_in": None, "grad_hits": None})
            qa.replay(stream)
            torch.cuda.synchronize()
            b0.record(stream)
            for _ in range(args.calib_steps):
                qa.replay(stream)
            b1.record(stream)
            torch.cuda.synchronize()
            qms = b0.elapsed_time(b1) / args.calib_steps
            qadj[name] = {
                "ms_per_step": qms, "ratio_vs_forward": qms / fms, "updates_per_s": upd4 / (qms / 1e3),
                "workspace_bytes": int(oq["workspace"].numel()), "queue_errors": qa.error_bits(stream),
                "grad_dr_event_max_rel_diff_vs_grid_path": float(
                    ((oq["grad_dr_event"] - ref_ev).abs().max() / ref_ev.abs().max()).item()),
                "grad_bz_event_max_rel_diff_vs_grid_path": float(
                    ((oq["grad_bz_event"] - ref_bz).abs().max() / ref_bz.abs().max()).item())}
            qa.release()
            del oq, qa
        del wq
        calib = {"workload": f"{c4.ntracks // c4.nevts} tracks x {c4.nevts} events x 40 layers, hits on r = 4..110 cm, "
                             "20-40 layers per track (uniform), dr ~ U[-100, 100] um, generated on the device",
                 "hits_bytes": h4.numel() * 4, "tracks_bytes": t4.numel() * 4, "updates": upd4,
                 "device_generation_ms": gen0.elapsed_time(gen1),
                 "forward": {"ms_per_step": fms, "updates_per_s": upd4 / (fms / 1e3),
                             "api": "p2r_forward_masked (fused, per-track layer counts)",
                             "sorted_by_layer_count": {"ms_per_step": fms_sorted,
                                                       "updates_per_s": upd4 / (fms_sorted / 1e3)},
                             "ordered_in_launch": {"ms_per_step": fms_ordered,
                                                   "updates_per_s": upd4 / (fms_ordered / 1e3),
                                                   "how": "P2R_FLAG_ORDER_BY_LAYERS: each CTA orders its "
                                                          "chunk of 256 tracks by layer count"}},
                 "forward_adjoint": {
                     "ms_per_step": qadj["ordered_by_layers"]["ms_per_step"],
                     "ratio_vs_forward": qadj["ordered_by_layers"]["ratio_vs_forward"],
                     "ratio_vs_forward_sorted": qadj["ordered_by_layers"]["ms_per_step"] / fms_sorted,
                     "api": "p2r_queue_adjoint_graph_create (P2R_FLAG_ORDER_BY_LAYERS): one CUDA graph of the "
                            "workspace clears, the per-event ordering by layer count, ONE persistent FP64 "
                            "forward + adjoint launch over the work queue, and the fixed-order per-event sums",
                     "persistent_queue": qadj},
                 "forward_adjoint_grid_path": {"ms_per_step": bms, "ratio_vs_forward": bms / fms, "ckpt_stride": ck4,
                                     "workspace_bytes": p2r.workspace_size(c4, ck4),
                                     "sorted_by_layer_count": {
                                         "ms_per_step": bms_sorted,
                                         "grad_dr_max_rel_diff_vs_unsorted": dr_rel,
                                         "how": "each event's tracks ordered by layer count (p2r.sort_by_layers_device), "
                                                "direct calls"},
                                     "ordered_in_call": {
                                         "ms_per_step": bms_ord, "ratio_vs_forward": bms_ord / fms,
                                         "workspace_bytes": ws_ord,
                                         "grad_dr_event_max_rel_diff_vs_unordered": ord_rel,
                                         "how": "P2R_FLAG_ORDER_BY_LAYERS: order computed on the device inside "
                                                "the call, replayed from one CUDA graph"},
                                     "api": f"p2r_forward_backward (FP64, ckpt {ck4}), per-event grad_dr/grad_bz, "
                                            "replayed from one CUDA graph"},
                 "per_event_sum_matches_total": ev_ok,
                 "steps": args.calib_steps}
        del t4, h4, nl4, gc4

    # end to end through the host-buffer C-ABI call: H2D + kernels + D2H every step
    h_trk = torch.from_numpy(trk.reshape(-1)).pin_memory().numpy()
    h_hit = torch.from_numpy(hit.reshape(-1)).pin_memory().numpy()
    h_out = torch.empty(trk.size, dtype=torch.float32).pin_memory().numpy()
    for _ in range(2):
        p2r.forward_host(cfg, h_trk, h_hit, h_out, d_trk, d_hit, d_out, nchunks=10, stream=stream)
    torch.cuda.synchronize()
    barrier()
    x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    for _ in range(args.e2e_steps):
        p2r.forward_host(cfg, h_trk, h_hit, h_out, d_trk, d_hit, d_out, nchunks=10, stream=stream)
    x1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(x0.elapsed_time(x1))
    e2e_value = world * updates * args.e2e_steps / (e2e_ms / 1e3)
    ok = np.array_equal(h_out.view(np.uint32), d_out.cpu().numpy().view(np.uint32))
    # the link the end-to-end call is bound by: one whole-buffer pinned copy each way, same bytes
    ht, hh, ho = torch.from_numpy(h_trk), torch.from_numpy(h_hit), torch.from_numpy(h_out)
    with torch.cuda.stream(stream):
        c0, c1, c2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        for rep in range(3):
            c0.record(stream)
            d_trk.copy_(ht, non_blocking=True)
            d_hit.copy_(hh, non_blocking=True)
            c1.record(stream)
            ho.copy_(d_out, non_blocking=True)
            c2.record(stream)
        torch.cuda.synchronize()
    h2d_gbs = (trk.nbytes + hit.nbytes) / (c0.elapsed_time(c1) / 1e3) / 1e9
    # bytes the end-to-end call copies in: restart mode copies only the last layer's hits
    h2d_step = trk.nbytes + (hit.nbytes // NLAYER if restart else hit.nbytes)
    d2h_gbs = trk.nbytes / (c1.elapsed_time(c2) / 1e3) / 1e9
    e2e_s = e2e_ms / 1e3 / args.e2e_steps
    pcie = {"h2d_gbs_measured": h2d_gbs, "d2h_gbs_measured": d2h_gbs,
            "achieved_h2d_gbs": h2d_step / e2e_s / 1e9,
            "frac": h2d_step / e2e_s / 1e9 / h2d_gbs,
            "how": "one whole-buffer pinned cudaMemcpyAsync per direction (torch copy_), after the "
                   "end-to-end steps; frac = the end-to-end step's H2D bytes / its time, over h2d_gbs_measured"}

    # the reference's own CUDA kernels on this GPU, same inputs (1-GPU runs of the default workload)
    ref_gpu, ref_gpu_out = None, None
    if world == 1 and not restart and not args.no_reference_gpu:
        try:
            ref_gpu, ref_gpu_out = reference_gpu(p2r, torch, cfg, d_trk, d_hit, stream, min(args.steps, 200),
                                                 ms_per_step)
        except Exception as exc:  # reported, not fatal
            ref_gpu = {"unavailable": str(exc)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not restart:  # timed on the chained loop
        try:
            nthreads = len(os.sched_getaffinity(0))
            v, sample, kind, thr = cpu_reference_rate(trk.reshape(-1), hit.reshape(-1), args.nevts, cfg.nb,
                                                      cfg.bsize, args.cpu_seconds, nthreads)
            cpu = {"value": v, "unit": "track-layer updates/s", "cores": thr, "kind": "reference",
                   "sample": sample + f"; reference build oracle/_ref ({kind}), Bz compiled in at 3.8112 T"}
            tw, hw = 28 * cfg.bsize * cfg.nb, 9 * cfg.bsize * cfg.nb * NLAYER
            cpu["accuracy_vs_fp64"] = accuracy_vs_fp64(
                trk.reshape(-1)[:tw], hit.reshape(-1)[:hw], d_out[:tw].cpu().numpy(), cfg.nb, cfg.bsize, BZ,
                nthreads, None if ref_gpu_out is None else ref_gpu_out[:tw].cpu().numpy())
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": "track-layer updates/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "track-layer updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args),
            "roofline": {"bound": "fp32", "achieved": achieved_tflops, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved_tflops / fp32_peak,
                         "traffic": traffic,
                         "peak_source": "measured in this run: the larger of p2r_fp32_fma_probe (FFMA) and "
                                        "p2r_fp32x2_fma_probe (packed f32x2 FMA), full occupancy; "
                                        f"nominal {NOMINAL_FP32_TFLOPS:.1f} at 1965 MHz",
                         "probe_tflops": probe_peaks,
                         "frac_of_nominal": achieved_tflops / NOMINAL_FP32_TFLOPS,
                         "flop_per_update": FLOP_PER_UPDATE, "updates_per_launch": updates,
                         "launch_ms": ms_per_step},
            "roofline_hbm": {"bound": "hbm", "achieved": alg_bytes / t_launch / 1e9,
                             "peak": hbm_peak, "unit": "GB/s",
                             "frac": (alg_bytes / t_launch / 1e9 / hbm_peak) if hbm_peak else None,
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                             "algorithmic_bytes_per_launch": alg_bytes},
            "e2e": {"value": e2e_value, "unit": "track-layer updates/s",
                    "h2d_bytes_per_step": int(h2d_step), "d2h_bytes_per_step": int(trk.nbytes),
                    "steps": args.e2e_steps, "api": "p2r_forward_host (pinned host buffers, 10 chunks)",
                    "output_matches_device_run": bool(ok), "pcie": pcie},
            "fwd_adjoint": adjoint,
            "bsize_sweep": sweep,
            "uneven_batch": uneven,
            "calibration_40_layers": calib,
            "reference_gpu": ref_gpu,
            "gpu_launches": args.steps,
            "clocks": clk,
            "nonfinite_tracks": nonfinite,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
        sys.stdout.flush()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
