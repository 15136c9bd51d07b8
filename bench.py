"""Benchmark: FP64 point-iterations/s of the implicit q-LSKUM iteration.

A step is one ``fpi_solver`` iteration (all seven phases) over one point
cloud resident on the GPU.  The default workload is the 1.1M-point sphere
(96 shells x 11,500 points, 1% jitter, M = 0.8, alpha = 2 deg, FP64); the
cloud is seeded synthetic data from the package generator.  Its state
(~1.5 GB) is larger than the 126 MB L2, so no flush is needed between steps.

``value``    device-timed throughput with the state resident in HBM
             (CUDA events on the library's stream, max over ranks).
``e2e``      the same metric through the C ABI with host buffers: every step
             copies prim and delU in from pinned host memory (mfcfd_set_state),
             iterates (mfcfd_fpi_step) and copies them back (mfcfd_get_state).
``roofline`` the dominant phase's algorithmic bytes (per point, from the
             byte model of each phase) over its event-timed duration.
Multi-GPU: independent replicas, one per rank (the LU-SGS sweep order is
global, so one cloud does not shard); value sums the ranks' points.

``--impl reference`` times the CPU oracle (the reference's algorithm restated
in C++, glibc libm) instead: one independent solve per host core on a 62,400
point sphere sample, one iteration per step.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "3d-mfcfd_b200")
for _p in (PKG, REPO):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

# Algorithmic bytes per point-iteration of each phase (FP64 SoA model: own
# point inputs read once, outputs written once, neighbour gathers counted as
# cache hits; 26-neighbour interior point).
PHASE_BYTES = {"qderiv": 372 + 180, "flux": 724, "dinv": 488, "sweep_fwd": 608,
               "sweep_bwd": 608, "update": 196, "residual": 8}
TOTAL_BYTES = 3368
# DRAM bytes (read + write) per swept point of one chain-sweep launch, from
# the ncu capture of the 62,400-point sphere's forward sweep (161.96 MB per
# launch, profiles/ncu_k_sweep_chain_sphere62k.txt); traffic grows with the
# point count, so a launch of n points moves about n times this.
SWEEP_TRAFFIC_PER_POINT = 161.96e6 / 62400

WORKLOADS = {
    "sphere-1.1M": dict(shells=96, per_shell=11500, jitter=0.01, mach=0.8, aoa=2.0, seed=2001),
    "sphere-62k": dict(shells=48, per_shell=1300, jitter=0.02, mach=0.4, aoa=0.0, seed=1001),
}
# kernels of one iteration per sweep mode (2 chains: k_qderiv, k_pending,
# k_flux, two k_sweep_chain, k_update, two reductions; 0/1 add k_dinv_gold)
KERNELS_PER_ITER = {2: 8, 0: 9, 1: 9}


def load_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


# ------------------------------------------------------------------ CPU side

def _cpu_worker(args):
    """One independent CPU solve (spawned process): time `steps` iterations.

    Runs the reference itself (its Fortran routines translated to C,
    oracle/_ref/libref.so, glibc libm) when that build is present, else the
    C++ restatement of it."""
    sys.path.insert(0, PKG)
    sys.path.insert(0, REPO)
    from mfcfd import cloud
    from oracle import oracle, ref_translated
    shells, per_shell, jitter, mach, aoa, seed, warm, steps = args
    c = cloud.shell_cloud(shells, per_shell, jitter=jitter, seed=seed)
    prim0 = cloud.initial_state(c, mach, aoa)
    if ref_translated.available("glibc"):
        o, kind = ref_translated.TranslatedReference(c, prim0, mach, aoa), "reference"
    else:
        o, kind = oracle.Oracle(c, mach, aoa, libm=oracle.LIBM_GLIBC), "port"
        o.set_prim(prim0)
    for t in range(1, warm + 1):
        o.step(t)
    t0 = time.perf_counter()
    for t in range(warm + 1, warm + steps + 1):
        o.step(t)
    return c.n, steps, time.perf_counter() - t0, kind


def cpu_reference(procs, warm, steps, mach, aoa):
    """CPU throughput: `procs` independent solves of the 62,400-point sphere."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    job = (48, 1300, 0.02, mach, aoa, 1001, warm, steps)
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [job] * procs)
    n = res[0][0]
    wall = max(r[2] for r in res)
    return procs * n * steps / wall, wall / steps, n, res[0][3]


# ------------------------------------------------------------------ main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mfcfd", choices=["mfcfd", "reference"])
    ap.add_argument("--workload", default="sphere-1.1M", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep-mode", type=int, default=2, help="2 chains, 0 dataflow, 1 levels")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurement")
    args = ap.parse_args()
    rank, world, local_rank = dist_env()
    wl = WORKLOADS[args.workload]
    metric = "point-iters/s FP64"

    if args.impl == "reference":
        if rank != 0:
            return
        procs = max(1, min(os.cpu_count() or 1, 32))
        value, sec_per_step, n, kind = cpu_reference(procs, args.warmup, args.steps, wl["mach"], wl["aoa"])
        what = ("the reference's Fortran routines translated to C (oracle/_ref), glibc libm"
                if kind == "reference" else "the C++ restatement of the reference, glibc libm")
        sample = (f"{what}, -O2 -ffp-contract=off; {procs} independent solves of a {n}-point "
                  f"sphere (M={wl['mach']}, alpha={wl['aoa']}), one iteration per step")
        line = {"metric": metric, "value": value, "unit": "point-iters/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec_per_step * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": args.workload, "sample_points": n},
                "cpu_baseline": {"value": value, "unit": "point-iters/s", "cores": procs,
                                 "kind": kind, "sample": sample},
                "e2e": {"value": value, "unit": "point-iters/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    from mfcfd import cloud as cl
    from mfcfd import replicas
    from mfcfd.solver import Solver

    torch.cuda.set_device(local_rank)
    rank, world = replicas.init("nccl", timeout_s=600)
    barrier = replicas.barrier

    c = cl.shell_cloud(wl["shells"], wl["per_shell"], jitter=wl["jitter"],
                       seed=replicas.replica_seed(wl["seed"], rank))
    s = Solver(c, wl["mach"], wl["aoa"], device=local_rank, sweep_mode=args.sweep_mode)
    prim0 = cl.initial_state(c, wl["mach"], wl["aoa"])
    s.initial_conditions(prim0)
    info = s.info()
    stream = torch.cuda.ExternalStream(s.stream())

    # warm-up
    t = 1
    s.q_lskum(args.warmup, t0=t)
    t += args.warmup
    torch.cuda.synchronize()

    # timed region: device events on the library's stream
    sampler = ClockSampler(local_rank)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.q_lskum(args.steps, t0=t)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    t += args.steps
    ms = e0.elapsed_time(e1)
    # FP64 forces and pressure after warmup + steps iterations, the state the
    # mixed-precision run is compared with
    cl64, cd64, _ = s.forces()
    p64 = s.get_state()[0][:, 4].copy()
    ms_max = replicas.max_over_ranks(ms, device="cuda")
    value = replicas.throughput(c.n, args.steps, ms_max / 1e3, world)

    # phase timing (separate pass, same workload) for the roofline
    s.set_profiling(True)
    s.q_lskum(args.steps, t0=t)
    t += args.steps
    phases, piters = s.phase_times()
    s.set_profiling(False)
    dom = max(phases, key=lambda k: phases[k])
    dom_ms = phases[dom] / max(piters, 1)
    peak, peak_kind = load_peaks()
    achieved = PHASE_BYTES[dom] * c.n / (dom_ms / 1e3) / 1e9
    traffic = SWEEP_TRAFFIC_PER_POINT * c.n if dom.startswith("sweep") and args.sweep_mode == 2 else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": dom,
                "peak_source": peak_kind,
                "phase_ms_per_iter": {k: v / max(piters, 1) for k, v in phases.items()},
                "iteration_bytes_model": TOTAL_BYTES,
                # the sweeps are bound by their dependency chain, not by HBM:
                # levels of the schedule and device time per level
                "sweep_us_per_level": dom_ms * 1e3 / max(1, info["n_levels_forward"]
                                                        if dom == "sweep_fwd" else info["n_levels_backward"])}

    # end to end through the C ABI with pinned host buffers
    prim_h = torch.empty((c.n, 5), dtype=torch.float64, pin_memory=True).numpy()
    delu_h = torch.empty((c.n, 5), dtype=torch.float64, pin_memory=True).numpy()
    p_, d_, ro = s.get_state()
    prim_h[:] = p_
    delu_h[:] = d_
    torch.cuda.synchronize()
    barrier()
    w0 = time.perf_counter()
    for k in range(args.steps):
        s.set_state(prim_h, delu_h, ro)
        s.fpi_solver(t + k)
        p_, d_, ro = None, None, None
        prim_out, delu_out, ro = s.get_state()
        prim_h[:] = prim_out
        delu_h[:] = delu_out
    torch.cuda.synchronize()
    w1 = time.perf_counter()
    e2e_s = replicas.max_over_ranks(w1 - w0, device="cuda")
    e2e_value = replicas.throughput(c.n, args.steps, e2e_s, world)
    io_bytes = c.n * 5 * 8 * 2

    # mixed precision on the same cloud and schedule: device time of the same
    # K iterations, and its CL/CD/pressure error against the FP64 run after
    # the same number of iterations
    mixed = None
    if args.sweep_mode == 2 and not args.no_mixed:
        from mfcfd import _lib
        sm = Solver(c, wl["mach"], wl["aoa"], device=local_rank, sweep_mode=2,
                    precision=_lib.PRECISION_MIXED)
        sm.initial_conditions(prim0)
        sm.q_lskum(args.warmup, t0=1)
        streamm = torch.cuda.ExternalStream(sm.stream())
        barrier()
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(streamm)
        sm.q_lskum(args.steps, t0=1 + args.warmup)
        f1.record(streamm)
        torch.cuda.synchronize()
        barrier()
        msm = replicas.max_over_ranks(f0.elapsed_time(f1), device="cuda")
        clm, cdm, _ = sm.forces()
        pm = sm.get_state()[0][:, 4]
        mixed = {"value": replicas.throughput(c.n, args.steps, msm / 1e3, world),
                 "unit": "point-iters/s", "ms_per_step": msm / args.steps,
                 "speedup_vs_fp64": ms_max / msm,
                 "dtype": "f32 reconstruction/limiter/fluxes of residual and sweeps; f64 "
                          "least-squares sums and solves, D_inv, increments, update, norms, forces",
                 "iterations_compared": args.warmup + args.steps,
                 "dCL": clm - cl64, "dCD": cdm - cd64,
                 "pressure_max_rel_err": float(np.max(np.abs(pm - p64) / np.abs(p64)))}
        sm.close()

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sps, n, kind = cpu_reference(1, 0, 3, wl["mach"], wl["aoa"])
        what = ("the reference's Fortran routines translated to C (oracle/_ref), glibc libm"
                if kind == "reference" else "the C++ restatement of the reference, glibc libm")
        cpu_base = {"value": v, "unit": "point-iters/s", "cores": 1, "kind": kind,
                    "sample": f"{what}; one solve of a {n}-point sphere (M={wl['mach']}, "
                              f"alpha={wl['aoa']}), 3 iterations, 1 thread"}

    if rank == 0:
        line = {"metric": metric, "value": value, "unit": "point-iters/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded sphere-shell generator)",
                "config": {"workload": args.workload, "points": c.n, "mach": wl["mach"],
                           "alpha_deg": wl["aoa"], "precision": "fp64",
                           "levels_forward": info["n_levels_forward"],
                           "levels_backward": info["n_levels_backward"],
                           "l2": "state larger than L2 (no flush)",
                           "sweep_mode": args.sweep_mode,
                           "parallelism": f"replicas x{world}"},
                "e2e": {"value": e2e_value, "unit": "point-iters/s",
                        "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
                "roofline": roofline, "cpu_baseline": cpu_base, "clocks": clocks, "mixed": mixed,
                "gpu_launches": KERNELS_PER_ITER[args.sweep_mode] * args.steps}
        print(json.dumps(line), flush=True)
    s.close()
    replicas.finalize()


if __name__ == "__main__":
    main()
