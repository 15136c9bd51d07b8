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
             byte model of each phase) over its event-timed duration; its
             ``fp64`` part gives the same phase's FP64 operations (counted
             by the oracle built with counting arithmetic) over that time
             against the device's FMA rate measured by an in-tree loop
             kernel, and ``sweep_latency_floor_us`` one warp's time per
             swept point when it sweeps a small cloud alone.
Multi-GPU: independent replicas, one per rank (the LU-SGS sweep order is
global, so one cloud does not shard); value sums the ranks' points.

``--impl reference`` times the reference's own routines on the host cores
instead: its Fortran translated mechanically to C (oracle/_ref/libref.so,
glibc libm), or the C++ restatement of them when that build is absent; one
independent solve per host core on a 62,400-point sphere sample, one
iteration per step.
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
# DRAM bytes (read + write) per point of one chain-sweep launch, from the
# ncu capture of the 256,000-point sphere's forward sweep (630.45 MB read +
# 75.31 MB written per launch, profiles/ncu_k_sweep_chain_sphere256k.txt);
# each point stages its own records once, so a launch of n points moves
# about n times this.
SWEEP_TRAFFIC_PER_POINT = (630.45e6 + 75.31e6) / 256000

# FP64 operations per point-iteration of each phase, counted by the oracle
# built with counting arithmetic (oracle/oracle_flops.cpp: add, multiply,
# divide and sqrt one each, fma two, exp/log/erf through their own
# arithmetic in mfmath.h) over the third iteration of each workload:
#   oracle.flop_counts(cloud.sphere_1m(), 0.8, 2.0, iters=1, skip=2)
#   oracle.flop_counts(cloud.sphere_62k(), 0.4, 0.0, iters=1, skip=2)
# divided by the point count.  The reference evaluates D_inv again in the
# backward sweep; that repeat is left out (the GPU evaluates it once).
PHASE_FLOPS = {
    "sphere-1.1M": {"qderiv": 2814.0, "flux": 54246.0, "dinv": 3525.5, "sweep_fwd": 17626.3,
                    "sweep_bwd": 16805.6, "update": 162.0, "residual": 0.0},
    "sphere-62k": {"qderiv": 2814.0, "flux": 55989.0, "dinv": 3488.0, "sweep_fwd": 18102.5,
                   "sweep_bwd": 16082.6, "update": 165.1, "residual": 0.0},
}

WORKLOADS = {
    "sphere-1.1M": dict(shells=96, per_shell=11500, jitter=0.01, mach=0.8, aoa=2.0, seed=2001),
    "sphere-62k": dict(shells=48, per_shell=1300, jitter=0.02, mach=0.4, aoa=0.0, seed=1001),
    # a mid-size case for profiler captures: its state (~350 MB) exceeds L2
    "sphere-256k": dict(shells=64, per_shell=4000, jitter=0.015, mach=0.8, aoa=2.0, seed=2501),
}
# kernels of one iteration per sweep mode (2 chains: k_qderiv, k_pending,
# k_flux, two k_sweep_chain, k_update, two reductions, and k_g0 when the
# cloud has points outside the shared frame; 0/1 add k_dinv_gold)
KERNELS_PER_ITER = {2: 8, 0: 9, 1: 9}


def fp64_peak(device):
    """FP64 TFLOP/s of the device, measured now by the FMA-loop kernel of
    mfcfd/libmfcfd_peak.so (best of 5 launches, CUDA events)."""
    import ctypes
    L = ctypes.CDLL(os.path.join(PKG, "mfcfd", "libmfcfd_peak.so"))
    L.mfcfd_fp64_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    tf, ms = ctypes.c_double(0.0), ctypes.c_double(0.0)
    rc = L.mfcfd_fp64_fma_peak(int(device), 5, ctypes.byref(tf), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"fp64 peak kernel failed: CUDA error {rc}")
    return tf.value


def sweep_latency_floor(device, sweep_mode_kw):
    """Microseconds per swept point of the backward sweep when one warp
    sweeps a small cloud (8 shells x 150 points) alone: every hand-off stays
    in the warp, so this is one point's critical path."""
    from mfcfd import cloud as cl
    from mfcfd.solver import Solver
    c = cl.small_sphere()
    s = Solver(c, 0.8, 2.0, device=device, chain_warps=1, **sweep_mode_kw)
    s.initial_conditions()
    s.q_lskum(3)
    s.set_profiling(True)
    s.q_lskum(5, t0=4)
    ph, it = s.phase_times()
    n_swept = c.n - int((c.status == cl.STATUS_OUTER).sum()) - 1
    info = s.info()
    s.close()
    return {"us_per_point": ph["sweep_bwd"] * 1e3 / max(it, 1) / max(n_swept, 1),
            "points": c.n, "warps": info["chain_warps"], "levels_backward": info["n_levels_backward"]}


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

def setup_measure(c, wl, args, local_rank, host_s):
    """Set-up of the workload's cloud: the host set-up (the handle the bench
    times, already built), the device-resident set-up (gpu_setup = 1; the
    same arrays, checked by tests/test_gpu_device_setup.py) and the
    connectivity from raw points (mfcfd_knn) on the GPU and on the host's
    threads.  Wall-clock seconds of the library calls, inputs on the host."""
    from mfcfd import cloud as cl
    from mfcfd.solver import Solver
    dev = []
    for _ in range(2):   # the first maps new device memory; the second reuses the pool's
        t = time.perf_counter()
        s2 = Solver(c, wl["mach"], wl["aoa"], device=local_rank, sweep_mode=args.sweep_mode,
                    chain_spread=args.chain_spread, gpu_setup=1)
        dev.append(time.perf_counter() - t)
        s2.close()
    dev_s = dev[1]
    cl.knn(c.x[:4096], c.y[:4096], c.z[:4096], 26, device=local_rank)   # module load
    t = time.perf_counter()
    _, conn_d, _ = cl.knn(c.x, c.y, c.z, 26, device=local_rank)
    knn_dev = time.perf_counter() - t
    t = time.perf_counter()
    _, conn_h, _ = cl.knn(c.x, c.y, c.z, 26, device=-1)
    knn_host = time.perf_counter() - t
    return {"points": c.n, "host_s": host_s, "device_s": dev_s, "device_first_s": dev[0],
            "speedup": host_s / dev_s,
            "knn_device_s": knn_dev, "knn_host_s": knn_host, "knn_host_threads": os.cpu_count(),
            "knn_equal": bool((conn_d == conn_h).all()),
            "what": "mfcfd_create with the host set-up (gpu_setup 0) and the device-resident set-up "
                    "(gpu_setup 1; device_s: a handle made after one was destroyed, its memory kept "
                    "in the pool; device_first_s: the first, mapping new memory), and mfcfd_knn "
                    "k=26 on the GPU and the host"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mfcfd", choices=["mfcfd", "reference"])
    ap.add_argument("--workload", default="sphere-1.1M",
                    choices=sorted(WORKLOADS) + ["serve", "batch", "batch-converged", "wing-4.2M", "wing-250k"])
    ap.add_argument("--wing-max-iters", type=int, default=6000)
    ap.add_argument("--wing-precision", type=int, default=2,
                    help="2 mixed-dc (FP64 residual, FP32 sweeps; converges), 1 mixed (stalls near a 1e-5 drop)")
    ap.add_argument("--wing-target", type=float, default=-6.0, help="residue (log10 drop) to converge to")
    ap.add_argument("--wing-compare-iters", type=int, default=200,
                    help="iterations after which mixed CL/CD are compared with an FP64 run")
    ap.add_argument("--batch-clouds", type=int, default=24)
    ap.add_argument("--batch-bodies", choices=["mixed", "ellipsoids"], default="mixed")
    ap.add_argument("--batch-mach", type=float, nargs=2, default=[0.3, 0.85],
                    help="Mach range of the batch workload's flows")
    ap.add_argument("--batch-budget-gb", type=float, default=120.0,
                    help="device memory of one wave of batched handles")
    ap.add_argument("--no-batch-fp64", dest="batch_fp64", action="store_false",
                    help="batch-converged: skip the FP64 one-at-a-time solves (no speed-up or CL/CD "
                         "error in the line; for comparing the batched forms alone)")
    ap.add_argument("--batch-graphs", type=int, choices=[0, 1], default=1,
                    help="batch workload: capture chunks as CUDA graphs (1) or launch kernel by kernel (0, "
                         "the form for profiling: launches run in the order issued)")
    ap.add_argument("--no-batch-grouped", dest="batch_grouped", action="store_false",
                    help="batch and batch-converged workloads: skip the lockstep group form "
                         "(mfcfd_run_group)")
    ap.add_argument("--batch-min-points", type=int, default=None,
                    help="smallest cloud (default 20000 for batch, 10000 for batch-converged)")
    ap.add_argument("--batch-max-points", type=int, default=None,
                    help="largest cloud (default 100000 for batch, 40000 for batch-converged)")
    ap.add_argument("--batch-max-iters", type=int, default=12000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep-mode", type=int, default=2, help="2 chains, 0 dataflow, 1 levels")
    ap.add_argument("--chain-spread", type=int, default=0, help="1: one 4-warp chain block per SM")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurement")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving measurement")
    ap.add_argument("--serve-requests", type=int, default=40)
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrivals per second")
    ap.add_argument("--serve-min-points", type=int, default=10000)
    ap.add_argument("--serve-max-points", type=int, default=160000)
    ap.add_argument("--serve-target", type=float, default=-1.0, help="residue (log10 drop) to converge to")
    ap.add_argument("--serve-max-iters", type=int, default=600)
    ap.add_argument("--serve-chunk", type=int, default=10)
    ap.add_argument("--serve-setup-threads", type=int, default=8)
    ap.add_argument("--serve-device-setup", action="store_true",
                    help="the server sets each request up on the device at admission")
    ap.add_argument("--no-setup-timing", action="store_true",
                    help="skip the set-up and kNN timings of the default line")
    ap.add_argument("--serve-precision", type=int, default=1, help="1 mixed, 2 mixed-dc (FP64 residual)")
    ap.add_argument("--serve-conv-requests", type=int, default=8)
    ap.add_argument("--serve-conv-min-points", type=int, default=5000)
    ap.add_argument("--serve-conv-max-points", type=int, default=10000)
    args = ap.parse_args()
    rank, world, local_rank = dist_env()
    if args.workload == "serve":
        return serve_main(args, rank, world, local_rank)
    if args.workload == "batch":
        return batch_main(args, rank, world, local_rank)
    if args.workload == "batch-converged":
        return batch_converged_main(args, rank, world, local_rank)
    if args.workload.startswith("wing"):
        return wing_main(args, rank, world, local_rank)
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
    t_setup = time.perf_counter()
    s = Solver(c, wl["mach"], wl["aoa"], device=local_rank, sweep_mode=args.sweep_mode,
               chain_spread=args.chain_spread)
    setup_host_s = time.perf_counter() - t_setup
    setup = None
    if world == 1 and not args.no_setup_timing:
        setup = setup_measure(c, wl, args, local_rank, setup_host_s)
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
                                                        if dom == "sweep_fwd" else info["n_levels_backward"]),
                "sweep_us_per_level_both": {
                    "forward": phases["sweep_fwd"] / max(piters, 1) * 1e3 / max(1, info["n_levels_forward"]),
                    "backward": phases["sweep_bwd"] / max(piters, 1) * 1e3 / max(1, info["n_levels_backward"])}}
    flops = PHASE_FLOPS.get(args.workload)
    if flops:
        pk64 = fp64_peak(local_rank)
        it_flops = sum(flops.values())
        dom_tf = flops[dom] * c.n / (dom_ms / 1e3) / 1e12
        it_tf = it_flops * c.n / (ms_max / args.steps / 1e3) / 1e12
        roofline["fp64"] = {"phase": dom, "flops_per_point": flops[dom], "achieved": dom_tf, "peak": pk64,
                            "unit": "TFLOP/s", "frac": dom_tf / pk64,
                            "iteration_flops_per_point": it_flops, "iteration_achieved": it_tf,
                            "iteration_frac": it_tf / pk64,
                            "phase_flops_per_point": flops,
                            "peak_source": "builder-measured: FMA loop kernel (libmfcfd_peak.so), best of 5, "
                                           "CUDA events, on this GPU in this run",
                            "counted_by": "oracle built with counting arithmetic (oracle/oracle_flops.cpp)"}
    if args.sweep_mode == 2:
        floor = sweep_latency_floor(local_rank, {})
        roofline["sweep_latency_floor_us"] = floor["us_per_point"]
        roofline["sweep_latency_floor"] = floor

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
        _, _, ro = s.get_state(out=(prim_h, delu_h))   # straight into the pinned buffers
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

    # served solves (a reduced stream: 24 requests of 10k-80k points) beside
    # the point-iteration rate, on one GPU
    serving = serving_conv = None
    if world == 1 and not args.no_serving:
        s.close()
        serving = serve_measure(args, rank, world, local_rank, 24, 80000)
        # converged solves: requests run to a 1e-6 drop of the density residual
        serving_conv = serve_measure(args, rank, world, local_rank, args.serve_conv_requests,
                                     args.serve_conv_max_points, min_points=args.serve_conv_min_points,
                                     target=-6.0, max_iters=8000, precision=2, seed=5500, polish=-5.0,
                                     mach=(0.3, 0.6), aspect=(1.0, 1.0))
        s = None

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
                "serving": serving, "serving_converged": serving_conv, "setup": setup,
                # + k_g0 when the cloud has points outside the shared frame
                "gpu_launches": (KERNELS_PER_ITER[args.sweep_mode] + (1 if info.get("g0_points") else 0))
                                * args.steps}
        print(json.dumps(line), flush=True)
    if s is not None:
        s.close()
    replicas.finalize()


def wing_main(args, rank, world, local_rank):
    """The seeded swept-wing cloud (NACA 0012, semispan 1, taper 0.56, 30 deg
    sweep, 400 x 120 wall points, ~4.2M points) at M 0.84, alpha 3.06 deg in
    mixed precision, run until the residue reaches --wing-target (a 1e-6 drop
    of the density residual) or --wing-max-iters.  Device-timed point-iters/s
    over the whole run; the mixed CL/CD after --wing-compare-iters iterations
    against an FP64 run of the same iterations, which also gives the FP64
    rate."""
    import torch
    from mfcfd import _lib, replicas, wing
    from mfcfd.solver import Solver
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable":
                              "the wing workload runs the GPU forms only; the reference's CPU solver is "
                              "timed by the point-iteration workloads"}), flush=True)
        return
    torch.cuda.set_device(local_rank)
    rank, world = replicas.init("nccl", timeout_s=3600)
    big = args.workload == "wing-4.2M"
    t0 = time.perf_counter()
    c = (wing.swept_wing(seed=replicas.replica_seed(3001, rank)) if big else
         wing.swept_wing(points=250_000, nc=160, ns=48, seed=replicas.replica_seed(3001, rank), name="wing-250k"))
    gen_s = time.perf_counter() - t0
    mach, aoa = 0.84, 3.06

    def run(precision, max_iters, target, snap):
        t1 = time.perf_counter()
        s = Solver(c, mach, aoa, device=local_rank, precision=precision)
        setup_s = time.perf_counter() - t1
        s.initial_conditions()
        st = torch.cuda.ExternalStream(s.stream())
        ms, t, hist, at_snap, polished, diverged = 0.0, 1, [], None, None, None
        chunk = 50
        while t <= max_iters:
            k = min(chunk, max_iters - t + 1)
            if snap and t <= snap < t + k:
                k = snap - t + 1
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            try:
                h = s.q_lskum(k, t0=t)
            except _lib.MfcfdError as err:     # the iteration diverged (non-finite residual)
                torch.cuda.synchronize()
                diverged = (t, str(err))
                break
            e1.record(st)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            hist.extend(h.tolist())
            t += k
            if snap and t - 1 == snap:
                at_snap = s.forces()[:2]
            if h[-1][1] <= target or not np.isfinite(h[-1][0]):
                break
            if precision == _lib.PRECISION_MIXED_DC and polished is None and t > 3 and h[-1][1] <= -5.0:
                s.set_precision(_lib.PRECISION_FP64)     # the last part of the solve in FP64
                polished = t - 1
        cl_, cd_ = s.forces()[:2] if diverged is None else (None, None)
        info = s.info()
        s.close()
        return dict(iters=t - 1, ms=ms, setup_s=setup_s, res=hist or [[float("nan"), float("nan")]], cl=cl_,
                    cd=cd_, at_snap=at_snap, info=info, polished_at=polished, diverged=diverged)

    mixed = run(args.wing_precision, args.wing_max_iters, args.wing_target, args.wing_compare_iters)
    fp64 = run(_lib.PRECISION_FP64, args.wing_compare_iters, -1e9, None)
    if mixed["diverged"] or fp64["diverged"]:
        if rank == 0:
            print(json.dumps({"metric": "point-iters/s mixed to a 1e-6 residual drop", "value": None,
                              "unit": "point-iters/s", "workload": args.workload, "points": c.n,
                              "diverged": {"mixed": mixed["diverged"], "fp64": fp64["diverged"]},
                              "note": "the iteration diverged on this cloud; the CPU oracle (the reference's "
                                      "algorithm) diverges on it as well"}), flush=True)
        replicas.finalize()
        return
    ms_m = replicas.max_over_ranks(mixed["ms"], device="cuda")
    ms_f = replicas.max_over_ranks(fp64["ms"], device="cuda")
    value = c.n * mixed["iters"] * world / (ms_m / 1e3)
    fvalue = c.n * fp64["iters"] * world / (ms_f / 1e3)
    if rank == 0:
        res = np.array(mixed["res"])
        conv = bool(res[-1, 1] <= args.wing_target)
        drops = {}
        for lv in range(1, 7):
            hit = np.nonzero(res[:, 1] <= -lv)[0]
            drops[str(-lv)] = int(hit[0]) + 1 if len(hit) else None
        cm, cf = mixed["at_snap"], (fp64["cl"], fp64["cd"])
        line = {"metric": "point-iters/s mixed to a 1e-6 residual drop", "value": value, "unit": "point-iters/s",
                "precision": {1: "mixed", 2: "mixed-dc (FP64 residual, FP32 sweeps)"}.get(args.wing_precision),
                "n_gpus": world, "steps": mixed["iters"], "warmup": 0,
                "ms_per_step": ms_m / max(1, mixed["iters"]), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "mixed f32/f64", "data": "synthetic (seeded swept-wing cloud)",
                "config": {"workload": args.workload, "points": c.n, "counts": c.counts(), "mach": mach,
                           "alpha_deg": aoa, "target_residue": args.wing_target,
                           "max_iters": args.wing_max_iters, "generate_s": gen_s,
                           "setup_s": mixed["setup_s"], "levels_forward": mixed["info"]["n_levels_forward"],
                           "levels_backward": mixed["info"]["n_levels_backward"],
                           "parallelism": f"replicas x{world}"},
                "converged": conv, "iterations": mixed["iters"], "first_iteration_at_drop": drops,
                "switched_to_fp64_at_iteration": mixed["polished_at"],
                "final_res_new": res[-1, 0], "final_residue": res[-1, 1], "cl": mixed["cl"], "cd": mixed["cd"],
                "solve_s": ms_m / 1e3,
                "fp64": {"value": fvalue, "unit": "point-iters/s", "iterations": fp64["iters"],
                         "ms_per_step": ms_f / max(1, fp64["iters"])},
                "mixed_vs_fp64_at_iteration": {"iteration": args.wing_compare_iters,
                                               "dCL": None if cm is None else cm[0] - cf[0],
                                               "dCD": None if cm is None else cm[1] - cf[1],
                                               "cl_fp64": cf[0], "cd_fp64": cf[1]},
                "residue_history_every_50": [round(float(x), 4) for x in res[49::50, 1]]}
        print(json.dumps(line), flush=True)
    replicas.finalize()


def batch_converged_main(args, rank, world, local_rank):
    """Converged solves of a batch: --batch-clouds seeded sphere and
    ellipsoid clouds of --batch-min-points to --batch-max-points points
    (log-uniform, Mach U[0.3, 0.85], alpha U[-5, 5] deg), each run to a 1e-6
    drop of the density residual (residue -6).  Batched: MIXED_DC (FP64
    residual, FP32 sweeps) with a switch to FP64 at residue -5, all clouds
    iterating together in rounds; against the plain FP64 path, one cloud at
    a time.  Solves/s = clouds / wall time of each; CL/CD of every cloud
    against its FP64 solve."""
    import torch
    from mfcfd import _lib, batch, replicas, serve
    from mfcfd.solver import Solver
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no batch runner; its CPU solver is timed by the "
                              "point-iteration workloads"}), flush=True)
        return
    torch.cuda.set_device(local_rank)
    rank, world = replicas.init("nccl", timeout_s=3600)
    # spheres at M 0.3-0.6: the seeded ellipsoid clouds and the higher Mach
    # numbers include solves that stall above a 1e-6 drop or diverge in FP64
    _, clouds, reqs = serve.request_stream(args.batch_clouds, 1.0, replicas.replica_seed(7100, rank),
                                           args.batch_min_points or 10000, args.batch_max_points or 40000,
                                           pool=args.batch_clouds, mach=(0.3, 0.6), aspect=(1.0, 1.0))
    flows = [(reqs[i][1], reqs[i][2]) for i in range(len(clouds))]
    # warm-up: one short batched round (graph capture, first launches)
    ws = [Solver(clouds[0], *flows[0], device=local_rank, precision=_lib.PRECISION_MIXED_DC)]
    ws[0].initial_conditions()
    batch.run_batch(ws, 20)
    ws[0].close()
    # plain FP64, one cloud after another
    t0 = time.perf_counter()
    fp64 = []
    for c, (m, a) in zip(clouds, flows):
        if not args.batch_fp64:
            fp64.append({"forces": (float("nan"), float("nan")), "iters": None, "converged": None})
            continue
        s = Solver(c, m, a, device=local_rank)
        s.initial_conditions()
        r = batch.solve_batch([s], max_iters=args.batch_max_iters, polish=None)[0]
        r["forces"] = s.forces()[:2]
        fp64.append(r)
        s.close()
    torch.cuda.synchronize()
    seq_s = replicas.max_over_ranks(time.perf_counter() - t0, device="cuda") if args.batch_fp64 else float("nan")
    # batched MIXED_DC with the FP64 polish
    ss = []
    for c, (m, a) in zip(clouds, flows):
        s = Solver(c, m, a, device=local_rank, precision=_lib.PRECISION_MIXED_DC)
        s.initial_conditions()
        ss.append(s)
    replicas.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = batch.solve_batch(ss, max_iters=args.batch_max_iters, polish=-5.0)
    torch.cuda.synchronize()
    bat_s = replicas.max_over_ranks(time.perf_counter() - t0, device="cuda")
    errs = []
    for s, r, f in zip(ss, out, fp64):
        cl_, cd_, _ = s.forces()
        errs.append((abs(cl_ - f["forces"][0]), abs(cd_ - f["forces"][1])))
        s.close()
    grouped = None
    if args.batch_grouped:
        # the same solves as lockstep groups (mfcfd_run_group), fresh handles
        ss = []
        for c, (m, a) in zip(clouds, flows):
            s = Solver(c, m, a, device=local_rank, precision=_lib.PRECISION_MIXED_DC)
            s.initial_conditions()
            ss.append(s)
        replicas.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gout = batch.solve_batch(ss, max_iters=args.batch_max_iters, polish=-5.0, grouped=True)
        torch.cuda.synchronize()
        grp_s = replicas.max_over_ranks(time.perf_counter() - t0, device="cuda")
        gerr = []
        for s, f in zip(ss, fp64):
            cl_, cd_, _ = s.forces()
            gerr.append((abs(cl_ - f["forces"][0]), abs(cd_ - f["forces"][1])))
            s.close()
        grouped = {"value": len(clouds) * world / grp_s, "unit": "solves/s", "seconds": grp_s,
                   "converged": sum(1 for r in gout if r["converged"]),
                   "iterations": [r["iters"] for r in gout],
                   "speedup_vs_fp64_one_at_a_time": seq_s / grp_s,
                   "max_abs_dCL": max(e[0] for e in gerr), "max_abs_dCD": max(e[1] for e in gerr),
                   "form": "mfcfd_run_group: each 100-iteration round as lockstep groups"}
    if rank == 0:
        n = len(clouds) * world
        line = {"metric": "converged solves/s (1e-6 residual drop) batched mixed-dc vs FP64 one at a time",
                "value": n / bat_s, "unit": "solves/s", "n_gpus": world, "steps": len(clouds), "warmup": 1,
                "ms_per_step": bat_s * 1e3 / len(clouds), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "mixed-dc f32 sweeps / f64 residual, f64 polish from residue -5",
                "data": "synthetic (seeded sphere/ellipsoid shell clouds)",
                "config": {"workload": "batch-converged", "clouds": len(clouds), "bodies": "spheres",
                           "mach_range": [0.3, 0.6], "alpha_range_deg": [-5.0, 5.0],
                           "points": [c.n for c in clouds], "target_residue": -6.0,
                           "max_iters": args.batch_max_iters, "polish_residue": -5.0, "round": 100,
                           "parallelism": f"replicas x{world}"},
                "converged": sum(1 for r in out if r["converged"]),
                "iterations": [r["iters"] for r in out],
                "fp64_one_at_a_time": {"value": n / seq_s, "unit": "solves/s", "seconds": seq_s,
                                       "converged": sum(1 for r in fp64 if r["converged"]),
                                       "iterations": [r["iters"] for r in fp64]},
                "speedup_vs_fp64_one_at_a_time": seq_s / bat_s,
                "max_abs_dCL": max(e[0] for e in errs), "max_abs_dCD": max(e[1] for e in errs)}
        if grouped:
            line["grouped"] = grouped
        print(json.dumps(line), flush=True)
    replicas.finalize()


def batch_main(args, rank, world, local_rank):
    """Batched clouds: a seeded set of sphere and ellipsoid clouds of uneven
    size (log-uniform --batch-min-points to --batch-max-points) iterated
    together in mixed precision, each chunk a captured graph and the chain
    schedules autotuned for the batch, against the same clouds run one after
    another on the plain FP64 path.  Both are device-timed over the same
    iterations; point-iters/s aggregate.  A batch larger than
    --batch-budget-gb of device memory runs in waves of handles that fit;
    every wave is tuned, warmed and timed the same way and the timed seconds
    add up.  Set-up and connectivity run on the device (gpu_setup 1,
    mfcfd_knn), outside the timed regions."""
    import torch
    from mfcfd import _lib, batch, replicas, serve
    from mfcfd.solver import Solver
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no batch runner; its CPU solver is timed by the "
                              "point-iteration workloads"}), flush=True)
        return
    torch.cuda.set_device(local_rank)
    rank, world = replicas.init("nccl", timeout_s=3600)
    t_gen = time.perf_counter()
    _, clouds, reqs = serve.request_stream(args.batch_clouds, 1.0, replicas.replica_seed(7000, rank),
                                           args.batch_min_points or 20000, args.batch_max_points or 100000,
                                           pool=args.batch_clouds, bodies=args.batch_bodies, knn_device=local_rank,
                                           mach=tuple(args.batch_mach))
    t_gen = time.perf_counter() - t_gen
    flows = [(reqs[i][1], reqs[i][2]) for i in range(len(clouds))]
    pts = sum(c.n for c in clouds)
    # plain FP64 path, one cloud after another (device time of `steps` iterations each)
    seq_ms = 0.0
    seq_restarted = 0
    for c, (m, a) in zip(clouds, flows):
        s = Solver(c, m, a, device=local_rank, gpu_setup=1)
        st = torch.cuda.ExternalStream(s.stream())
        for attempt in range(2):   # a diverging cloud starts again from the freestream
            try:
                s.initial_conditions()
                s.q_lskum(args.warmup)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                s.q_lskum(args.steps, t0=1 + args.warmup)
                e1.record(st)
                torch.cuda.synchronize()
                seq_ms += e0.elapsed_time(e1)
                break
            except _lib.MfcfdError:
                seq_restarted += 1
                if attempt == 1:
                    raise
        s.close()
    # batched: mixed precision, tuned schedules, graph-captured chunks, in
    # waves of handles within the memory budget
    budget = args.batch_budget_gb * 1e9
    bat_s, grp_s, t_setup, t_tune, waves = 0.0, 0.0, 0.0, 0.0, []
    percents, warps = [], []
    j = 0
    while j < len(clouds):
        ss, used = [], 0
        t1 = time.perf_counter()
        while j < len(clouds):
            c, (m, a) = clouds[j], flows[j]
            s = Solver(c, m, a, device=local_rank, precision=_lib.PRECISION_MIXED, gpu_setup=1,
                       graphs=args.batch_graphs)
            s.initial_conditions()
            ss.append(s)
            used += s.info()["device_bytes"]
            j += 1
            if used > budget:
                break
        t_setup += time.perf_counter() - t1
        t1 = time.perf_counter()
        percent, _ = batch.tune_batch(ss, iters=4)
        t_tune += time.perf_counter() - t1
        percents.append(percent)
        warps += [s.info()["chain_warps"] for s in ss]
        def restart_failed(st, ss=ss):
            # a cloud whose residual went non-finite starts again from the
            # freestream (the reference scheme diverges on some seeded
            # ellipsoids); the batch keeps its shape
            bad = [i for i, v in enumerate(st) if v != 0]
            for i in bad:
                ss[i].initial_conditions()
            return len(bad)

        # warm-up: the timed chunk length, for both U/q parities (graphs captured)
        st = [0] * len(ss)
        restarted = 0
        batch.run_batch(ss, args.warmup, statuses=st)
        restarted += restart_failed(st)
        for _ in range(1 if args.steps % 2 == 0 else 2):
            batch.run_batch(ss, args.steps, statuses=st)
            restarted += restart_failed(st)
        for attempt in range(3):
            replicas.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            batch.run_batch(ss, args.steps, statuses=st)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            k = restart_failed(st)
            restarted += k
            if k == 0:
                break
        bat_s += dt
        waves.append({"clouds": len(ss), "points": sum(s.n for s in ss), "device_bytes": used, "timed_s": dt,
                      "restarted_clouds": restarted})
        if args.batch_grouped:
            # the same handles in lockstep groups, each sweep direction of a
            # group in one launch (mfcfd_run_group); warmed the same way
            groups = batch.plan_groups(ss)
            for _ in range(1 if args.steps % 2 == 0 else 2):
                batch.run_grouped(ss, args.steps, groups, statuses=st)
                restart_failed(st)
            for attempt in range(3):
                replicas.barrier()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                batch.run_grouped(ss, args.steps, groups, statuses=st)
                torch.cuda.synchronize()
                gdt = time.perf_counter() - t0
                if restart_failed(st) == 0:
                    break
            grp_s += gdt
            waves[-1].update({"grouped_timed_s": gdt, "groups": [len(g) for g in groups]})
        print(f"wave {len(waves)}: {len(ss)} clouds, {waves[-1]['points']} points, {used / 1e9:.1f} GB, "
              f"{dt:.3f} s, restarted {restarted}", file=sys.stderr, flush=True)
        for s in ss:
            s.close()
    bat_s = replicas.max_over_ranks(bat_s, device="cuda")
    seq_s = replicas.max_over_ranks(seq_ms / 1e3, device="cuda")
    value = pts * args.steps * world / bat_s
    if rank == 0:
        line = {"metric": "point-iters/s batched mixed vs FP64 one at a time", "value": value,
                "unit": "point-iters/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": bat_s * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "mixed f32/f64",
                "data": "synthetic (seeded sphere/ellipsoid shell clouds)",
                "config": {"workload": "batch", "clouds": len(clouds), "points_total": pts,
                           "points_min": min(c.n for c in clouds), "points_max": max(c.n for c in clouds),
                           "bodies": args.batch_bodies, "mach_range": list(args.batch_mach),
                           "alpha_range_deg": [-5.0, 5.0],
                           "tuned_percent_of_widest_level": percents, "tuned_warps": warps,
                           "waves": waves, "budget_gb": args.batch_budget_gb,
                           "generate_s": t_gen, "setup_s": t_setup, "tune_s": t_tune,
                           "parallelism": f"replicas x{world}",
                           "timing": "batched: wall clock with device synchronisation around the K "
                                     "iterations of each wave, summed; FP64: device events, clouds one "
                                     "after another"},
                "fp64_one_at_a_time": {"value": pts * args.steps * world / seq_s, "unit": "point-iters/s",
                                       "ms_per_step": seq_s * 1e3 / args.steps, "restarted": seq_restarted},
                "speedup_vs_fp64_one_at_a_time": seq_s / bat_s}
        if args.batch_grouped:
            line["grouped"] = {"value": pts * args.steps * world / grp_s, "unit": "point-iters/s",
                               "ms_per_step": grp_s * 1e3 / args.steps,
                               "speedup_vs_fp64_one_at_a_time": seq_s / grp_s,
                               "form": "mfcfd_run_group: lockstep groups of up to 32 clouds of similar size, "
                                       "one chain-sweep launch per direction per group iteration, groups "
                                       "one after another"}
        print(json.dumps(line), flush=True)
    replicas.finalize()


def serve_main(args, rank, world, local_rank):
    """Served steady-state solves: a Poisson stream of requests (clouds of
    log-uniform size, random Mach and angle of attack) through the request
    server in mixed precision, against the same stream served one request at
    a time in FP64; latency is submit to retirement.  A sample of the mixed
    results (at least 5%) is re-solved alone in FP64 for the CL/CD error."""
    import torch
    from mfcfd import _lib, replicas, serve
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no request server; its CPU solver is timed by the "
                              "point-iteration workloads"}), flush=True)
        return
    torch.cuda.set_device(local_rank)
    rank, world = replicas.init("nccl", timeout_s=1800)
    line = serve_measure(args, rank, world, local_rank, args.serve_requests, args.serve_max_points,
                         precision=args.serve_precision)
    if rank == 0:
        line.update({"metric": "served solves/s", "n_gpus": world, "steps": line["requests"], "warmup": 0,
                     "ms_per_step": 1e3 / line["value"] * world, "higher_is_better": True,
                     "scaling": "weak", "vs_baseline": None, "dtype": "mixed f32/f64",
                     "data": "synthetic (seeded sphere/ellipsoid shell clouds)",
                     "e2e": {"value": line["value"], "unit": "solves/s",
                             "h2d_bytes_per_step": line.pop("h2d_bytes_per_request"),
                             "d2h_bytes_per_step": line.pop("d2h_bytes_per_request")}})
        print(json.dumps(line), flush=True)
    replicas.finalize()


def serve_measure(args, rank, world, local_rank, count, max_points, min_points=None, target=None,
                  max_iters=None, precision=None, seed=5000, polish=0.0, mach=(0.3, 0.85), aspect=(1.0, 3.0)):
    """The serving measurement (see serve_main) for `count` requests of
    clouds of `min_points` to `max_points` points, each run until its residue
    is <= `target` (or `max_iters`), served in `precision` with continuous
    batching against the same stream one request at a time in FP64; returns
    its summary (rank 0).  Every request's CL/CD is compared with its FP64
    solve."""
    from mfcfd import _lib, replicas, serve
    min_points = args.serve_min_points if min_points is None else min_points
    target = args.serve_target if target is None else target
    max_iters = args.serve_max_iters if max_iters is None else max_iters
    precision = _lib.PRECISION_MIXED if precision is None else precision
    arrivals, clouds, reqs = serve.request_stream(count, args.serve_rate,
                                                  replicas.replica_seed(seed, rank),
                                                  min_points, max_points, mach=mach, aspect=aspect,
                                                  knn_device=local_rank)

    def run(prec, max_live):
        # many requests at once: chain schedules of the widest level's width;
        # one at a time: each request's own (twice that)
        with serve.Server(device=local_rank, chunk=args.serve_chunk, setup_threads=args.serve_setup_threads,
                          max_live=max_live, chain_percent=100 if max_live == 0 else 0,
                          device_setup=args.serve_device_setup) as srv:
            # warm-up request (untimed): first graph capture and launches in the process
            small = min(range(len(clouds)), key=lambda i: clouds[i].n)
            srv.wait(srv.submit(clouds[small], 0.5, 0.0, max_iters=args.serve_chunk, residue_target=-99.0,
                                precision=prec))
            replicas.barrier()
            st0 = srv.stats()
            t0 = time.perf_counter()
            ids = []
            for ta, (ci, m, a) in zip(arrivals, reqs):
                wait = ta - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
                ids.append(srv.submit(clouds[ci], m, a, max_iters=max_iters, residue_target=target,
                                      precision=prec, polish_residue=polish if prec == 2 else 0.0))
            res = [srv.wait(i) for i in ids]
            wall = time.perf_counter() - t0
            st = srv.stats()
            for k in ("busy_s", "slot_s"):   # the stream's share, not the warm-up's
                st[k] -= st0[k]
        return res, replicas.max_over_ranks(wall, device="cuda"), st

    res_m, wall_m, st_m = run(precision, 0)
    res_b, wall_b, _ = run(_lib.PRECISION_FP64, 1)
    total = len(reqs) * world
    lat = serve.latency_summary([r["latency"] for r in res_m])
    lat_b = serve.latency_summary([r["latency"] for r in res_b])
    # CL/CD of every request against its FP64 solve (the one-at-a-time run)
    errs = [(abs(a["cl"] - b["cl"]), abs(a["cd"] - b["cd"])) for a, b in zip(res_m, res_b)]
    k = len(errs)
    conv = sum(1 for r in res_m if r["converged"])
    conv_b = sum(1 for r in res_b if r["converged"])

    def phases(res):
        # host preparation, wait for HBM / SM slots, time on the GPU
        return {"prepare": float(np.mean([r["t_ready"] - r["t_submit"] for r in res])),
                "admit_wait": float(np.mean([r["t_admit"] - r["t_ready"] for r in res])),
                "solve": float(np.mean([r["t_done"] - r["t_admit"] for r in res])),
                "of_which_running": float(np.mean([r["run_s"] for r in res]))}
    pts = [clouds[ci].n for ci, _, _ in reqs]
    return {"value": total / wall_m, "unit": "solves/s", "requests": len(reqs),
            "config": {"workload": "serve", "requests": len(reqs), "rate_per_s": args.serve_rate,
                       "points_min": min(pts), "points_max": max(pts), "points_total": sum(pts),
                       "residue_target": target, "max_iters": max_iters, "polish_residue": polish,
                       "chunk": args.serve_chunk, "mach_range": list(mach), "aspect_range": list(aspect),
                       "setup": "device, at admission" if args.serve_device_setup else "host, at arrival",
                       "precision": {1: "mixed", 2: "mixed-dc (FP64 residual, FP32 sweeps)"}.get(precision, "fp64"),
                       "parallelism": f"replicas x{world}"},
            "latency_s": lat, "latency_phases_mean_s": phases(res_m), "converged": conv, "failed": sum(1 for r in res_m if r["status"]),
            "iterations_mean": float(np.mean([r["iters"] for r in res_m])),
            "iterations_mean_fp64": float(np.mean([r["iters"] for r in res_b])), "converged_fp64": conv_b,
            "peak_live": st_m["peak_live"], "peak_bytes_live": st_m["peak_bytes_live"],
            # seconds with a chunk on the GPU, and the chain-sweep slots held,
            # over the stream's wall time (slot_capacity slots in all)
            "gpu_busy_frac": st_m["busy_s"] / wall_m,
            "slot_occupancy": st_m["slot_s"] / (st_m["slot_capacity"] * wall_m) if st_m["slot_capacity"] else None,
            "fp64_one_at_a_time": {"value": total / wall_b, "unit": "solves/s", "latency_s": lat_b,
                                   "latency_phases_mean_s": phases(res_b)},
            "speedup_vs_fp64_one_at_a_time": wall_b / wall_m,
            "fp64_resolve_sample": {"requests": k, "max_abs_dCL": max(e[0] for e in errs),
                                    "max_abs_dCD": max(e[1] for e in errs),
                                    "of": "every request against its FP64 solve"},
            # per point: status, xyz, frames, nbhs, conn(27), min_dist, prim in; prim out
            "h2d_bytes_per_request": int(np.mean(pts) * (4 + 24 + 72 + 4 + 108 + 8 + 40)),
            "d2h_bytes_per_request": int(np.mean(pts) * 5 * 8)}


if __name__ == "__main__":
    main()
