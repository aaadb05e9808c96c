#!/usr/bin/env python
"""Benchmark of the Crank-Nicolson step: mode*node*steps/s on one binary.

Workload (the single-GPU configuration the headline metric is quoted on): the
plain FP64 drop-in on one binary with an evolving orbit -- 2p hydrogenic cloud
(n=2, l=1, m=1) on the primary, mu=0.25, q=0.5, R=50, back-reaction + GW decay +
accretion on, s-wave absorption on; l_max=8 (45 modes); N=20000, L=2000,
r_ex=1500; dt=0.5 (steps_per_period = P0/0.5); complex128 throughout.  Keys the
configuration does not name take the reference's minimal-example values:
ramp_periods=2, epsilon=0, epsilon_smear=2, M_c=0.01, damping mask 0.85/1/6.
The timed steps start one initial period after the start-up ramp, where the
absorbers, the back-reaction and the orbit evolution are all at full strength.
The initial state is synthetic (analytic 2p state projected on the modes).

Arms:
  (default)          the CUDA path through the Python binding of the C ABI;
  --impl reference   the reference's CPU algorithm on the host cores: the oracle
                     restatement (oracle/, C++17 + OpenMP), the reference itself
                     being unbuildable here (Eigen 3 and GSL absent).
Under torchrun each rank advances its own replica (no collective on the data
path; "replicas only"), timings are maxed over ranks.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(workload="fp64_single_binary_evolving_orbit", Nr=20000, L=2000.0, l_max=8, n_modes=45, mu=0.25,
                q=0.5, R=50.0, dt=0.5, r_ex=1500.0, counter=False, absorption=True, evolve_orbit=True,
                M_c=0.01, epsilon=0.0, epsilon_smear=2.0, ramp_periods=2.0, mask=[0.85, 1.0, 6],
                state="2p hydrogenic (2,1,1) on the primary", precision="fp64")
METRIC = "CN mode*node*steps/s"
UNIT = "mode*node*steps/s"

# DRAM traffic (read + write) per launch of the dominant kernel, the operator apply,
# from the ncu capture summarised in profiles/k_apply5_fp64_binary_n45_N20000.md:
# dram__bytes.sum.per_second x gpu__time_duration.sum = 242.04 GB/s x 73.952 us (below the
# algorithmic bytes: the input vector, written by the launch before, is read from L2).
NCU_TRAFFIC_BYTES = 242.035482e9 * 73.952e-6


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p.get("hbm_gbs", 6650.0), p.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_solver(cls, w, psi0=None):
    cn = cls(w["Nr"], w["L"], w["dt"], w["epsilon"], w["l_max"], w["mu"], w["M_c"], w["q"], 0.0, w["R"],
             w["counter"], w["absorption"], 10 ** 9, w["ramp_periods"], w["epsilon_smear"])
    if psi0 is None:
        from boson_cloud_binary_b200.initial_state import hydrogenic_on_primary
        psi0 = hydrogenic_on_primary(cn.r, cn.modes, w["mu"], w["q"], w["R"])
    cn.set_initial_state_full(psi0)
    cn.evolve_orbit = w["evolve_orbit"]
    cn.steps_per_period = cn.P / w["dt"]
    cn.initialize()
    cn.build_damping_mask(*w["mask"])
    cn.run(10 ** 9, w["r_ex"])
    # one initial period past the start-up ramp: absorbers and back-reaction at full strength
    t_start = (w["ramp_periods"] + 1.0) * cn.P
    cn.t_i = t_start
    cn.refresh(t_start)
    return cn, psi0


def algorithmic(kernel, w, n_terms):
    """Algorithmic bytes and flops of one launch of a hot kernel on the workload."""
    n, N = w["n_modes"], w["Nr"]
    K = 2 * w["l_max"] + 1
    c128 = 16
    if kernel == "apply":
        # x in, y out, hh table; per interior node T FMAs for Ahat + n^2 complex*real MACs + stencil
        return 2 * c128 * n * N + 8 * K * N, (N - 2) * (2 * n_terms + 4 * n * n) + 30 * n * N
    if kernel == "precond_solve":
        return 3 * c128 * n * N, 16 * n * N      # b and inverse pivots in, x out
    if kernel == "precond_factor":
        return c128 * n * N + 8 * K * N, 20 * n * N
    if kernel == "diagnostics":
        return c128 * n * N + 8 * K * N, (N - 2) * (2 * n_terms + 8 * n * n) + 60 * n * N
    raise KeyError(kernel)


def cpu_oracle_sample(w, psi0, target_s=20.0, max_steps=10, threads=0):
    """Time the CPU oracle on a bounded sample of the same workload."""
    from oracle import oracle as O
    O.build()
    cores = O.set_threads(threads if threads > 0 else (os.cpu_count() or 1))
    cn, _ = make_solver(O.OracleCNM, w, psi0)
    t0 = time.perf_counter()
    cn.step(1)   # warm-up step (first-touch of the assembled operators)
    first = time.perf_counter() - t0
    steps = int(max(1, min(max_steps, math.floor(target_s / max(first, 1e-3)))))
    t0 = time.perf_counter()
    for k in range(2, 2 + steps):
        cn.step(k)
    el = time.perf_counter() - t0
    value = w["n_modes"] * w["Nr"] * steps / el
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} CN steps of the {w['workload']} workload ({w['n_modes']} modes x {w['Nr']} nodes) "
                      f"after 1 warm-up step, oracle restatement (assembled CSR, OpenMP) on {cores} threads, "
                      f"{el:.1f} s"}, steps, el


def run_reference(args):
    ws, rank, _ = dist_env()
    w = dict(WORKLOAD)
    if rank != 0:
        return 0
    from boson_cloud_binary_b200.initial_state import hydrogenic_on_primary
    r = np.linspace(w["epsilon"], w["epsilon"] + w["L"], w["Nr"])
    modes = [(l, m) for l in range(w["l_max"] + 1) for m in range(-l, l + 1) if (l - m) % 2 == 0]
    psi0 = hydrogenic_on_primary(r, modes, w["mu"], w["q"], w["R"])
    base, steps, el = cpu_oracle_sample(w, psi0, target_s=30.0, max_steps=max(1, min(args.steps, 10)))
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": ws,
            "steps": steps, "warmup": 1, "ms_per_step": 1e3 * el / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {k: w[k] for k in ("workload", "Nr", "l_max", "n_modes", "dt", "precision")},
            "cpu_baseline": base, "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from boson_cloud_binary_b200 import CrankNicolsonModes, select_device
    from boson_cloud_binary_b200.initial_state import hydrogenic_on_primary
    select_device(local)
    w = dict(WORKLOAD)
    r = np.linspace(w["epsilon"], w["epsilon"] + w["L"], w["Nr"])
    modes = [(l, m) for l in range(w["l_max"] + 1) for m in range(-l, l + 1) if (l - m) % 2 == 0]
    psi0 = hydrogenic_on_primary(r, modes, w["mu"], w["q"], w["R"])
    cn, _ = make_solver(CrankNicolsonModes, w, psi0)
    T = cn.coupling_info()[1]

    def barrier():
        if dist is not None:
            dist.barrier()

    k = 0
    for _ in range(args.warmup):
        k += 1
        cn.step(k)
    # device-timed region, inputs resident in HBM (psi never leaves the GPU); no
    # per-kernel events inside it
    iters = []
    barrier()
    with ClockSampler(local) as clocks:
        cn.timer_start()
        for _ in range(args.steps):
            k += 1
            d = cn.step(k)
            iters.append(d["iterations"])
        ms = cn.timer_stop()
    barrier()
    # per-kernel device time of the four hot kernel classes on a further stretch of
    # the same run (events around every launch of those classes)
    prof_steps = max(1, min(args.steps, 50))
    cn.set_profiling(True)
    cn.timer_start()
    for _ in range(prof_steps):
        k += 1
        cn.step(k)
    prof_ms = cn.timer_stop()
    kt = {name: cn.kernel_times(name) for name in ("apply", "precond_solve", "precond_factor", "diagnostics")}
    cn.set_profiling(False)
    plan = cn.plan_info()
    if dist is not None:
        import torch
        tt = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    units = w["n_modes"] * w["Nr"] * args.steps * ws
    value = units / (ms / 1e3)

    # end to end through the public API with host buffers: upload the state from
    # pinned host memory, run the steps (each returns its diagnostics to the host),
    # download the final state (the snapshot the reference writes at save_every).
    try:
        import torch
        host = torch.empty(2 * w["n_modes"] * w["Nr"], dtype=torch.float64, pin_memory=True).numpy()
    except Exception:
        host = np.empty(2 * w["n_modes"] * w["Nr"])
    host[:] = cn.psi.view(np.float64)
    diag_bytes = 8 * (12 + 4 * w["n_modes"])
    barrier()
    t0 = time.perf_counter()
    cn.psi = host.view(np.complex128)
    for _ in range(args.steps):
        k += 1
        cn.step(k)
    host[:] = cn.psi.view(np.float64)
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        import torch
        tt = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    state_bytes = 16 * w["n_modes"] * w["Nr"]
    e2e = {"value": units / e2e_s, "unit": UNIT, "h2d_bytes_per_step": state_bytes / args.steps,
           "d2h_bytes_per_step": diag_bytes + state_bytes / args.steps,
           "note": "state uploaded once and downloaded once per timed run (save_every = steps); "
                   "diagnostics returned to the host every step"}

    hbm, bf16, src = peaks()
    from boson_cloud_binary_b200 import measure_fp64_peak
    fp64_peak = measure_fp64_peak()
    dom = max(kt, key=lambda kname: kt[kname][0])
    tot, launches = kt[dom]
    avg_s = tot / max(launches, 1) / 1e3
    nbytes, nflops = algorithmic(dom, w, T)
    # The schema's roofline is the HBM one; the operator kernel is bound by the FP64 FMA
    # pipe instead, so its compute roofline (against the FP64 peak measured on this
    # device by cnm_measure_fp64_peak) is reported beside it.
    roof = {"kernel": dom, "bound": "hbm", "achieved": nbytes / avg_s / 1e9, "peak": hbm, "unit": "GB/s",
            "frac": nbytes / avg_s / 1e9 / hbm, "traffic": NCU_TRAFFIC_BYTES,
            "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback",
            "algorithmic_bytes_per_launch": nbytes, "algorithmic_flops_per_launch": nflops,
            "avg_launch_us": avg_s * 1e6, "launches": launches,
            "fp64": {"achieved_tflops": nflops / avg_s / 1e12, "peak_tflops": fp64_peak,
                     "frac": nflops / avg_s / 1e12 / fp64_peak,
                     "peak_source": "measured here (cnm_measure_fp64_peak: FP64 FMA chains, device events)"}}
    kshare = {kname: {"ms": v[0], "launches": v[1], "share_of_step": v[0] / prof_ms} for kname, v in kt.items()}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": w["workload"], "Nr": w["Nr"], "L": w["L"], "l_max": w["l_max"],
                       "n_modes": w["n_modes"], "mu": w["mu"], "q": w["q"], "R": w["R"], "dt": w["dt"],
                       "precision": "fp64", "parallelism": f"replicas{ws}",
                       "l2": "working set > L2 (20 vectors of 14.4 MB plus pivots)",
                       "bicgstab_iterations_mean": float(np.mean(iters)) if iters else None,
                       "plan": plan, "kernel_breakdown_steps": prof_steps},
            "roofline": roof, "kernels": kshare, "e2e": e2e, "clocks": clocks.summary(),
            "gpu_launches": None}
    # launches of our kernels in the timed region (counted by the instrumented classes plus
    # the streaming/scalar kernels per BiCGSTAB iteration and per step)
    # per step: 1 right-hand-side apply, 1 factorisation, 1 Woodbury set-up, 1 residual
    # apply, 1 diagnostics, start, mask, 3 sink projections, 1 hh table, 1 absorber
    # moments, 1 projector, 1 slot sum = 15; per iteration 2 solves, 2 applies, 2
    # Woodbury corrections, 1 update = 7 (with sinks, as in this workload)
    it_total = int(np.sum(iters))
    line["gpu_launches"] = int(it_total * 7 + args.steps * 15)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        base, _, _ = cpu_oracle_sample(w, psi0)
        line["cpu_baseline"] = base
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
