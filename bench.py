#!/usr/bin/env python
"""Benchmark of the Crank-Nicolson step: mode*node*steps/s, mixed precision against FP64.

Default workload (the headline: the mixed-precision solver against the plain FP64 path on
the same binary): 2p hydrogenic cloud (n=2, l=1, m=1) on the primary, mu=0.25, q=0.5,
R=50, back-reaction + GW decay + accretion + s-wave absorption on; l_max=12 (91 modes);
N=40000, L=4000, r_ex=1500; dt=0.5 (steps_per_period = P0/0.5); both arms stop at the
fp64 relative residual 1e-12.  The mixed arm solves each step by defect correction
(complex64 inner iterations on the tensor-core coupling apply, fp64 residuals, dots,
diagnostics and orbit); the FP64 arm is the complex128 drop-in.  `value` is the mixed
arm; the FP64 arm, their ratio and the difference of the two solutions after the run are
reported beside it.  Other workloads (--config): c2 (the FP64 drop-in on 45 modes x
20000 nodes, the configuration the FP64 path was first measured on), c1 (15 modes x 3000
nodes, fixed orbit), c4 (the batched sweep: 64 binaries of uneven N and l_max from seed 0,
bench_c4_binaries.json, mixed against FP64), c5 (the stress case on the FP64 path:
equal-mass counter-rotating binary, (3,2,2) cloud, 153 modes x 65536 nodes, dt 0.25).  Keys the configurations do not name take the reference's minimal-
example values: ramp_periods=2, epsilon=0, epsilon_smear=2, M_c=0.01, mask 0.85/1/6.  The
timed steps start one initial period after the start-up ramp (absorbers, back-reaction
and orbit evolution at full strength).  Synthetic input: the analytic 2p state projected
on the modes.

Arms:
  (default)          the CUDA path through the Python binding of the C ABI;
  --impl reference   the reference's CPU algorithm on the host cores: the oracle
                     restatement (oracle/, C++17 + OpenMP), the reference itself being
                     unbuildable here (Eigen 3 and GSL absent).
Under torchrun each rank advances its own replica (no collective on the data path;
"replicas only"); timings are maxed over ranks.
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

BASE = dict(mu=0.25, q=0.5, R=50.0, dt=0.5, counter=False, absorption=True, evolve_orbit=True, M_c=0.01,
            epsilon=0.0, epsilon_smear=2.0, ramp_periods=2.0, mask=[0.85, 1.0, 6],
            state="2p hydrogenic (2,1,1) on the primary")
WORKLOADS = {
    "c3": dict(BASE, workload="mixed_vs_fp64_single_binary_l12_N40000", Nr=40000, L=4000.0, l_max=12, n_modes=91,
               r_ex=1500.0, precision="mixed", tolerance=1e-12),
    "c2": dict(BASE, workload="fp64_single_binary_evolving_orbit", Nr=20000, L=2000.0, l_max=8, n_modes=45,
               r_ex=1500.0, precision="fp64", tolerance=1e-10),
    "c1": dict(BASE, workload="fp64_single_binary_fixed_orbit_l4_N3000", Nr=3000, L=300.0, l_max=4, n_modes=15,
               mu=0.2, q=0.1, R=30.0, dt=1.0, r_ex=250.0, evolve_orbit=False, precision="fp64", tolerance=1e-10),
}
WORKLOADS["c5"] = dict(BASE, workload="fp64_stress_counter_rotating_l16_N65536", Nr=65536, L=6000.0, l_max=16,
                       n_modes=153, mu=0.3, q=1.0, R=60.0, dt=0.25, counter=True, r_ex=5000.0, precision="fp64",
                       tolerance=1e-10, state="3d hydrogenic (3,2,2) on the primary", atom=(3, 2, 2))
WORKLOADS["c4"] = dict(BASE, workload="batched_sweep_64_binaries_seed0", precision="mixed", tolerance=1e-12,
                       batch_file="bench_c4_binaries.json")
METRIC = "CN mode*node*steps/s"


def c4_binaries(count=64, seed=0):
    """The batched sweep's binaries, drawn per binary in this order from
    numpy.random.default_rng(seed): q ~ U[0.05, 1], R ~ U[20, 80], mu from {0.1, 0.15, 0.2,
    0.3}, l_max from {4, 6, 8, 10}, N ~ U{4000..32000} (L = N / 10), the initial state: a
    hydrogenic (2,1,1) or (3,2,2) atom on the primary, or a spherical Gaussian of width
    sigma ~ U[5, 20] (sigma drawn only for a Gaussian).  dt = 0.5, absorption on."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        q = float(rng.uniform(0.05, 1.0))
        R = float(rng.uniform(20.0, 80.0))
        mu = float(rng.choice([0.1, 0.15, 0.2, 0.3]))
        l_max = int(rng.choice([4, 6, 8, 10]))
        N = int(rng.integers(4000, 32001))
        kind = int(rng.integers(0, 3))
        if kind == 0:
            state = {"kind": "hydrogenic", "n": 2, "l": 1, "m": 1}
        elif kind == 1:
            state = {"kind": "hydrogenic", "n": 3, "l": 2, "m": 2}
        else:
            state = {"kind": "gaussian", "sigma": float(rng.uniform(5.0, 20.0))}
        out.append({"q": q, "R": R, "mu": mu, "l_max": l_max, "Nr": N, "L": N / 10.0, "dt": 0.5, "state": state})
    return out


def c4_load():
    """The frozen list (bench_c4_binaries.json), checked against its generator."""
    with open(os.path.join(ROOT, WORKLOADS["c4"]["batch_file"])) as f:
        frozen = json.load(f)
    if frozen != c4_binaries():
        raise RuntimeError("bench_c4_binaries.json differs from c4_binaries(seed 0)")
    return frozen


def c4_modes(l_max):
    return [(l, m) for l in range(l_max + 1) for m in range(-l, l + 1) if (l - m) % 2 == 0]


def c4_state(b):
    """Initial state of one binary of the sweep (device generator for the atoms)."""
    from boson_cloud_binary_b200 import gaussian_state, hydrogenic_state
    r = np.linspace(BASE["epsilon"], BASE["epsilon"] + b["L"], b["Nr"])
    modes = c4_modes(b["l_max"])
    st = b["state"]
    if st["kind"] == "gaussian":
        return gaussian_state(r, modes, st["sigma"])
    return hydrogenic_state(r, modes, b["mu"], b["q"], b["R"], n=st["n"], l=st["l"], m=st["m"])
UNIT = "mode*node*steps/s"

# DRAM traffic (read + write) per launch of each measured kernel class, from the ncu
# captures summarised in profiles/ (bytes per launch on the named workload).
NCU_TRAFFIC = {
    ("c2", "apply"): 242.035482e9 * 73.952e-6,   # profiles/k_apply5_fp64_binary_n45_N20000.md
}


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
    """nvidia-smi clocks and throttle reasons sampled while the measured steps run."""

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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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


def initial_state(w, device=False):
    """The workload's hydrogenic atom on the primary projected on the modes: by the device
    generator (cnm_hydrogenic_state) for the GPU arm, by the host generator for the CPU arm
    (the same quadrature; the two agree to 1e-12)."""
    from boson_cloud_binary_b200.initial_state import hydrogenic_on_primary
    r = np.linspace(w["epsilon"], w["epsilon"] + w["L"], w["Nr"])
    modes = [(l, m) for l in range(w["l_max"] + 1) for m in range(-l, l + 1) if (l - m) % 2 == 0]
    n, l, m = w.get("atom", (2, 1, 1))
    if device:
        from boson_cloud_binary_b200 import hydrogenic_state
        return hydrogenic_state(r, modes, w["mu"], w["q"], w["R"], n=n, l=l, m=m)
    return hydrogenic_on_primary(r, modes, w["mu"], w["q"], w["R"], n=n, l=l, m=m)


def make_solver(cls, w, psi0, precision=None):
    kw = {} if precision is None else {"precision": precision}
    cn = cls(w["Nr"], w["L"], w["dt"], w["epsilon"], w["l_max"], w["mu"], w["M_c"], w["q"], 0.0, w["R"],
             w["counter"], w["absorption"], 10 ** 9, w["ramp_periods"], w["epsilon_smear"], **kw)
    cn.set_initial_state_full(psi0)
    cn.evolve_orbit = w["evolve_orbit"]
    cn.steps_per_period = cn.P / w["dt"]
    cn.tolerance = w["tolerance"]
    cn.initialize()
    cn.build_damping_mask(*w["mask"])
    cn.run(10 ** 9, w["r_ex"])
    # one initial period past the start-up ramp: absorbers and back-reaction at full strength
    t_start = (w["ramp_periods"] + 1.0) * cn.P
    cn.t_i = t_start
    cn.refresh(t_start)
    return cn


def hh_table(w, cn):
    """Radial multipole weights h_l*(r_i) of the current orbit (the kernels' hh table)."""
    K = 2 * w["l_max"] + 1
    r = cn.r
    R1, R2, q, Mt = cn.R1, cn.R2, cn.q, cn.M1 + cn.M2
    hh = np.zeros((K, len(r)))
    for l in range(K):
        f1 = 1 / (1 + q) * np.minimum(r, R1) ** l / np.maximum(r, R1) ** (l + 1)
        f2 = q / (1 + q) * np.minimum(r, R2) ** l / np.maximum(r, R2) ** (l + 1)
        hh[l] = -w["mu"] * Mt * (f1 + (-1) ** l * f2)
    hh[:, 0] = hh[:, -1] = 0.0
    return hh


def tc_mma_flops(w, cn):
    """Tensor-core flops one tensor-core apply issues: per tile of nt nodes, multipoles 0 ..
    the tile's cut (the highest one above 1e-9 of the monopole at some node of the tile, and
    at least the multipoles every tile runs), one M128 x N(2 nt) x K16 MMA per non-zero
    16-column Gaunt slice (M = 128 mode rows, padded; N = the tile's 2 nt node components)."""
    kp, nblk, lc_min, nt = cn.tc_blocks()
    hh = hh_table(w, cn)
    N = w["Nr"]
    slices = 0
    for i0 in range(0, N, nt):
        h = np.abs(hh[:, i0:i0 + nt])
        keep = (h[1:] > 1e-9 * h[0][None, :]).any(axis=1)
        lc = max(lc_min, int(np.max(np.nonzero(keep)[0]) + 1) if keep.any() else 0)
        slices += int(np.sum(nblk[:lc + 1]))
    return slices * 2 * 128 * (2 * nt) * 16


def algorithmic(kernel, w, n_terms, cn=None):
    """Algorithmic bytes and flops of one launch of a hot kernel on the workload."""
    n, N = w["n_modes"], w["Nr"]
    K = 2 * w["l_max"] + 1
    c128, c64 = 16, 8
    if kernel == "apply":
        # x in, y out, hh table; per interior node 2T FMA flops for Ahat + n^2 complex*real MACs + stencil
        return 2 * c128 * n * N + 8 * K * N, (N - 2) * (2 * n_terms + 4 * n * n) + 30 * n * N
    if kernel == "tc_apply":
        # x in, y out (complex64), hh table, one fused reduction operand; tensor flops issued
        return 3 * c64 * n * N + 8 * K * N, tc_mma_flops(w, cn)
    if kernel == "precond_solve":
        return 3 * c128 * n * N, 16 * n * N      # b and inverse pivots in, x out
    if kernel == "precond_solve32":
        return 3 * c64 * n * N, 16 * n * N
    if kernel == "precond_factor":
        return c128 * n * N + 8 * K * N, 20 * n * N
    if kernel == "diagnostics":
        return c128 * n * N + 8 * K * N, (N - 2) * (2 * n_terms + 8 * n * n) + 60 * n * N
    raise KeyError(kernel)


def cpu_oracle_sample(w, psi0, target_s=20.0, max_steps=10, threads=0):
    """Time the CPU oracle on a bounded sample of the same workload (fp64, the reference's
    algorithm; the workload's tolerance)."""
    from oracle import oracle as O
    O.build()
    cores = O.set_threads(threads if threads > 0 else (os.cpu_count() or 1))
    t0 = time.perf_counter()
    cn = make_solver(O.OracleCNM, w, psi0)
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    cn.step(1)   # warm-up step (first touch of the assembled operators)
    first = time.perf_counter() - t0
    steps = int(max(1, min(max_steps, math.floor(target_s / max(first, 1e-3)))))
    t0 = time.perf_counter()
    for k in range(2, 2 + steps):
        cn.step(k)
    el = time.perf_counter() - t0
    value = w["n_modes"] * w["Nr"] * steps / el
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} CN steps of the {w['workload']} workload ({w['n_modes']} modes x {w['Nr']} nodes, "
                      f"tolerance {w['tolerance']:g}) after 1 warm-up step, oracle restatement (assembled CSR, "
                      f"OpenMP) on {cores} threads, {el:.1f} s (set-up {setup:.0f} s)"}, steps, el


def host_memory_gb():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return 0.0


def oracle_memory_gb(w):
    """Host memory of the oracle's assembled operators (about nine n^2 N complex128 arrays;
    measured 13.8 GB at 91 modes x 4000 nodes)."""
    return 13.8 * (w["n_modes"] / 91.0) ** 2 * (w["Nr"] / 4000.0)


def c4_workload(b):
    """One binary of the batched sweep as a single-binary workload dict."""
    w = dict(BASE, workload="batched_sweep_binary", Nr=b["Nr"], L=b["L"], l_max=b["l_max"],
             n_modes=len(c4_modes(b["l_max"])), mu=b["mu"], q=b["q"], R=b["R"], dt=b["dt"], r_ex=0.75 * b["L"],
             precision="fp64", tolerance=WORKLOADS["c4"]["tolerance"])
    return w


def run_reference_batch(args):
    """CPU arm of the batched sweep: the oracle on the three binaries with the smallest
    assembled operators (the rest need tens of GB of host memory), a bounded sample of
    steps each; the metric over the sample."""
    binaries = sorted(c4_load(), key=lambda b: len(c4_modes(b["l_max"])) ** 2 * b["Nr"])[:3]
    units, secs, parts, cores = 0, 0.0, [], 0
    for b in binaries:
        w = c4_workload(b)
        base, steps, el = cpu_oracle_sample(w, c4_state_host(b), target_s=10.0, max_steps=max(1, min(args.steps, 4)))
        units += w["n_modes"] * w["Nr"] * steps
        secs += el
        cores = base["cores"]
        parts.append(f"{w['n_modes']}x{w['Nr']} ({steps} steps)")
    value = units / secs
    base = {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "oracle restatement (assembled CSR, OpenMP) on the three binaries of the sweep with the "
                      "smallest operators: " + ", ".join(parts) + f", {secs:.1f} s"}
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic", "config": {"workload": WORKLOADS["c4"]["workload"],
                                                           "precision": "fp64"},
            "cpu_baseline": base, "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}


def c4_state_host(b):
    """The host generator's state of one binary (the CPU arm runs without a GPU)."""
    from boson_cloud_binary_b200.cnm import gaussian_state
    from boson_cloud_binary_b200.initial_state import hydrogenic_on_primary
    r = np.linspace(BASE["epsilon"], BASE["epsilon"] + b["L"], b["Nr"])
    modes = c4_modes(b["l_max"])
    st = b["state"]
    if st["kind"] == "gaussian":
        return gaussian_state(r, modes, st["sigma"])
    return hydrogenic_on_primary(r, modes, b["mu"], b["q"], b["R"], n=st["n"], l=st["l"], m=st["m"])


def oracle_sample_workload(w, budget_gb=8.0):
    """The workload the CPU oracle is timed on: the workload itself when its assembled
    operators fit in `budget_gb` (and half the host's free memory), else the same binary
    on fewer nodes at the same spacing (the oracle's cost per mode*node*step does not
    depend on N: every operator is a pass over n^2 N stored entries).  Returns the
    workload and a note."""
    have = host_memory_gb()
    budget = min(budget_gb, 0.5 * have) if have else budget_gb
    need = oracle_memory_gb(w)
    if need <= budget:
        return w, ""
    dr = w["L"] / (w["Nr"] - 1)
    n2 = max(600, int(w["Nr"] * budget / need))
    w2 = dict(w, Nr=n2, L=dr * (n2 - 1))
    w2["r_ex"] = min(w["r_ex"], 0.75 * w2["L"])
    return w2, (f"the same binary on {n2} of its {w['Nr']} nodes at its spacing dr = {dr:g} (the full grid's "
                f"assembled operators need about {need:.0f} GB of host memory)")


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    if args.config == "c4":
        print(json.dumps(run_reference_batch(args)), flush=True)
        return 0
    w_full = dict(WORKLOADS[args.config])
    w, note = oracle_sample_workload(w_full)
    psi0 = initial_state(w)
    base, steps, el = cpu_oracle_sample(w, psi0, target_s=30.0, max_steps=max(1, min(args.steps, 10)))
    if note:
        base["sample"] += "; " + note
    w = w_full
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": ws,
            "steps": steps, "warmup": 1, "ms_per_step": 1e3 * el / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {k: w[k] for k in ("workload", "Nr", "l_max", "n_modes", "dt", "precision")},
            "cpu_baseline": base, "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def reduce_max(v, dist, device):
    """The largest value over the ranks of the process group (v itself without one)."""
    if dist is None:
        return v
    import torch
    tt = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def whole_job(units_per_rank, ms_max, ws):
    """Replicas: every rank advances its own binary, so the job's units are the ranks' sum and
    its time the slowest rank's (ms_max, already maxed over the ranks)."""
    units = units_per_rank * ws
    return units, units / (ms_max / 1e3)


def timed_steps(cn, k0, steps):
    """Device-event time (ms) of `steps` steps with the state resident in HBM, the launches
    the steps made, and the solver iterations / passes of each step."""
    iters = []
    n0 = cn.launch_count()
    cn.timer_start()
    for q in range(steps):
        d = cn.step(k0 + q)
        iters.append(d["iterations"])
    ms = cn.timer_stop()
    return ms, cn.launch_count() - n0, iters


def kernel_breakdown(cn, k0, steps):
    cn.set_profiling(True)
    cn.timer_start()
    for q in range(steps):
        cn.step(k0 + q)
    prof_ms = cn.timer_stop()
    names = ("apply", "tc_apply", "precond_solve", "precond_solve32", "precond_factor", "diagnostics")
    kt = {name: cn.kernel_times(name) for name in names}
    cn.set_profiling(False)
    return {k: {"ms": v[0], "launches": v[1], "share_of_step": v[0] / prof_ms} for k, v in kt.items() if v[1] > 0}


def run_ours(args):
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from boson_cloud_binary_b200 import CrankNicolsonModes, select_device, measure_fp64_peak
    select_device(local)
    w = dict(WORKLOADS[args.config])
    mixed = w["precision"] == "mixed"
    psi0 = initial_state(w, device=True)
    cn = make_solver(CrankNicolsonModes, w, psi0, w["precision"])
    ref = make_solver(CrankNicolsonModes, w, psi0, "fp64") if mixed and not args.no_fp64_arm else None
    # launch plans by timed search (the operator kernel's row groups, the tensor-core apply's
    # Gaunt stages), before any timed work
    tuning = cn.autotune() if not args.no_autotune else None
    tuning_ref = ref.autotune() if ref is not None and not args.no_autotune else None
    T = cn.coupling_info()[1]

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        return reduce_max(v, dist, f"cuda:{local}")

    k = 1
    for _ in range(args.warmup):
        cn.step(k)
        if ref is not None:
            ref.step(k)
        k += 1
    # clocks over a window of at least two seconds: a soak of the same steps (both arms,
    # so their states stay aligned), then the timed region
    barrier()
    with ClockSampler(local) as clocks:
        t_soak = time.perf_counter()
        while time.perf_counter() - t_soak < 2.0:
            cn.step(k)
            if ref is not None:
                ref.step(k)
            k += 1
        ms, launches, iters = timed_steps(cn, k, args.steps)
    if ref is not None:
        ms_ref, _, iters_ref = timed_steps(ref, k, args.steps)
    k += args.steps
    barrier()
    ms = max_over_ranks(ms)
    units, value = whole_job(w["n_modes"] * w["Nr"] * args.steps, ms, ws)
    accuracy = None
    if ref is not None:
        ms_ref = max_over_ranks(ms_ref)
        pa, pb = cn.psi, ref.psi
        mu_dr = w["mu"] * (w["L"] / (w["Nr"] - 1))
        ma, mb = mu_dr * np.sum(np.abs(pa) ** 2), mu_dr * np.sum(np.abs(pb) ** 2)
        accuracy = {"steps_compared": k - 1, "U_lm_rel": float(np.linalg.norm(pa - pb) / np.linalg.norm(pb)),
                    "mass_rel": float(abs(ma - mb) / mb), "R_rel": float(abs(cn.R - ref.R) / ref.R),
                    "against": "the FP64 GPU path (the drop-in, pinned to the CPU oracle by the parity tests) "
                               "from the same state, both at fp64 relative residual 1e-12"}

    # per-kernel device time on a further stretch of the same run (events around every
    # launch of the hot kernel classes)
    prof_steps = max(1, min(args.steps, 20))
    kshare = kernel_breakdown(cn, k, prof_steps)
    kshare_ref = kernel_breakdown(ref, k, prof_steps) if ref is not None else None
    k += prof_steps
    plan = cn.plan_info()

    # end to end through the public API with host buffers: the state uploaded from pinned
    # host memory, the steps (each returns its diagnostics to the host), the final state
    # downloaded (the snapshot the reference writes at save_every)
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
        cn.step(k)
        k += 1
    host[:] = cn.psi.view(np.float64)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    state_bytes = 16 * w["n_modes"] * w["Nr"]
    e2e = {"value": units / e2e_s, "unit": UNIT, "h2d_bytes_per_step": state_bytes / args.steps,
           "d2h_bytes_per_step": diag_bytes + state_bytes / args.steps,
           "note": "state uploaded once and downloaded once per timed run (save_every = steps); "
                   "diagnostics returned to the host every step"}

    # roofline of the dominant kernel class of the measured arm
    hbm, bf16, src = peaks()
    dom = max(kshare, key=lambda kname: kshare[kname]["ms"])
    avg_s = kshare[dom]["ms"] / kshare[dom]["launches"] / 1e3
    nbytes, nflops = algorithmic(dom, w, T, cn)
    roof = {"kernel": dom, "avg_launch_us": avg_s * 1e6, "launches": kshare[dom]["launches"],
            "algorithmic_bytes_per_launch": nbytes, "algorithmic_flops_per_launch": nflops,
            "traffic": NCU_TRAFFIC.get((args.config, dom))}
    if dom == "tc_apply":
        # the binding roofline is the one with the longer lower-bound time: algorithmic bytes
        # at the HBM peak, or the issued tensor-core flops at the dense fp16 peak
        tensor = {"achieved": nflops / avg_s / 1e12, "peak": bf16, "unit": "TFLOP/s",
                  "frac": nflops / avg_s / 1e12 / bf16,
                  "peak_source": (f"{src} (MEASURED_PEAKS.json bf16_tflops: dense fp16 and bf16 rates are "
                                  "the same)") if src == "measured" else "fallback"}
        memory = {"achieved": nbytes / avg_s / 1e9, "peak": hbm, "unit": "GB/s", "frac": nbytes / avg_s / 1e9 / hbm,
                  "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback"}
        if nbytes / (hbm * 1e9) >= nflops / (bf16 * 1e12):
            roof.update({"bound": "hbm", **memory, "tensor": tensor})
        else:
            roof.update({"bound": "tensor", **tensor, "hbm": memory})
    else:
        fp64_peak = measure_fp64_peak()
        roof.update({"bound": "hbm", "achieved": nbytes / avg_s / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": nbytes / avg_s / 1e9 / hbm,
                     "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback",
                     "fp64": {"achieved_tflops": nflops / avg_s / 1e12, "peak_tflops": fp64_peak,
                              "frac": nflops / avg_s / 1e12 / fp64_peak,
                              "peak_source": "measured here (cnm_measure_fp64_peak: FP64 FMA chains, device "
                                             "events)"}})

    cfg = {k_: w[k_] for k_ in ("workload", "Nr", "L", "l_max", "n_modes", "mu", "q", "R", "dt", "precision",
                                "tolerance")}
    cfg.update({"parallelism": f"replicas{ws}", "l2": "working set > L2 (the state alone is "
                f"{w['n_modes'] * w['Nr'] * 16 / 1e6:.0f} MB complex128)",
                "iterations_mean": float(np.mean(iters)) if iters else None, "plan": plan, "autotune": tuning,
                "autotune_fp64_arm": tuning_ref,
                "kernel_breakdown_steps": prof_steps})
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64+c128" if mixed else "c128", "data": "synthetic", "config": cfg,
            "roofline": roof, "kernels": kshare, "e2e": e2e, "clocks": clocks.summary(),
            "gpu_launches": int(launches)}
    if ref is not None:
        line["fp64_arm"] = {"value": units / (ms_ref / 1e3), "ms_per_step": ms_ref / args.steps,
                            "iterations_mean": float(np.mean(iters_ref)), "kernels": kshare_ref}
        line["mixed_over_fp64"] = ms_ref / ms
        line["accuracy"] = accuracy
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        ws_, note = oracle_sample_workload(w)
        base, _, _ = cpu_oracle_sample(ws_, psi0 if ws_ is w else initial_state(ws_), target_s=20.0, max_steps=5)
        if note:
            base["sample"] += "; " + note
        line["cpu_baseline"] = base
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch(args):
    """The batched sweep: 64 binaries of uneven N and l_max stepped together (cnm_batch_step:
    every binary's step queued on its own stream before any is completed), mixed precision,
    the same binaries in FP64 beside it.  Wall time of the synchronous batch steps (the
    library returns after every binary's step completed)."""
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from boson_cloud_binary_b200 import Batch, select_device
    select_device(local)
    w = dict(WORKLOADS["c4"])
    binaries = c4_load()
    states = [c4_state(b) for b in binaries]

    def build(precision):
        args_ = [(b["Nr"], b["L"], b["dt"], BASE["epsilon"], b["l_max"], b["mu"], BASE["M_c"], b["q"], 0.0, b["R"],
                  BASE["counter"], BASE["absorption"], 10 ** 9, BASE["ramp_periods"], BASE["epsilon_smear"])
                 for b in binaries]
        bt = Batch(args_, precision=precision)
        for b, cn, psi0 in zip(binaries, bt.binaries, states):
            cn.set_initial_state_full(psi0)
            cn.evolve_orbit = True
            cn.steps_per_period = cn.P / b["dt"]
            cn.tolerance = w["tolerance"]
            cn.initialize()
            cn.build_damping_mask(*BASE["mask"])
            cn.run(10 ** 9, 0.75 * b["L"])
            t_start = (BASE["ramp_periods"] + 1.0) * cn.P
            cn.t_i = t_start
            cn.refresh(t_start)
        return bt

    t0 = time.perf_counter()
    mixed = build("mixed")
    setup_s = time.perf_counter() - t0
    fp64 = None if args.no_fp64_arm else build("fp64")
    units_per_step = sum(len(c4_modes(b["l_max"])) * b["Nr"] for b in binaries)

    def timed(bt, k0, steps):
        n0 = sum(cn.launch_count() for cn in bt.binaries)
        t = time.perf_counter()
        for q in range(steps):
            bt.step(k0 + q)
        return time.perf_counter() - t, sum(cn.launch_count() for cn in bt.binaries) - n0

    k = 1
    for _ in range(args.warmup):
        mixed.step(k)
        if fp64 is not None:
            fp64.step(k)
        k += 1
    with ClockSampler(local) as clocks:
        t_soak = time.perf_counter()
        while time.perf_counter() - t_soak < 2.0:
            mixed.step(k)
            if fp64 is not None:
                fp64.step(k)
            k += 1
        if dist is not None:
            dist.barrier()
        el, launches = timed(mixed, k, args.steps)
    el64 = timed(fp64, k, args.steps)[0] if fp64 is not None else None
    k += args.steps
    el = reduce_max(el, dist, f"cuda:{local}")
    if el64 is not None:
        el64 = reduce_max(el64, dist, f"cuda:{local}")
    units_job, value = whole_job(units_per_step * args.steps, 1e3 * el, ws)
    # per-class kernel times over the binaries (device events on each binary's stream)
    names = ("apply", "tc_apply", "precond_solve", "precond_solve32", "precond_factor", "diagnostics")
    for cn in mixed.binaries:
        cn.set_profiling(True)
    prof_steps = max(1, min(args.steps, 5))
    for q in range(prof_steps):
        mixed.step(k + q)
    k += prof_steps
    kt = {name: [0.0, 0, 0.0] for name in names}   # ms, launches, algorithmic bytes
    for b, cn in zip(binaries, mixed.binaries):
        wb = {"n_modes": len(c4_modes(b["l_max"])), "Nr": b["Nr"], "l_max": b["l_max"]}
        for name in names:
            ms, nl = cn.kernel_times(name)
            if nl > 0:
                nbytes, _ = algorithmic(name, wb, cn.coupling_info()[1], cn) if name != "tc_apply" else \
                    (3 * 8 * wb["n_modes"] * wb["Nr"] + 8 * (2 * wb["l_max"] + 1) * wb["Nr"], 0)
                kt[name][0] += ms
                kt[name][1] += nl
                kt[name][2] += nbytes * nl
        cn.set_profiling(False)
    kshare = {n_: {"ms": v[0], "launches": v[1]} for n_, v in kt.items() if v[1] > 0}
    dom = max(kshare, key=lambda n_: kshare[n_]["ms"])
    hbm, _, src = peaks()
    achieved = kt[dom][2] / (kt[dom][0] / 1e3) / 1e9
    roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback",
            "launches": kt[dom][1], "avg_launch_us": kt[dom][0] / kt[dom][1] * 1e3,
            "algorithmic_bytes": "sum over the binaries' launches of each launch's algorithmic bytes", "traffic": None}
    # end to end: every binary's state uploaded from pinned host memory, K steps, the states
    # downloaded
    try:
        import torch
        hosts = [torch.empty(2 * s_.size, dtype=torch.float64, pin_memory=True).numpy() for s_ in states]
    except Exception:
        hosts = [np.empty(2 * s_.size) for s_ in states]
    for h_, cn in zip(hosts, mixed.binaries):
        h_[:] = cn.psi.view(np.float64)
    t0 = time.perf_counter()
    for h_, cn in zip(hosts, mixed.binaries):
        cn.psi = h_.view(np.complex128)
    for q in range(args.steps):
        mixed.step(k + q)
    for h_, cn in zip(hosts, mixed.binaries):
        h_[:] = cn.psi.view(np.float64)
    e2e_s = reduce_max(time.perf_counter() - t0, dist, f"cuda:{local}")
    state_bytes = sum(16 * s_.size for s_ in states)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64+c128", "data": "synthetic",
            "config": {"workload": w["workload"], "binaries": len(binaries), "units_per_step": units_per_step,
                       "precision": "mixed", "tolerance": w["tolerance"], "parallelism": f"replicas{ws}",
                       "batch_file": w["batch_file"], "setup_s": setup_s,
                       "l2": "working set > L2 (the states alone are %.0f MB complex128)" % (state_bytes / 1e6),
                       "timing": "wall time of synchronous batch steps"},
            "roofline": roof, "kernels": kshare,
            "e2e": {"value": units_job / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": state_bytes / args.steps, "d2h_bytes_per_step": state_bytes / args.steps,
                    "note": "states uploaded once and downloaded once per timed run"},
            "clocks": clocks.summary(), "gpu_launches": int(launches)}
    if el64 is not None:
        line["fp64_arm"] = {"value": units_job / el64, "ms_per_step": 1e3 * el64 / args.steps}
        line["mixed_over_fp64"] = el64 / el
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--config", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the creation-time launch plans")
    ap.add_argument("--no-fp64-arm", action="store_true",
                    help="mixed workload only: skip the FP64 arm beside it (for profiling one arm)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "c4":
        return run_batch(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
