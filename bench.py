#!/usr/bin/env python
"""Benchmark of the Hydist ADI time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|fp32|fp32-refine] [--workload sediment-2048x1024|channel-256x128]
                    [--eager]

A step is one full ADI step (two half-steps, with the concentration sweeps)
of the 2048x1024 sediment workload: dx=dy=5 m, dt=2 s, seeded synthetic
bathymetry, sediment from t=600 s. The state is spun up to t=600 s before
timing so that every timed step runs the sediment sweeps. value is
cell-steps/s (N*M interior cells x steps / device seconds), whole job. Each
step is one replay of the step's CUDA graph (hydist_step_graph), the path the
ensembles and the server take; --eager launches the kernels one by one
(hydist_step).

Multi-GPU: scenarios are independent, so N GPUs run N replicas with no
data-path collective (weak scaling); the time is the max over ranks.

--impl reference times the reference's CPU path: the reference has none
(every computation is a CUDA kernel), so the FP64 CPU restatement of its
time step runs with all host threads, on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from hydist_c_b200 import replicas as R  # noqa: E402

BYTES_PER_CELL_STEP = {  # algorithmic bytes per interior cell and full step
    ("fp64", False): 168, ("fp64", True): 232, ("fp32", False): 112, ("fp32", True): 152}
# Algorithmic bytes per cell of one line-solver launch (FP64), each field the
# kernel's formulas read counted once and each field it writes once:
#   hydraulic sweeps: read u, v, z, H_moi, Htdu, Htdv, visco, Kx1 (Ky1),
#     Tsxw (Tsyw) = 9 x 8 B; write t_z and t_u (t_v) = 2 x 8 B  -> 88 B
#   concentration sweeps: read FS, H_moi, VTH, Fw, t_u, t_v, Htdu, Htdv, Kx,
#     Ky = 10 x 8 B; write tFS = 8 B                             -> 88 B
#     (a concentration sweep is timed over its two launches: the per-cell
#     row kernel k_fs_rows and the line solve)
# The line-solver scratch (3 doubles per unknown) and the concentration rows
# passed between the two launches (4 doubles per cell) are not counted.
# In the FP32 form z is read (8 B) and t_z written (8 B) in FP64, the other
# fields are 4 B: hydraulic 8 + 8 x 4 + 8 + 4 = 52 B, concentration 11 x 4 = 44 B.
SWEEP_BYTES_PER_CELL = {
    "fp64": {"line_solve_hydro_x": 88, "line_solve_hydro_y": 88,
             "line_solve_conc_x": 88, "line_solve_conc_y": 88},
    "fp32": {"line_solve_hydro_x": 52, "line_solve_hydro_y": 52,
             "line_solve_conc_x": 44, "line_solve_conc_y": 44}}


def sweep_cells(name, N, M):
    """Cells one launch of a line solver processes (lines x cells per line)."""
    return {"line_solve_hydro_x": (M - 1) * (N - 1), "line_solve_hydro_y": (N - 1) * (M - 1),
            "line_solve_conc_x": (M - 3) * (N - 1), "line_solve_conc_y": (N - 3) * (M - 1)}[name]


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every 10 ms during a
    region (one sample at its start and one at its end as well, so that a
    region of a few tens of milliseconds still has samples); nvidia-smi at
    100 ms where NVML cannot be opened."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.nvml = None
        self.handle = None
        self.proc = None
        self._halt = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            try:
                import torch
                uuid = str(torch.cuda.get_device_properties(index).uuid)
                self.handle = pynvml.nvmlDeviceGetHandleByUUID(
                    uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                self.handle = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.nvml = pynvml
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
            self.bits = (pynvml.nvmlClocksEventReasonHwSlowdown,
                         pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                         pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                         pynvml.nvmlClocksEventReasonSwPowerCap)
        except Exception:
            self.nvml = None

    def _sample(self):
        n = self.nvml
        mhz = float(n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM))
        mask = int(n.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
        self.samples.append((mhz, mask))

    def _loop(self):
        while not self._halt.wait(0.01):
            try:
                self._sample()
            except Exception:
                return

    def start(self):
        if self.nvml is not None:
            self._sample()
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
            return
        try:
            self.lines = []
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self._halt.set()
            self.t.join()
            self._sample()
            sm = [m for m, _ in self.samples]
            reasons = {nm for _, mask in self.samples for nm, b in zip(self.NAMES, self.bits) if mask & b}
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(self.NAMES, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 100 ms"}


def workload(name: str, rank: int = 0):
    """The scenario of one replica (rank r solves its own seeded scenario)
    and the untimed spin-up steps."""
    from hydist_c_b200 import scenario as S
    from hydist_c_b200.replicas import replica_seed
    if name == "sediment-2048x1024":
        # spin-up to t = 600 s, where the sediment sweeps start
        return S.config1(seed=replica_seed(20260001, rank)), 300
    if name == "channel-256x128":
        return S.config0(seed=replica_seed(20260000, rank)), 0
    if name == "sediment-1024x512":
        # one ensemble member's scenario alone (a state of ~30 fields of
        # 4.2 MB, still larger than L2: the size for per-kernel profiles)
        return S.config3_member(0, seed=replica_seed(20263000, rank)), 150
    raise SystemExit(f"unknown workload {name}")


def cpu_baseline(bundle, steps: int, threads: int):
    """The FP64 CPU oracle on the host cores, on the same workload with the
    sediment sweeps on from t = 0 (so each step does the timed work)."""
    from oracle import oracle as O
    b = dict(bundle)
    b["options"] = dict(bundle["options"], sediment_start=0.0, bed_change_start=0.0)
    o = O.OracleSim(b, nthreads=threads)
    o.step(1)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    cells = bundle["meta"]["cells"]
    return cells * steps / dt, dt


TRIDIAG = "tridiag-16384"
# algorithmic bytes per unknown of a batched solve: read dl, d, du, b, write x
TRIDIAG_BYTES = {"f64": 40, "f32": 20}


def tridiag_workload(rank: int = 0):
    """16384 diagonally dominant systems, lengths log-uniform in [16, 4096]."""
    from hydist_c_b200 import scenario as S
    from hydist_c_b200.replicas import replica_seed
    return S.tridiag_batch(16384, seed=replica_seed(20262000, rank))


ENSEMBLE = "ensemble-64x1024x512"


def run_ensemble(args):
    """64 scenarios of 1024x512 (config 3: per-member bathymetry, Manning,
    inflow and tide; sediment from 300 s) stepped as one ensemble: one graph
    launch per step covering every member. The members are spun up to the
    sediment start untimed, then K steps are timed on the ensemble's stream."""
    import torch
    import hydist_c_b200 as H
    from hydist_c_b200 import scenario as S
    from hydist_c_b200.replicas import replica_seed
    rank, local, ws = R.init("nccl")
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    nmem = 64
    bundles = [S.config3_member(k, seed=replica_seed(20263000, rank)) for k in range(nmem)]
    cells = sum(b["meta"]["cells"] for b in bundles)
    prec = {"fp64": H.FP64, "fp32": H.FP32, "fp32-refine": H.FP32_REFINE}[args.precision]
    sims = [H.Simulation(b, device=dev.index, precision=prec) for b in bundles]
    ens = H.Ensemble(sims)
    spin = int(round(300.0 / 2.0))  # to t = 300 s, where the sediment sweeps start
    ens.step(spin)
    ens.step(max(args.warmup, 3))
    ens.sync()
    stream = torch.cuda.ExternalStream(ens.stream, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    l0 = sims[0].kernel_launches
    clocks = ClockSampler(torch.cuda.current_device())
    R.barrier(ws)
    torch.cuda.synchronize(dev)
    clocks.start()
    ev[0].record(stream)
    for k in range(args.steps):
        ens.step(1)
        ev[k + 1].record(stream)
    torch.cuda.synchronize(dev)
    R.barrier(ws)
    clk = clocks.stop()
    per = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    ms = sum(per)
    ms_max = R.max_over_ranks(ms, ws)
    launches = sims[0].kernel_launches - l0
    value = ws * cells * args.steps / (ms_max * 1e-3)
    hbm, peak_kind = _peaks()
    step_bytes = BYTES_PER_CELL_STEP[("fp64" if args.precision == "fp64" else "fp32", True)] * cells
    ach = step_bytes / (ms / args.steps * 1e-3) / 1e9
    mass = [m.mass() for m in sims[:4]]
    # the same steps with every member on its own launches (one graph of
    # the members' kernels on their streams), for comparison
    ens.batched(False)
    ens.step(max(args.warmup, 3))
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    ens.step(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    per_member_ms = ev0.elapsed_time(ev1) / args.steps
    ens.close()
    for m in sims:
        m.close()
    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        v_cpu, t_cpu = cpu_baseline(bundles[0], args.cpu_steps, threads)
        cpu = {"value": v_cpu, "unit": "cell-steps/s", "cores": threads, "kind": "port",
               "sample": f"{args.cpu_steps} full steps of one member (1024x512) with the sediment "
                         f"sweeps on ({t_cpu:.1f} s), FP64 CPU restatement, OpenMP over lines"}
    e2e = None
    if rank == 0 and not args.no_e2e:
        # the public API from pinned host buffers: create every member, the
        # timed steps with a mass read-back per member per step, downloads
        import time as _t
        pinned = []
        for b in bundles:
            sc = dict(b["scenario"])
            for k, v in list(sc.items()):
                if isinstance(v, np.ndarray) and v.dtype == np.float64:
                    sc[k] = torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy()
            pinned.append(dict(b, scenario=sc,
                               options=dict(b["options"], sediment_start=0.0, bed_change_start=0.0)))
        torch.cuda.synchronize(dev)
        t0 = _t.perf_counter()
        ms2 = [H.Simulation(b, device=dev.index, precision=prec) for b in pinned]
        en2 = H.Ensemble(ms2)
        for _ in range(args.steps):
            en2.step(1)
            for m in ms2:
                m.mass()
        outs = [m.download("z") for m in ms2]
        wall = _t.perf_counter() - t0
        en2.close()
        for m in ms2:
            m.close()
        n = (bundles[0]["scenario"]["N"] + 3) * (bundles[0]["scenario"]["M"] + 3)
        h2d = sum(a.nbytes for b in pinned for a in b["scenario"].values() if isinstance(a, np.ndarray))
        e2e = {"value": cells * args.steps / wall, "unit": "cell-steps/s",
               "h2d_bytes_per_step": h2d / args.steps,
               "d2h_bytes_per_step": (8 * nmem * args.steps + 8 * n * nmem) / args.steps,
               "wall_s": wall, "steps": args.steps}
    if rank == 0:
        line = {
            "metric": "ADI cell-steps/s", "value": value, "unit": "cell-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp64": "f64", "fp32": "f32 (f64 z, bed, mass)",
                                            "fp32-refine": "f32 + f64-residual refinement"}[args.precision],
            "data": "synthetic (seeded per member)",
            "config": {"workload": ENSEMBLE, "members": nmem, "N": 1024, "M": 512, "cells": cells,
                       "precision": args.precision,
                       "sediment": True,
                       "cuda_graph": "one graph launch per step; each kernel one launch over all "
                                     "members (batched)",
                       "l2": "inputs larger than L2", "parallelism": f"replicas x{ws}"},
            "p50_step_ms": float(np.percentile(per, 50)), "p99_step_ms": float(np.percentile(per, 99)),
            "member_mass": mass,
            "per_member_launches_ms_per_step": per_member_ms,
            "batched_speedup": per_member_ms / (ms / args.steps),
            "roofline": {"bound": "hbm", "kernel": "ensemble step (all members' kernels)",
                         "bytes_per_launch": step_bytes, "achieved": ach, "peak": hbm,
                         "unit": "GB/s", "frac": ach / hbm, "traffic": None,
                         "peak_source": peak_kind},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    R.finish(ws)


SERVING = "serving-poisson"


def run_serving(args):
    """Config 4: a Poisson stream of scenario solves at 20 requests/s, meshes
    drawn from {256x128, 512x256, 1024x512, 2048x1024}, horizons U(10, 60)
    simulated minutes, each request a channel scenario of its own seed.
    Requests are submitted to the server at their arrival times (wall clock)
    and admitted against a fixed HBM budget; latency is arrival -> retired.
    --steps sets the number of requests."""
    import torch
    import hydist_c_b200 as H
    from hydist_c_b200 import scenario as S
    rank, local, ws = R.init("nccl")
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    nreq = max(args.steps, 4)
    reqs = S.serving_requests(nreq, rate=20.0, seed=20264000 + 7919 * rank)
    dt = 2.0
    for r in reqs:  # inputs are built before the clock starts
        r["bundle"] = S.make_channel(N=r["N"], M=r["M"], seed=r["seed"], dx=10.0, dt=dt,
                                     hours=r["minutes"] / 60.0)
        r["nsteps"] = int(round(r["minutes"] * 60.0 / dt))
    budget = int(args.budget_gb * (1 << 30))
    srv = H.Server(budget, steps_per_round=args.round_steps, device=dev.index)
    pending = sorted(reqs, key=lambda r: r["arrival"])
    by_id, lat, work = {}, [], 0.0
    max_active = 0
    R.barrier(ws)
    t0 = time.perf_counter()
    while pending or by_id:
        now = time.perf_counter() - t0
        while pending and pending[0]["arrival"] <= now:
            r = pending.pop(0)
            by_id[srv.submit(r["bundle"], r["nsteps"])] = r
        q, a, _ = srv.counts()
        max_active = max(max_active, a)
        if a == 0 and q == 0:
            if pending:
                time.sleep(max(0.0, pending[0]["arrival"] - (time.perf_counter() - t0)))
            continue
        for rid in srv.round():
            r = by_id.pop(rid)
            done_t = time.perf_counter() - t0
            lat.append(done_t - r["arrival"])
            work += r["N"] * r["M"] * r["nsteps"]
            srv.release(rid)
    makespan = time.perf_counter() - t0
    srv.close()
    # the baseline: the plain FP64 form, one request at a time in arrival
    # order (each request created, stepped through its step graph, its
    # result read back, released, before the next starts; the device is
    # idle while no request has arrived), the same requests and inputs
    base_lat, vt = [], 0.0
    for r in sorted(reqs, key=lambda r: r["arrival"]):
        vt = max(vt, r["arrival"])
        t1 = time.perf_counter()
        sim = H.Simulation(r["bundle"], device=dev.index, precision=H.FP64)
        sim.step_graph(r["nsteps"])
        sim.download("z")
        sim.close()
        vt += time.perf_counter() - t1
        base_lat.append(vt - r["arrival"])
    R.barrier(ws)
    span = R.max_over_ranks(makespan, ws)
    value = R.sum_over_ranks(work, ws) / span
    if rank == 0:
        line = {
            "metric": "ADI cell-steps/s", "value": value, "unit": "cell-steps/s",
            "n_gpus": ws, "steps": nreq, "warmup": 0, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded per request)",
            "config": {"workload": SERVING, "requests": nreq, "rate_per_s": 20.0,
                       "meshes": [list(m) for m in S.SERVING_MESHES], "horizon_min": [10, 60],
                       "budget_gb": args.budget_gb, "steps_per_round": args.round_steps,
                       "max_active": max_active, "parallelism": f"replicas x{ws}"},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(np.max(lat))},
            "makespan_s": makespan, "cell_steps": work,
            "offered_cell_steps_per_s": work / (reqs[-1]["arrival"] + 1e-9),
            "one_at_a_time_fp64": {
                "makespan_s": vt, "value": work / vt,
                "latency_s": {"p50": float(np.percentile(base_lat, 50)),
                              "p99": float(np.percentile(base_lat, 99)),
                              "max": float(np.max(base_lat))},
                "note": "the same requests run one after another in arrival order, each "
                        "created, stepped and read back alone; idle time until an arrival "
                        "counted, not slept"},
            "speedup_vs_one_at_a_time": vt / makespan,
            "e2e": {"value": value, "unit": "cell-steps/s",
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "note": "wall clock from the first arrival, host inputs copied at submit"},
        }
        print(json.dumps(line), flush=True)
    R.finish(ws)


def run_tridiag_reference(args):
    """The reference's algorithm for a batch (serial Thomas per system) on the
    host cores: the oracle's batched Thomas with OpenMP over systems."""
    from oracle import oracle as O
    a, d, c, b, off, ln = tridiag_workload(0)
    threads = os.cpu_count() or 1
    n = int(ln.sum())
    O.thomas_batched(a, d, c, b, off, ln, nthreads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.thomas_batched(a, d, c, b, off, ln, nthreads=threads)
        times.append(time.perf_counter() - t0)
    v = n * args.steps / sum(times)
    line = {
        "metric": "tridiagonal unknowns/s", "value": v, "unit": "unknowns/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": TRIDIAG, "systems": len(ln), "unknowns": n},
        "cpu_baseline": {"value": v, "unit": "unknowns/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} solves of the whole batch, FP64 serial Thomas "
                                   "per system (the reference's tridiag()), OpenMP over systems"},
        "e2e": {"value": v, "unit": "unknowns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def rel_residual(a, d, c, b, off, ln, x):
    """max over rows of |b - A x| / (|a x_{-1}| + |d x| + |c x_{+1}| + |b|):
    the componentwise backward error of a packed batch's solution (dl of a
    system's first row and du of its last row ignored)."""
    n = len(d)
    first = np.zeros(n, bool)
    last = np.zeros(n, bool)
    nz = ln > 0
    first[off[nz]] = True
    last[off[nz] + ln[nz] - 1] = True
    xm = np.where(first, 0.0, np.roll(x, 1))
    xp = np.where(last, 0.0, np.roll(x, -1))
    am = np.where(first, 0.0, a)
    cp = np.where(last, 0.0, c)
    r = np.abs(b - am * xm - d * x - cp * xp)
    den = np.abs(am * xm) + np.abs(d * x) + np.abs(cp * xp) + np.abs(b)
    return float(np.max(r / np.maximum(den, 1e-300)))


def run_tridiag(args):
    """Batched solves of the tridiagonal microbenchmark through
    hydist_gtsv_batched (autotuned), inputs resident in HBM; e2e from pinned
    host buffers with the copies inside the timed region."""
    import torch
    import hydist_c_b200 as H
    from hydist_c_b200 import capi
    rank, local, ws = R.init("nccl")
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    lib = H.library()
    a, d, c, b, off, ln = tridiag_workload(rank)
    n = int(ln.sum())
    tdt = torch.float64 if args.dtype == "f64" else torch.float32
    dt_code = 0 if args.dtype == "f64" else 1
    host = [torch.from_numpy(v).to(tdt).pin_memory() for v in (a, d, c, b)]
    hoff = torch.from_numpy(off).pin_memory()
    hlen = torch.from_numpy(ln).pin_memory()
    t = [h.to(dev) for h in host]
    o_d, l_d = hoff.to(dev), hlen.to(dev)
    x = torch.empty_like(t[1])
    stream = torch.cuda.current_stream(dev)
    table = (C.c_int32 * capi.GTSV_BANDS)()
    if args.gtsv_algo:
        # one solver for every band (the library hands a band it cannot take
        # to a more general one)
        for k in range(capi.GTSV_BANDS):
            table[k] = args.gtsv_algo
    else:
        capi.check(lib, lib.hydist_gtsv_autotune(dt_code, C.c_void_p(stream.cuda_stream), table),
                   "hydist_gtsv_autotune")

    def solve(xo, tt, oo, ll):
        st = lib.hydist_gtsv_batched(tt[0].data_ptr(), tt[1].data_ptr(), tt[2].data_ptr(),
                                     tt[3].data_ptr(), xo.data_ptr(), oo.data_ptr(), ll.data_ptr(),
                                     len(ln), dt_code, args.gtsv_algo or capi.GTSV_AUTO,
                                     C.c_void_p(stream.cuda_stream))
        capi.check(lib, st, "hydist_gtsv_batched")

    for _ in range(max(args.warmup, 3)):
        solve(x, t, o_d, l_d)
    torch.cuda.synchronize(dev)
    # inputs (484 MB FP64) exceed the 126 MB L2: no flush between solves
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    clocks = ClockSampler(torch.cuda.current_device())
    R.barrier(ws)
    torch.cuda.synchronize(dev)
    clocks.start()
    ev[0].record(stream)
    for k in range(args.steps):
        solve(x, t, o_d, l_d)
        ev[k + 1].record(stream)
    torch.cuda.synchronize(dev)
    R.barrier(ws)
    clk = clocks.stop()
    per = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    ms = sum(per)
    ms_max = R.max_over_ranks(ms, ws)
    value = ws * n * args.steps / (ms_max * 1e-3)
    bands = (C.c_int32 * capi.GTSV_BANDS)()
    lib.hydist_gtsv_band_bounds(bands)
    nonempty = 0
    lo = 0
    for hi in list(bands):
        nonempty += int(((ln > lo) & (ln <= hi)).sum() > 0)
        lo = hi
    # accuracy against the FP64 oracle, and e2e through host buffers
    from oracle import oracle as O
    ref = O.thomas_batched(a, d, c, b, off, ln, nthreads=os.cpu_count() or 1) if rank == 0 else None
    xs = x.double().cpu().numpy()
    e2e = None
    if rank == 0 and not args.no_e2e:
        xh = torch.empty(n, dtype=tdt).pin_memory()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            td = [h.to(dev, non_blocking=True) for h in host]
            od, ld = hoff.to(dev, non_blocking=True), hlen.to(dev, non_blocking=True)
            xd = torch.empty_like(td[1])
            solve(xd, td, od, ld)
            xh.copy_(xd, non_blocking=True)
            torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
        esz = 8 if args.dtype == "f64" else 4
        e2e = {"value": n * args.steps / wall, "unit": "unknowns/s",
               "h2d_bytes_per_step": 4 * n * esz + 8 * len(ln), "d2h_bytes_per_step": n * esz,
               "wall_s": wall, "steps": args.steps}
    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        O.thomas_batched(a, d, c, b, off, ln, nthreads=threads)
        tc = time.perf_counter() - t0
        cpu = {"value": n / tc, "unit": "unknowns/s", "cores": threads, "kind": "port",
               "sample": f"one solve of the whole batch ({tc:.2f} s), FP64 serial Thomas per "
                         "system, OpenMP over systems"}
    refined = None
    if rank == 0 and args.dtype == "f64":
        # the same FP64 systems solved in FP32 with one FP64-residual
        # refinement (hydist_gtsv_batched_refine), timed the same way
        xr = torch.empty_like(t[1])

        def solve_ref():
            st = lib.hydist_gtsv_batched_refine(
                t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), t[3].data_ptr(),
                xr.data_ptr(), o_d.data_ptr(), l_d.data_ptr(), len(ln),
                args.gtsv_algo or capi.GTSV_AUTO, C.c_void_p(stream.cuda_stream))
            capi.check(lib, st, "hydist_gtsv_batched_refine")

        for _ in range(3):
            solve_ref()
        torch.cuda.synchronize(dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            solve_ref()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        rms = ev0.elapsed_time(ev1) / args.steps
        xrs = xr.cpu().numpy()
        refined = {"ms_per_step": rms, "value": n / (rms * 1e-3),
                   "max_rel_err_vs_fp64_oracle":
                       float(np.max(np.abs(xrs - ref) / np.maximum(np.abs(ref), 1.0))),
                   "max_rel_residual": rel_residual(a, d, c, b, off, ln, xrs)}
    if rank == 0:
        hbm, peak_kind = _peaks()
        alg = TRIDIAG_BYTES[args.dtype] * n
        ach = alg / (ms / args.steps * 1e-3) / 1e9
        err = float(np.max(np.abs(xs - ref) / np.maximum(np.abs(ref), 1.0)))
        line = {
            "metric": "tridiagonal unknowns/s", "value": value, "unit": "unknowns/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.dtype, "data": "synthetic (seeded)",
            "config": {"workload": TRIDIAG, "systems": len(ln), "unknowns": n,
                       "lengths": "log-uniform [16, 4096]", "algo": args.gtsv_algo or "auto",
                       "autotuned": dict(zip([str(v) for v in bands], list(table))),
                       "l2": "inputs larger than L2", "parallelism": f"replicas x{ws}"},
            "p50_step_ms": float(np.percentile(per, 50)), "p99_step_ms": float(np.percentile(per, 99)),
            "max_rel_err_vs_fp64_oracle": err,
            "max_rel_residual": rel_residual(a, d, c, b, off, ln, xs),
            "roofline": {"bound": "hbm", "kernel": "batched solve (classify + per-band solvers)",
                         "bytes_per_launch": alg, "achieved": ach, "peak": hbm, "unit": "GB/s",
                         "frac": ach / hbm, "traffic": None, "peak_source": peak_kind},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps * (1 + nonempty),
            "clocks": clk,
        }
        if refined is not None:
            line["fp32_refined"] = refined
        print(json.dumps(line), flush=True)
    R.finish(ws)


def run_reference(args):
    # rank 0 alone times the CPU implementation; no process group is needed
    rank, local, ws = R.env_ranks()
    if rank != 0:
        return
    if args.workload == TRIDIAG:
        return run_tridiag_reference(args)
    bundle, _ = workload(args.workload)
    threads = os.cpu_count() or 1
    cells = bundle["meta"]["cells"]
    from oracle import oracle as O
    b = dict(bundle)
    b["options"] = dict(bundle["options"], sediment_start=0.0, bed_change_start=0.0)
    o = O.OracleSim(b, nthreads=threads)
    o.step(max(args.warmup, 1))
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.step(1)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    v = cells * args.steps / total
    line = {
        "metric": "ADI cell-steps/s", "value": v, "unit": "cell-steps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "cells": cells},
        "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full steps of the {args.workload} workload, "
                                   "sediment sweeps on, FP64 CPU restatement of the reference "
                                   "time step (the reference has no CPU path), OpenMP over lines"},
        "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import hydist_c_b200 as H
    rank, local, ws = R.init("nccl")
    dev = local
    torch.cuda.set_device(dev)
    prec = {"fp64": H.FP64, "fp32": H.FP32, "fp32-refine": H.FP32_REFINE}[args.precision]
    bundle, spin = workload(args.workload, rank)
    if args.sed0 and bundle["options"]["sediment_start"] < 1e11:
        # sediment sweeps from the first step: the same per-step work without
        # the spin-up (used for short profiling runs)
        bundle["options"] = dict(bundle["options"], sediment_start=0.0, bed_change_start=0.0)
        spin = 0
    cells = bundle["meta"]["cells"]
    N, M = bundle["meta"]["N"], bundle["meta"]["M"]
    sim = H.Simulation(bundle, device=dev, precision=prec)
    sed = bundle["options"]["sediment_start"] < 1e11
    # spin-up to the sediment phase (untimed), then warm-up steps
    if spin:
        sim.step(spin)
    # warm-up in the timed mode (a graph is captured on its first step)
    (sim.step_graph if args.graph else sim.step)(max(args.warmup, 3))
    sim.sync()
    l0 = sim.kernel_launches
    stream = torch.cuda.ExternalStream(sim.stream, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    step_ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    clocks = ClockSampler(torch.cuda.current_device() if ws == 1 else local)
    R.barrier(ws)
    torch.cuda.synchronize(dev)
    clocks.start()
    e0.record(stream)
    step_ev[0].record(stream)
    for k in range(args.steps):
        if args.graph:
            sim.step_graph(1)
        else:
            sim.step(1)
        step_ev[k + 1].record(stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    R.barrier(ws)
    clk = clocks.stop()
    sim.sync()
    ms = e0.elapsed_time(e1)
    launches = sim.kernel_launches - l0
    per_step = [step_ev[k].elapsed_time(step_ev[k + 1]) for k in range(args.steps)]
    ms_max = R.max_over_ranks(ms, ws)
    value = ws * cells * args.steps / (ms_max * 1e-3)
    # per-kernel times: the same K steps again, each traced (an event at the
    # end of every phase and around every line-solver launch)
    ph_sum, sw_sum, sw_n = {}, {}, {}
    for _ in range(args.steps):
        ph, sw = sim.step_traced_sweeps()
        for k, v in ph.items():
            ph_sum[k] = ph_sum.get(k, 0.0) + v
        for k, v in sw.items():
            if v > 0:
                sw_sum[k] = sw_sum.get(k, 0.0) + v
                sw_n[k] = sw_n.get(k, 0) + 1
    phases = {k: v / args.steps for k, v in ph_sum.items()}
    sweeps = {k: sw_sum[k] / sw_n[k] for k in sw_sum}
    hbm, peak_kind = _peaks()
    # dominant kernel: the longest line-solver launch (the launch list shows
    # the four line solvers as the top kernels)
    dom = max(sweeps, key=sweeps.get)
    dom_cells = sweep_cells(dom, N, M)
    pkey = "fp64" if args.precision == "fp64" else "fp32"
    alg_bytes = SWEEP_BYTES_PER_CELL[pkey][dom] * dom_cells
    ach = alg_bytes / (sweeps[dom] * 1e-3) / 1e9
    step_bytes = BYTES_PER_CELL_STEP[(pkey, sed)] * cells
    step_ms = ms / args.steps
    roof = {"bound": "hbm", "kernel": dom, "kernel_ms": round(sweeps[dom], 4),
            "bytes_per_launch": alg_bytes, "achieved": ach, "peak": hbm, "unit": "GB/s",
            "frac": ach / hbm, "traffic": None, "peak_source": peak_kind,
            "sweeps_ms": {k: round(v, 4) for k, v in sweeps.items()},
            "step_achieved": step_bytes / (step_ms * 1e-3) / 1e9,
            "step_frac": step_bytes / (step_ms * 1e-3) / 1e9 / hbm}
    traffic_file = ROOT / "profiles" / "traffic.json"
    if traffic_file.exists():
        try:
            tj = json.loads(traffic_file.read_text())
            roof["traffic"] = tj.get(args.workload if args.precision == "fp64"
                                     else args.workload + "-" + args.precision, {}).get(dom)
        except Exception:
            pass
    acc = None
    if prec != H.FP64 and rank == 0:
        acc = accuracy_vs_fp64(H, sim, bundle, dev, spin + max(args.warmup, 3) + 2 * args.steps)
    forms = None
    if prec == H.FP64 and rank == 0 and not args.no_forms and sed:
        forms = measure_forms(H, sim, bundle, dev, args, ms_max / args.steps)
    # the handle is released before the end-to-end run (its device memory
    # goes back to the library's pool, as between two requests of a server)
    sim.close()
    e2e = measure_e2e(H, bundle, dev, prec, args) if rank == 0 and not args.no_e2e else None
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        csteps = args.cpu_steps
        v_cpu, t_cpu = cpu_baseline(bundle, csteps, threads)
        cpu = {"value": v_cpu, "unit": "cell-steps/s", "cores": threads, "kind": "port",
               "sample": f"{csteps} full steps of the {args.workload} workload with the "
                         f"sediment sweeps on ({t_cpu:.1f} s), FP64 CPU restatement, OpenMP "
                         "over lines"}
    if rank == 0:
        line = {
            "metric": "ADI cell-steps/s", "value": value, "unit": "cell-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp64": "f64", "fp32": "f32 (f64 z, bed, mass)",
                      "fp32-refine": "f32 + f64-residual refinement (f64 z, bed, mass)"}[args.precision],
            "data": "synthetic (seeded bathymetry, Manning, boundaries)",
            "config": {"workload": args.workload, "N": bundle["meta"]["N"],
                       "M": bundle["meta"]["M"], "cells": cells, "dx": 5.0, "dt": 2.0,
                       "sediment": sed, "precision": args.precision,
                       "cuda_graph": bool(args.graph),
                       "l2": "inputs larger than L2 (state of ~30 fields of 16.9 MB)",
                       "parallelism": f"replicas x{ws}"},
            "p50_step_ms": float(np.percentile(per_step, 50)),
            "p99_step_ms": float(np.percentile(per_step, 99)),
            "phases_ms": {k: round(v, 4) for k, v in phases.items()},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        if acc is not None:
            line["accuracy_vs_fp64"] = acc
        if forms is not None:
            line["forms"] = forms
        print(json.dumps(line), flush=True)
    R.finish(ws)


# the state that carries from one step to the next (uploaded to start the
# other forms and the oracle from the FP64 form's state)
CARRY_FIELDS = ["u", "v", "z", "t_u", "t_v", "t_z", "H_moi", "Htdu", "Htdv", "FS", "tFS", "dH"]


def measure_forms(H, sim, bundle, dev, args, fp64_ms, window=10):
    """The FP32 and FP32 + FP64-residual refinement forms on the benchmarked
    workload, started from the FP64 form's current state: each form's device
    time per step (graph replay, CUDA events over args.steps steps, after a
    window of `window` steps) and its ratio to the FP64 form's, and the
    errors of every form after the window against the FP64 CPU oracle run
    from the same state: max |dz| (m), relative L2 of u, v, the
    concentration and the bed change dH, wet/dry cells that differ, and
    the relative difference of the water volume."""
    import torch
    from oracle import oracle as O
    start = {f: sim.download(f) for f in CARRY_FIELDS + ["khouot"]}
    t0 = sim.t
    orc = O.OracleSim(bundle, nthreads=os.cpu_count() or 1)
    orc.load_state(start)
    orc.t = t0
    tw = time.perf_counter()
    orc.step(window)
    tw = time.perf_counter() - tw
    want = {f: orc.get(f) for f in ("z", "u", "v", "FS", "dH", "khouot")}
    k = want["khouot"]
    ht = orc.get("htaiz")
    N, M = bundle["meta"]["N"], bundle["meta"]["M"]
    sl = (slice(2, N + 1), slice(2, M + 1))
    p = H.capi.params_from_dict(bundle.get("params", {}))
    vol_ref = float(np.sum(np.where(k[sl] == 0, ht[sl] + want["z"][sl], 0.0))) * p.dX * p.dY
    orc.close()
    out = {"window_steps": window, "oracle_s": round(tw, 2),
           "start_t_s": t0, "oracle_threads": os.cpu_count() or 1}
    for name, prec in (("fp64", H.FP64), ("fp32", H.FP32), ("fp32-refine", H.FP32_REFINE)):
        f = H.Simulation(bundle, device=dev, precision=prec)
        for fld, a in start.items():
            f.upload(fld, a)
        f.t = t0
        f.step_graph(window)
        f.sync()
        got = {fld: f.download(fld) for fld in ("z", "u", "v", "FS", "dH", "khouot")}
        err = {"max_abs_dz_m": float(np.abs(got["z"] - want["z"]).max())}
        for fld in ("u", "v", "FS", "dH"):
            den = float(np.linalg.norm(want[fld]))
            err[f"rel_l2_{fld}"] = float(np.linalg.norm(got[fld] - want[fld]) / den) if den else 0.0
        err["mask_cells_differing"] = int((got["khouot"] != want["khouot"]).sum())
        err["rel_volume_diff"] = float(abs(f.mass() - vol_ref) / abs(vol_ref))
        entry = {"errors_vs_oracle": err}
        if name != "fp64":
            stream = torch.cuda.ExternalStream(f.stream, device=dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f.step_graph(3)
            torch.cuda.synchronize(dev)
            e0.record(stream)
            f.step_graph(args.steps)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1) / args.steps
            entry.update(ms_per_step=ms, value=bundle["meta"]["cells"] / (ms * 1e-3),
                         vs_fp64=fp64_ms / ms)
        else:
            entry["ms_per_step"] = fp64_ms
        out[name] = entry
        f.close()
    try:
        out["batched"] = measure_batched_forms(H, dev, args,
                                               bundle["meta"]["cells"] / (fp64_ms * 1e-3))
    except Exception as e:  # reported, not fatal to the benchmark line
        out["batched"] = {"error": str(e)[:300]}
    return out


def measure_batched_forms(H, dev, args, fp64_plain_value, nmem=64, steps=10):
    """The batched forms of the ensemble workload (64 scenarios of 1024x512,
    per-member bathymetry, Manning, inflow and tide; sediment sweeps and the
    bed change from t = 300 s), each form one graph launch per step over
    every member: the members spun up to t = 300 s untimed, then the device
    time per step (CUDA events over `steps` steps after 3 warm-up steps),
    cell-steps/s, and the ratio of each to the plain FP64 form of the
    benchmarked workload (fp64_plain_value, cell-steps/s). The errors of the
    FP32 forms against the oracle are those of the single-scenario forms
    above (the same kernels, batched)."""
    import torch
    from hydist_c_b200 import scenario as S
    out = {"workload": ENSEMBLE, "members": nmem, "steps": steps}
    for name, prec in (("fp64", H.FP64), ("fp32", H.FP32), ("fp32-refine", H.FP32_REFINE)):
        bundles = [S.config3_member(k, seed=20263000) for k in range(nmem)]
        cells = sum(b["meta"]["cells"] for b in bundles)
        sims = [H.Simulation(b, device=dev, precision=prec) for b in bundles]
        ens = H.Ensemble(sims)
        ens.step(150 + 3)  # to the sediment start, then warm-up
        ens.sync()
        stream = torch.cuda.ExternalStream(ens.stream, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        ens.step(steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ens.sync()
        ms = e0.elapsed_time(e1) / steps
        v = cells * steps / (e0.elapsed_time(e1) * 1e-3)
        out[name] = {"ms_per_step": ms, "value": v, "vs_fp64_plain": v / fp64_plain_value}
        ens.close()
        for m in sims:
            m.close()
    out["fp32-refine"]["vs_fp64_batched"] = out["fp32-refine"]["value"] / out["fp64"]["value"]
    out["fp32"]["vs_fp64_batched"] = out["fp32"]["value"] / out["fp64"]["value"]
    return out


def accuracy_vs_fp64(H, sim, bundle, dev, nsteps):
    """Errors of an FP32 form after nsteps steps against the FP64 form (whose
    steps match the FP64 CPU oracle to 1e-10 per step) run from the same
    start: max |dz| in metres, relative L2 of u, v and the concentration, and
    the relative difference of the water volume (mass)."""
    ref = H.Simulation(bundle, device=dev, precision=H.FP64)
    ref.step(nsteps)
    out = {"steps": nsteps}
    got = {f: sim.download(f) for f in ("z", "u", "v", "FS")}
    want = {f: ref.download(f) for f in ("z", "u", "v", "FS")}
    out["max_abs_dz_m"] = float(np.abs(got["z"] - want["z"]).max())
    for f in ("u", "v", "FS"):
        den = float(np.linalg.norm(want[f]))
        out[f"rel_l2_{f}"] = float(np.linalg.norm(got[f] - want[f]) / den) if den > 0 else 0.0
    m_ref = ref.mass()
    out["rel_volume_diff"] = float(abs(sim.mass() - m_ref) / abs(m_ref))
    ref.close()
    return out


def measure_e2e(H, bundle, dev, prec, args):
    """The same metric through the public API from host buffers: create the
    scenario from pinned host arrays (H2D of every input), run the timed
    steps with the sediment sweeps on from the first step (the same work per
    step as the device-timed region) and a device->host read of the water
    volume (mass) after each, then download u, v, z, FS."""
    import torch
    sc = bundle["scenario"]
    pinned = {}
    for k, v in sc.items():
        if isinstance(v, np.ndarray) and v.dtype == np.float64:
            t = torch.from_numpy(np.ascontiguousarray(v)).pin_memory()
            pinned[k] = t.numpy()
    b = dict(bundle)
    b["scenario"] = dict(sc, **pinned)
    sed = bundle["options"]["sediment_start"] < 1e11
    if sed:
        b["options"] = dict(bundle["options"], sediment_start=0.0, bed_change_start=0.0)
    h2d = sum(a.nbytes for a in pinned.values())
    n = (sc["N"] + 3) * (sc["M"] + 3)
    # pinned host buffers for the results, as for the inputs
    outs = {f: torch.empty((sc["N"] + 3, sc["M"] + 3), dtype=torch.float64).pin_memory().numpy()
            for f in ("u", "v", "z", "FS")}
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    sim = H.Simulation(b, device=dev, precision=prec)
    sim.sync()
    t1 = time.perf_counter()
    create = {k: round(v, 3) for k, v in sim.create_phases().items()}
    for _ in range(args.steps):
        (sim.step_graph if args.graph else sim.step)(1)
        sim.mass()
    t2 = time.perf_counter()
    for f, o in outs.items():
        sim.download(f, out=o)
    dt = time.perf_counter() - t0
    sim.close()
    steps = args.steps
    cells = bundle["meta"]["cells"]
    return {"value": cells * steps / dt, "unit": "cell-steps/s",
            "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": (8 * args.steps + 4 * 8 * n) / steps,
            "wall_s": dt, "create_s": t1 - t0, "create_phases_ms": create, "steps_s": t2 - t1,
            "download_s": dt - (t2 - t0), "steps": steps}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "fp32-refine"])
    ap.add_argument("--workload", default="sediment-2048x1024",
                    help="sediment-2048x1024 | sediment-1024x512 | channel-256x128 | " + TRIDIAG +
                         " | " + ENSEMBLE +
                         " | " + SERVING)
    ap.add_argument("--budget-gb", type=float, default=120.0,
                    help="HBM budget of the " + SERVING + " workload")
    ap.add_argument("--round-steps", type=int, default=100,
                    help="steps per request and scheduling round (" + SERVING + ")")
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"],
                    help="arithmetic of the " + TRIDIAG + " workload")
    ap.add_argument("--gtsv-algo", type=int, default=0,
                    help="solver of every band of the " + TRIDIAG + " workload (enum "
                         "HydistGtsvAlgo; 0: the autotuned one per band)")
    ap.add_argument("--eager", action="store_true",
                    help="launch each step's kernels one by one instead of replaying the "
                         "step's CUDA graph (hydist_step instead of hydist_step_graph)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the FP32 forms and their errors against the oracle")
    ap.add_argument("--cpu-steps", type=int, default=4)
    ap.add_argument("--sed0", action="store_true",
                    help="sediment sweeps from t=0 instead of a spin-up to t=600 s")
    args = ap.parse_args()
    args.graph = not args.eager
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == TRIDIAG:
        run_tridiag(args)
    elif args.workload == ENSEMBLE:
        run_ensemble(args)
    elif args.workload == SERVING:
        run_serving(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
