"""TEST INFRASTRUCTURE: times the reference's own GPU code beside this
library on the same inputs, on one B200.

    python -m oracle.time_reference_gpu [--steps 1800] [--reps 10]

Needs the reference-built binaries under oracle/_ref (oracle/build.py):

1. The plain hydraulic workload (256x128 channel, dx = dy = 10 m, dt = 2 s,
   one simulated hour = 1800 steps): the reference's Hydraulic_Calculation
   (engine.cpp:41-296, oracle/_ref/hydist_ref_driver; its SN scratch padded,
   nothing else changed) timed with CUDA events around the call, against this
   library's step (hydist_step_graph and hydist_step) on the same scenario,
   each on a fresh handle (its graph captured inside the timed call) after a
   warm-up handle has taken the process's one-time costs.
   The reference synchronises after every kernel and prints the time every
   half-step (its stdout goes to /dev/null here).
2. The batched tridiagonal workload (16384 systems, lengths log-uniform in
   [16, 4096], FP64): the reference's device tridiag()
   (UVZSolver_multithread.cpp:19-43, one thread per system,
   oracle/_ref/hydist_ref_tridiag) against hydist_gtsv_batched (autotuned).

Prints one JSON object; values are device milliseconds.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from oracle import build as OB  # noqa: E402


def time_reference_step(bundle, steps, workdir):
    """The reference's Hydraulic_Calculation over `steps` steps, ms."""
    from hydist_c_b200 import scenario as S
    d = Path(workdir) / "inputs"
    S.write_reference_inputs(bundle["scenario"], d)
    out = Path(workdir) / "out"
    out.mkdir(parents=True, exist_ok=True)
    cmd = [str(OB.REF_DRIVER), str(d) + "/", str(out), str(steps)]
    with open(os.devnull, "w") as f:
        r = subprocess.run(cmd, stdout=f, stderr=subprocess.PIPE, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference driver failed: " + r.stderr[-2000:])
    m = re.search(r"Hydraulic_Calculation steps \d+\.\.(\d+): ([0-9.]+) ms", r.stderr)
    if not m:
        raise RuntimeError("no timing in the driver's output: " + r.stderr[-2000:])
    return float(m.group(2))


def time_library_step(bundle, steps):
    import torch
    import hydist_c_b200 as H
    out = {}
    # one-time costs of the process (module load, kernel attributes) outside
    # the timed calls: a few steps of a separate handle first
    warm = H.Simulation(bundle)
    warm.step_graph(3)
    warm.step(3)
    warm.sync()
    warm.close()
    for name in ("graph", "eager"):
        sim = H.Simulation(bundle)
        stream = torch.cuda.ExternalStream(sim.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        (sim.step_graph if name == "graph" else sim.step)(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1)
        sim.close()
    return out


def time_reference_tridiag(batch, reps, workdir):
    a, d, c, b, off, ln = batch
    p = Path(workdir) / "tri_in.bin"
    q = Path(workdir) / "tri_out.bin"
    with open(p, "wb") as f:
        np.array([len(ln), int(ln.sum())], np.int32).tofile(f)
        off.astype(np.int32).tofile(f)
        ln.astype(np.int32).tofile(f)
        for v in (a, d, c, b):
            np.ascontiguousarray(v, dtype="<f8").tofile(f)
    r = subprocess.run([str(OB.REF_TRIDIAG), str(p), str(q), str(reps)], capture_output=True,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError("reference tridiag failed: " + r.stderr[-2000:])
    raw = np.fromfile(q, dtype="<f8")
    return float(raw[-1]), raw[:-1]


def time_library_tridiag(batch, reps):
    import torch
    import hydist_c_b200 as H
    a, d, c, b, off, ln = batch
    t = [torch.from_numpy(v).cuda() for v in (a, d, c, b)]
    o, n = torch.from_numpy(off).cuda(), torch.from_numpy(ln).cuda()
    x = H.gtsv_batched(*t, o, n)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        H.gtsv_batched(*t, o, n, x=x)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps, x.cpu().numpy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1800)
    ap.add_argument("--reps", type=int, default=10)
    args = ap.parse_args()
    from hydist_c_b200 import scenario as S
    from oracle import oracle as O
    res = {}
    with tempfile.TemporaryDirectory() as wd:
        b = S.config0()
        cells = b["meta"]["cells"]
        ref_ms = time_reference_step(b, args.steps, wd)
        ours = time_library_step(b, args.steps)
        res["channel-256x128"] = {
            "steps": args.steps, "cells": cells,
            "reference_ms": ref_ms,
            "reference_cell_steps_per_s": cells * args.steps / (ref_ms * 1e-3),
            "ours_graph_ms": ours["graph"], "ours_eager_ms": ours["eager"],
            "ours_cell_steps_per_s": cells * args.steps / (ours["graph"] * 1e-3),
            "speedup_graph": ref_ms / ours["graph"], "speedup_eager": ref_ms / ours["eager"]}
        batch = S.tridiag_batch(16384)
        n = int(batch[5].sum())
        rms, rx = time_reference_tridiag(batch, args.reps, wd)
        oms, ox = time_library_tridiag(batch, args.reps)
        ref = O.thomas_batched(*batch, nthreads=os.cpu_count() or 1)
        scale = np.maximum(np.abs(ref), 1.0)
        res["tridiag-16384"] = {
            "unknowns": n, "reference_ms": rms, "ours_ms": oms, "speedup": rms / oms,
            "reference_unknowns_per_s": n / (rms * 1e-3), "ours_unknowns_per_s": n / (oms * 1e-3),
            "reference_max_rel_err_vs_oracle": float(np.max(np.abs(rx - ref) / scale)),
            "ours_max_rel_err_vs_oracle": float(np.max(np.abs(ox - ref) / scale))}
    print(json.dumps(res))


if __name__ == "__main__":
    main()
