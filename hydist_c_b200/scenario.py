"""Seeded synthetic scenarios in the reference's input format.

A scenario is a dict of numpy arrays with the meaning of the reference's text
inputs after ``Inputs/standardize_inp.py`` (loader.cpp:120-168): node depth
``h`` (bandodosau), Manning ``hsnham``, eddy viscosity ``visco``
(hsnhotroiA), ``Fw`` (Fw_map), hourly boundary series per side and the
80-entry ``boundary_type`` (4 sides x 20 segments, side-major).

The named workloads (sizes are N x M = x-cells x y-cells):

* ``channel``  -- the plain hydraulic case: bed depth rising linearly from
  2 m to 10 m along x plus 8 Gaussian bumps (amplitude U(-1.5,1.5) m, sigma
  U(5,20) cells), Manning n ~ U(0.020,0.035), eddy viscosity 1.0 m^2/s,
  discharge inflow on the left side (i = 2), tidal water level
  0.5*sin(2*pi*t/44712 s) on the right side (i = N), solid up/down sides.
  Solid sides are dry bank columns (node depth 0 = NANGDAY for node columns
  0..2 and M-1..M+2), so the wet channel spans cell columns 3..M-1.
* ``sediment`` -- the same physics with the suspended-sediment sweeps on.

Boundary series are sampled hourly, as the reference reads them, and
linearly interpolated in time by the solver (support_funcs.cpp:606-624).
"""
from __future__ import annotations

import math
import os
from pathlib import Path

import numpy as np

SEG = 20
TIDE_PERIOD = 44712.0


def _bumps(rng, N, M, n=8):
    out = []
    for _ in range(n):
        amp = rng.uniform(-1.5, 1.5)
        sig = rng.uniform(5.0, 20.0)
        ci = rng.uniform(2, N)
        cj = rng.uniform(3, M - 1)
        out.append((amp, sig, ci, cj))
    return out


def make_channel(N=256, M=128, seed=20260000, dx=10.0, dt=2.0, hours=1.0,
                 inflow=500.0, tide_amp=0.5, manning=(0.020, 0.035), visco=1.0,
                 fw=(0.5, 1.5), sediment=False, sediment_start=600.0,
                 fs0_kgm3=0.05, fs_in_kgm3=0.1, toe=0.2, tod=0.1, mbochat=1e-4,
                 wss=5e-4, n_bumps=8):
    """Build one channel scenario. Returns dict(scenario=..., params=...,
    options=..., meta=...)."""
    if N < 8 or M < 8:
        raise ValueError("mesh too small")
    rng = np.random.default_rng(seed)
    H, W = N + 3, M + 3
    ii = np.arange(H, dtype=np.float64)[:, None]
    jj = np.arange(W, dtype=np.float64)[None, :]
    depth = 2.0 + 8.0 * (np.clip(ii, 2, N) - 2.0) / (N - 2.0) + 0.0 * jj
    for amp, sig, ci, cj in _bumps(rng, N, M, n_bumps):
        depth = depth + amp * np.exp(-((ii - ci) ** 2 + (jj - cj) ** 2) / (2.0 * sig * sig))
    depth = np.maximum(depth, 0.1)
    bank = np.zeros((1, W), dtype=bool)
    bank[0, :3] = True
    bank[0, M - 1:] = True
    h = np.where(bank, 0.0, depth)
    hsnham = rng.uniform(manning[0], manning[1], size=(H, W))
    vis = np.full((H, W), float(visco))
    Fw = rng.uniform(fw[0], fw[1], size=(H, W))
    T = max(3, int(math.ceil(hours)) + 3)
    hrs = np.arange(T, dtype=np.float64)
    bc_left = np.full(T, float(inflow))
    bc_right = tide_amp * np.sin(2.0 * math.pi * hrs * 3600.0 / TIDE_PERIOD)
    zeros = np.zeros(T)
    CC_left = np.full(T, float(fs_in_kgm3))
    btype = np.zeros(4 * SEG, dtype=np.int32)
    btype[2] = 2            # flat entry 2 -> bienQ[2] (left is discharge), loader.cpp:157-164
    btype[2 * SEG] = 2      # left side, segment 0: discharge
    btype[3 * SEG] = 1      # right side, segment 0: water level
    bienQ = [int(btype[k] == 2) for k in range(4)]
    sc = dict(M=M, N=N, total_time=T, h=h, hsnham=hsnham, visco=vis, Fw=Fw,
              bc_up=zeros.copy(), bc_down=zeros.copy(), bc_left=bc_left, bc_right=bc_right,
              CC_up=zeros.copy(), CC_down=zeros.copy(), CC_left=CC_left, CC_right=zeros.copy(),
              boundary_type=btype, bienQ=bienQ, FS0=None)
    params = dict(dX=dx, dY=dx, dT=dt)
    options = dict(t_start=0.0, sediment_start=1e12, bed_change_start=1e12, ketdinh=1)
    if sediment:
        fs0 = fs0_kgm3 / 2000.0
        sc["FS0"] = np.full((H, W), fs0)
        params.update(Toe=toe, Tod=tod, Mbochat=mbochat, wss=wss)
        options.update(sediment_start=float(sediment_start),
                       bed_change_start=float(sediment_start))
    nsteps = int(round(hours * 3600.0 / dt))
    meta = dict(name="sediment" if sediment else "channel", N=N, M=M, seed=seed,
                steps=nsteps, cells=N * M)
    return dict(scenario=sc, params=params, options=options, meta=meta)


# The benchmark plan's configurations.
def config0(seed=20260000):
    """Plain FP64 hydraulics, 256x128, dx=dy=10 m, dt=2 s, 1 h (1800 steps)."""
    return make_channel(N=256, M=128, seed=seed, dx=10.0, dt=2.0, hours=1.0)


def config1(seed=20260001):
    """Hydraulics + sediment, 2048x1024, dx=dy=5 m, dt=2 s, sediment from
    600 s, 1 h, with the bed change (Calculate_Qb + BedLoad,
    sediment_transport.cpp:352-537) accumulated once per step from then on.
    Fw ~ U(0.5,1.5) is used as the reference's tau_b = ro*Fw*V^2
    coefficient (sediment_transport.cpp:17) literally."""
    b = make_channel(N=2048, M=1024, seed=seed, dx=5.0, dt=2.0, hours=1.0,
                     sediment=True, sediment_start=600.0)
    b["options"]["bed_change"] = 1
    return b


def config3_member(k, seed=20263000):
    """One of the 64 ensemble scenarios of 1024x512, 30 min, sediment (and
    the bed change) from 300 s; per-member bumps, Manning U(0.018,0.040),
    inflow U(200,1200), tidal amplitude U(0.2,1.0)."""
    rng = np.random.default_rng(seed + 7919 * k)
    b = make_channel(N=1024, M=512, seed=seed + k, dx=5.0, dt=2.0, hours=0.5,
                     inflow=rng.uniform(200, 1200), tide_amp=rng.uniform(0.2, 1.0),
                     manning=(0.018, 0.040), sediment=True, sediment_start=300.0)
    b["options"]["bed_change"] = 1
    return b


SERVING_MESHES = ((256, 128), (512, 256), (1024, 512), (2048, 1024))


def tridiag_batch(nsys=16384, seed=20262000, lo=16, hi=4096, lengths=None):
    """The batched tridiagonal microbenchmark: nsys diagonally dominant
    systems with lengths log-uniform in [lo, hi] (uneven wet segments), packed
    one after another. a, c ~ U(-1, 1); b = |a| + |c| + U(0.1, 1.0); rhs
    ~ N(0, 1). Returns dl, d, du, rhs (FP64), offsets, lengths (int32)."""
    rng = np.random.default_rng(seed)
    if lengths is None:
        lengths = np.exp(rng.uniform(np.log(lo), np.log(hi), nsys)).astype(np.int32)
    lengths = np.asarray(lengths, dtype=np.int32)
    offsets = np.zeros(len(lengths), np.int32)
    offsets[1:] = np.cumsum(lengths[:-1])
    rows = int(lengths.sum())
    a = rng.uniform(-1, 1, rows)
    c = rng.uniform(-1, 1, rows)
    d = np.abs(a) + np.abs(c) + rng.uniform(0.1, 1.0, rows)
    b = rng.standard_normal(rows)
    return a, d, c, b, offsets, lengths


def serving_requests(n, rate=20.0, seed=20264000):
    """Poisson request stream: arrival times, mesh drawn uniformly from
    SERVING_MESHES, horizon U(10,60) simulated minutes."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n)
    arrivals = np.cumsum(gaps) - gaps[0]
    reqs = []
    for k in range(n):
        N, M = SERVING_MESHES[rng.integers(0, len(SERVING_MESHES))]
        minutes = rng.uniform(10.0, 60.0)
        reqs.append(dict(id=k, arrival=float(arrivals[k]), N=int(N), M=int(M),
                         minutes=float(minutes), seed=int(seed + 1 + k)))
    return reqs


# ---------------------------------------------------------------- text I/O
def _write_matrix(path, a, fmt="%.17g"):
    a = np.atleast_2d(a)
    with open(path, "w") as f:
        for row in a:
            f.write(" ".join(fmt % x for x in row))
            f.write("\n")


def write_reference_inputs(sc: dict, directory):
    """Write a scenario as the reference's Inputs/ directory.

    main.cpp:138 passes its bc_down/bc_right vectors to load_inputs in the
    order of loader.cpp:126-128's (bc_right, ..., bc_down) parameters, so the
    down side reads bienphai.txt and the right side reads bienduoi.txt, and
    total_time is the row count of bienduoi.txt (loader.cpp:165). The files
    are written to match.
    """
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    _write_matrix(d / "bandodosau.txt", sc["h"])
    _write_matrix(d / "hsnham.txt", sc["hsnham"])
    _write_matrix(d / "hsnhotroiA.txt", sc["visco"])
    _write_matrix(d / "Fw_map.txt", sc["Fw"])
    col = lambda a: np.asarray(a, dtype=np.float64).reshape(-1, 1)
    _write_matrix(d / "bientren.txt", col(sc["bc_up"]))
    _write_matrix(d / "bienphai.txt", col(sc["bc_down"]))
    _write_matrix(d / "bientrai.txt", col(sc["bc_left"]))
    _write_matrix(d / "bienduoi.txt", col(sc["bc_right"]))
    _write_matrix(d / "FS_bientren.txt", col(sc["CC_up"]))
    _write_matrix(d / "FS_bienduoi.txt", col(sc["CC_down"]))
    _write_matrix(d / "FS_bientrai.txt", col(sc["CC_left"]))
    _write_matrix(d / "FS_bienphai.txt", col(sc["CC_right"]))
    with open(d / "boundary_type.txt", "w") as f:
        for v in np.asarray(sc["boundary_type"]).ravel():
            f.write(f"{int(v)}\n")


def save_npz(path, bundle):
    sc = bundle["scenario"]
    arrs = {k: np.asarray(v) for k, v in sc.items() if isinstance(v, np.ndarray)}
    np.savez_compressed(path, **arrs, M=sc["M"], N=sc["N"], total_time=sc["total_time"],
                        bienQ=np.asarray(sc["bienQ"], dtype=np.int32))
