"""GPU parity on the benchmarked workload: 2048x1024 cells, dx = dy = 5 m,
dt = 2 s, the concentration sweeps and the bed change on from t = 600 s
(scenario.config1 with the bed change accumulated).

The GPU advances the scenario to t = 604 s (past the sediment start, so that
every step runs both concentration sweeps and the bed change); its state is
loaded into the FP64 CPU oracle, and from that identical state

* one step on each side agrees to 1e-10 relative per field (u, v, z, the
  provisional fields, the total depths, the concentration, its sweep
  buffer, the speed and diffusivities, the bed-load flux and dH) with an
  identical wet/dry mask;
* a 30-step window agrees to 1e-8 (u, v, z, FS, dH);
* the FP32 and FP32 + FP64-residual refinement forms, started from the same
  state, stay within the stated error bars of the oracle after the same 30
  steps: max |dz| <= 1e-4 m, relative L2 of u, v, FS and dH <= 1e-3, and an
  identical mask.

The oracle runs 31 steps of 2.1 M cells with one OpenMP thread per host
core (about 0.4 s a step on 16 cores).
"""
import os

import numpy as np
import pytest

from hydist_c_b200 import scenario as S

pytestmark = pytest.mark.gpu

# the fields that carry from one step to the next (VTH, Kx, Ky, the
# boundary arrays and the segment tables are rebuilt inside a step)
CARRY = ["u", "v", "z", "t_u", "t_v", "t_z", "H_moi", "Htdu", "Htdv", "FS", "tFS", "dH"]
STEP_FIELDS = ["u", "v", "z", "t_u", "t_v", "t_z", "H_moi", "Htdu", "Htdv", "FS", "tFS", "VTH",
               "Kx", "Ky", "Qbx", "Qby", "dH"]
WINDOW = 30
SPINUP = 302  # t = 604 s


def _bundle():
    b = S.config1()
    assert b["options"]["bed_change"] == 1
    return b


def _max_rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def run(hyd, oracle_mod):
    """The start state from the GPU, the oracle one step and WINDOW + 1
    steps on from it, and the FP64 GPU form over the same steps."""
    b = _bundle()
    sim = hyd.Simulation(b)
    sim.step(SPINUP)
    sim.sync()
    start = {f: sim.download(f) for f in CARRY + ["khouot"]}
    t0 = sim.t
    assert t0 == pytest.approx(604.0)
    orc = oracle_mod.OracleSim(b, nthreads=os.cpu_count() or 1)
    orc.load_state(start)
    orc.t = t0
    sim.step(1)
    orc.step(1)
    sim.sync()
    one = {"gpu": {f: sim.download(f) for f in STEP_FIELDS + ["khouot"]},
           "orc": {f: orc.get(f) for f in STEP_FIELDS + ["khouot"]}}
    sim.step(WINDOW)
    orc.step(WINDOW)
    sim.sync()
    win_fields = ["u", "v", "z", "FS", "dH", "khouot"]
    window = {"gpu": {f: sim.download(f) for f in win_fields},
              "orc": {f: orc.get(f) for f in win_fields}}
    sim.close()
    orc.close()
    return dict(bundle=b, start=start, t0=t0, one=one, window=window)


def test_config1_one_step_matches_oracle(run):
    g, o = run["one"]["gpu"], run["one"]["orc"]
    assert np.array_equal(g["khouot"], o["khouot"])
    # the step exercised what it is meant to: concentration and bed change
    assert np.abs(o["dH"]).max() > 0 and np.abs(o["Qbx"]).max() > 0
    assert np.abs(o["FS"] - run["start"]["FS"]).max() > 0
    bad = {f: _max_rel(g[f], o[f]) for f in STEP_FIELDS}
    bad = {f: r for f, r in bad.items() if not r <= 1e-10}
    assert not bad, bad


def test_config1_window_matches_oracle(run):
    g, o = run["window"]["gpu"], run["window"]["orc"]
    assert np.array_equal(g["khouot"], o["khouot"])
    bad = {f: _max_rel(g[f], o[f]) for f in ("u", "v", "z", "FS", "dH")}
    bad = {f: r for f, r in bad.items() if not r <= 1e-8}
    assert not bad, bad


@pytest.mark.parametrize("precision", ["FP32", "FP32_REFINE"])
def test_config1_fp32_forms_against_oracle(hyd, run, precision):
    """The FP32 forms from the same start state (fields rounded to FP32 where
    the form keeps them in FP32) against the oracle after WINDOW + 1 steps."""
    sim = hyd.Simulation(run["bundle"], precision=getattr(hyd, precision))
    for f, a in run["start"].items():
        sim.upload(f, a)
    sim.t = run["t0"]
    sim.step(WINDOW + 1)
    sim.sync()
    o = run["window"]["orc"]
    err = {"dz_max_m": float(np.abs(sim.download("z") - o["z"]).max())}
    for f in ("u", "v", "FS", "dH"):
        err[f] = _rel_l2(sim.download(f), o[f])
    mask_diff = int((sim.download("khouot") != o["khouot"]).sum())
    sim.close()
    assert mask_diff == 0, (mask_diff, err)
    assert err["dz_max_m"] <= 1e-4, err
    assert all(err[f] <= 1e-3 for f in ("u", "v", "FS", "dH")), err
