"""GPU parity of the step's optional modes against the FP64 CPU oracle:

* wind stress and Coriolis force (Constant_Coeffs Windx / Windy /
  CORIOLIS_FORCE, loader.cpp:75,81-82, zero in the shipped coefficients);
* the narrow-channel modes -kd / -kn (engine.cpp:24-30, 77-80, 190-193: no
  boundary update, the sweeps' index ranges), from a sloshing initial level;
* the narrow-channel standing wave of boundary_up/down/left/right
  (support_funcs.cpp:366-478), whose calls the reference keeps commented out;
* wetting and drying along rows as well (Reset_states_horizontal,
  support_funcs.cpp:88-138), in the first half-step.

The oracle side of the first two is pinned to the reference's own run
(tests/test_oracle.py, cases windcor, narrow_d, narrow_n). Tolerances as in
tests/test_gpu_parity.py: 1e-10 relative after the first step, 1e-8 after
tens of steps.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
FIELDS_STEP = ["u", "v", "z", "t_u", "t_v", "t_z", "H_moi", "Htdu", "Htdv"]
STATE = ["u", "v", "z", "t_u", "t_v", "t_z", "H_moi", "Htdu", "Htdv", "FS", "tFS"]


def _fixtures():
    sys.path.insert(0, str(GOLDEN))
    import make_reference_fixtures as F
    return F


def _max_rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _compare(sim, orc, fields, tol):
    bad = {}
    for f in fields:
        r = _max_rel(sim.download(f), orc.get(f))
        if not r <= tol:
            bad[f] = r
    ka, kb = sim.download("khouot"), orc.get("khouot")
    if not np.array_equal(ka, kb):
        bad["khouot"] = int((ka != kb).sum())
    return bad


def _run_pair(hyd, oracle_mod, b, first=1, more=30, tol_more=1e-8):
    sim = hyd.Simulation(b)
    orc = oracle_mod.OracleSim(b, nthreads=4)
    sim.step(first)
    orc.step(first)
    sim.sync()
    bad = _compare(sim, orc, FIELDS_STEP, 1e-10)
    assert not bad, bad
    sim.step(more)
    orc.step(more)
    sim.sync()
    bad = _compare(sim, orc, ["u", "v", "z"], tol_more)
    assert not bad, bad
    return sim, orc


def test_wind_and_coriolis(hyd, oracle_mod):
    F = _fixtures()
    b = F.bundle("windcor")
    sim, orc = _run_pair(hyd, oracle_mod, b)
    # the forcing moved the flow: the same scenario without it differs
    calm = dict(b, params={k: v for k, v in b["params"].items()
                           if k not in ("Wind", "huonggio", "CORIOLIS_FORCE")})
    c = hyd.Simulation(calm)
    c.step(31)
    c.sync()
    assert _max_rel(c.download("v"), sim.download("v")) > 1e-6


@pytest.mark.parametrize("kind", ["d", "n"])
def test_narrow_channel(hyd, oracle_mod, kind):
    F = _fixtures()
    b = F.narrow_bundle(kind)
    sim, orc = _run_pair(hyd, oracle_mod, b, first=1, more=50)
    # no boundary series is applied; the initial level sloshes
    assert np.abs(orc.get("u")).max() > 1e-4


def test_narrow_channel_standing_wave(hyd, oracle_mod):
    F = _fixtures()
    b = F.narrow_bundle("d")
    b["scenario"]["z0"] = None
    b["options"] = dict(b["options"], channel_wave=1)
    sim, orc = _run_pair(hyd, oracle_mod, b, first=2, more=40)
    assert np.abs(orc.get("z")).max() > 1e-3


def _front_mask(k, radius=3):
    dry = k != 0
    out = dry.copy()
    for di in range(-radius, radius + 1):
        for dj in range(-radius, radius + 1):
            out |= np.roll(np.roll(dry, di, 0), dj, 1)
    return out


def test_reset_states_horizontal(hyd, oracle_mod):
    """The wetting/drying basin with Reset_states_horizontal on: per-step
    parity from the oracle's own state while cells dry and re-wet along rows
    and columns (the mask exactly; fields as in test_wetting_and_drying)."""
    F = _fixtures()
    b = F.wetdry_bundle()
    b["options"] = dict(b["options"], reset_horizontal=1)
    orc = oracle_mod.OracleSim(b)
    sim = hyd.Simulation(b)
    done = 0
    seen_dry = seen_rewet = False
    # windows that see rows and columns dry (from step 288) and re-wet (from
    # step 637); this basin with the horizontal reset stays finite in the
    # oracle to about step 1560 and diverges after it, so targets stay below
    for target in (285, 634, 735, 1400):
        orc.step(target - done)
        done = target
        for f in STATE:
            sim.upload(f, orc.get(f))
        k_before = orc.get("khouot")
        sim.upload("khouot", k_before)
        sim.t = orc.t
        for _ in range(5):
            orc.step(1)
            done += 1
            sim.step(1)
            sim.sync()
            k = orc.get("khouot")
            seen_dry |= bool(((k_before == 0) & (k == 1)).any())
            seen_rewet |= bool(((k_before == 1) & (k == 0)).any())
            assert np.array_equal(sim.download("khouot"), k), orc.t
            front = _front_mask(k_before) | _front_mask(k)
            diffs = {}
            for f in FIELDS_STEP:
                a, r = sim.download(f), orc.get(f)
                diffs[f] = np.abs(a - r) / max(np.abs(r).max(), 1e-300)
            front_hit = any(d[front].max() > 1e-10 for d in diffs.values())
            for f, d in diffs.items():
                assert d.max() <= 2e-2, (orc.t, f, d.max())
                assert d[~front].max() <= (1e-6 if front_hit else 1e-10), (orc.t, f)
            for f in STATE:
                sim.upload(f, orc.get(f))
            sim.upload("khouot", k)
            k_before = k
    assert seen_dry and seen_rewet


def test_bed_feedback(hyd, oracle_mod):
    """The bed change fed back into the bed (h, htaiz, Kx1, Ky1 from the
    initial bed and dH once per step): against the oracle's restatement after
    the first steps with it (1e-10) and 30 more (1e-8); the bed has moved."""
    from hydist_c_b200 import scenario as S
    # Fw in the range of the reference's own Fw_map (0..0.0755): with the
    # U(0.5, 1.5) of the benchmark workload the bed-load flux moves the bed
    # by decimetres per step and the fed-back bed runs away
    b = S.make_channel(N=96, M=48, seed=20269000, dx=10.0, dt=2.0, hours=1.0, sediment=True,
                       sediment_start=10.0, fw=(0.02, 0.06))
    b["options"] = dict(b["options"], bed_change=1, bed_change_start=20.0, bed_feedback=1)
    sim = hyd.Simulation(b)
    orc = oracle_mod.OracleSim(b, nthreads=4)
    h_init = sim.download("h")
    sim.step(10)
    orc.step(10)
    sim.sync()
    fields = ["u", "v", "z", "FS", "dH", "h", "htaiz", "Kx1", "Ky1", "H_moi"]
    bad = _compare(sim, orc, fields, 1e-10)
    assert not bad, bad
    sim.step(30)
    orc.step(30)
    sim.sync()
    bad = _compare(sim, orc, fields, 1e-8)
    assert not bad, bad
    assert np.abs(sim.download("h") - h_init).max() > 0
