"""The C++ drop-in (include/hydist_compat.h): the reference's own main.cpp,
loader.cpp and set-up kernels linked against this library in place of the
reference's engine.cpp (oracle/_ref/hydist_ref_main_b200, built by
oracle/build.py from the reference sources where they lie).

The executable reads the scenario in the reference's text format, runs the
reference's set-up on its device arrays and calls Hydraulic_Calculation,
which this library implements on those arrays in place; the reference's
save_result / save_FS write the outputs. They must equal the library's own
run of the same scenario at the same times (to the 6 significant digits of
the text files): u, v, z at every saved time -- written in half-step B
before its commit, so the state after half-step A -- and FS at 360 s.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "oracle" / "_ref" / "hydist_ref_main_b200"


def _bundle():
    from hydist_c_b200 import scenario as S
    b = S.make_channel(N=96, M=48, seed=20265000, dx=10.0, dt=2.0, hours=1.0)
    # as main.cpp -b 0 -B 0: sediment sweeps and erosion source from t = 0;
    # the reference cannot load an initial concentration (loader.cpp:300)
    b["options"] = dict(b["options"], sediment_start=0.0, bed_change_start=0.0, ketdinh=1)
    b["scenario"]["FS0"] = None
    return b


def _read(path, N, M):
    a = np.loadtxt(path)
    assert a.shape == (N, M), (path, a.shape)
    return a


@pytest.mark.gpu
def test_reference_main_runs_on_library(hyd, tmp_path):
    if not EXE.exists():
        pytest.skip("oracle/_ref/hydist_ref_main_b200 not built (needs the reference sources)")
    from hydist_c_b200 import scenario as S
    b = _bundle()
    sc = b["scenario"]
    N, M = sc["N"], sc["M"]
    inputs = tmp_path / "Inputs"
    S.write_reference_inputs(sc, inputs)
    for d in ("U", "V", "Z", "FS"):
        (tmp_path / "Outputs" / d).mkdir(parents=True, exist_ok=True)
    cmd = [str(EXE), "-f", str(inputs) + "/", "-h", "0", "-m", "6", "-i", "60", "-b", "0", "-B", "0"]
    r = subprocess.run(cmd, cwd=tmp_path, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    sim = hyd.Simulation(b)
    t = 0
    for ts in (60, 120, 180, 240, 300, 360):
        # the reference writes at t = ts in half-step B before its commit:
        # the state after half-step A of the step ending at ts
        while t < ts - 2:
            sim.step(1)
            t += 2
        sim.half_step(0)
        got = {k: sim.download(k) for k in ("u", "v", "z")}
        sim.half_step(1)
        t += 2
        for k, name in (("u", "U/u"), ("v", "V/v"), ("z", "Z/z")):
            ref = _read(tmp_path / "Outputs" / f"{name}_{ts}.txt", N, M)
            ours = got[k][1:N + 1, 1:M + 1]
            np.testing.assert_allclose(ref, ours, rtol=2e-5, atol=1e-9, err_msg=f"{k} at t={ts}")
    fs_ref = _read(tmp_path / "Outputs" / "FS" / "fs_360.txt", N, M)
    fs = sim.download("FS")[1:N + 1, 1:M + 1] * 2000.0
    np.testing.assert_allclose(fs_ref, fs, rtol=2e-5, atol=1e-9)
    assert np.abs(fs).max() > 0  # the concentration sweeps ran
    sim.close()
