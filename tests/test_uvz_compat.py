"""The kernel-level drop-in (include/hydist_uvz_compat.h,
include/hydist_gtsv_device.cuh).

1. The reference's own engine.cpp, support_funcs.cpp, loader.cpp and
   sediment_transport.cpp, linked with this library's UVZSolver kernels in
   place of UVZSolver_multithread.cpp and gtsv.cpp
   (oracle/_ref/hydist_ref_driver_uvz_b200, built by oracle/build.py from
   the reference sources where they lie), must give the reference's own
   results (oracle/_ref/hydist_ref_driver) on the same inputs: a channel with
   a discharge first end and a water-level last end on the x sweep, solid
   ends on the y sweep, and the concentration sweeps (whose systems the
   reference's Scan_FSj/Scan_FSi assemble and this library's tridiagSolver
   solves) from t = 0.
2. gtsv_spike_partial_diag_pivot_v1 solves diagonally dominant systems and
   systems that need 2x2 pivots to a small backward error, and leaves b
   unchanged.
"""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = ROOT / "oracle" / "_ref" / "hydist_ref_driver"
UVZ = ROOT / "oracle" / "_ref" / "hydist_ref_driver_uvz_b200"
STEPS = [1, 2, 10, 60]


def _run(exe, inputs, out, fs0):
    out.mkdir(parents=True, exist_ok=True)
    cmd = [str(exe), str(inputs) + "/", str(out), ",".join(map(str, STEPS)), "sediment_start=0",
           "bed_change_start=0", "dX=5", "Toe=0.2", "Tod=0.1", "Mbochat=0.0001", "wss=0.0005",
           f"fs0={fs0}"]
    # the reference prints t every half-step: stdout is discarded
    with open(os.devnull, "w") as f:
        r = subprocess.run(cmd, stdout=f, stderr=subprocess.PIPE, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.gpu
def test_reference_engine_on_library_kernels(hyd, tmp_path):
    if not (REF.exists() and UVZ.exists()):
        pytest.skip("oracle/_ref drivers not built (needs the reference sources)")
    from hydist_c_b200 import scenario as S
    from oracle.oracle import read_ref_state
    b = S.make_channel(N=96, M=48, seed=20265000, dx=5.0, dt=2.0, hours=1.0, sediment=True,
                       sediment_start=0.0)
    inputs = tmp_path / "inputs"
    S.write_reference_inputs(b["scenario"], inputs)
    fs0 = inputs / "fs0.bin"
    np.ascontiguousarray(b["scenario"]["FS0"], dtype="<f8").tofile(fs0)
    _run(REF, inputs, tmp_path / "ref", fs0)
    _run(UVZ, inputs, tmp_path / "uvz", fs0)
    for st in STEPS:
        ref = read_ref_state(tmp_path / "ref" / f"state_{st}.bin")["fields"]
        got = read_ref_state(tmp_path / "uvz" / f"state_{st}.bin")["fields"]
        np.testing.assert_array_equal(got["khouot"], ref["khouot"], err_msg=f"mask at step {st}")
        for f in ("u", "v", "z", "t_u", "t_v", "t_z", "FS"):
            scale = max(np.abs(ref[f]).max(), 1e-30)
            err = np.abs(got[f] - ref[f]).max() / scale
            # the cell arithmetic multiplies by reciprocals where the
            # reference divides: rounding-level differences that grow slowly
            assert err < 1e-9, f"{f} at step {st}: max difference {err:.3e} of max |{f}|"
    assert np.abs(read_ref_state(tmp_path / "uvz" / f"state_{STEPS[-1]}.bin")["fields"]["FS"]).max() > 0


@pytest.mark.gpu
def test_device_gtsv_pivoting(hyd, tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "gtsv_device_check"
    src = ROOT / "tests" / "native" / "gtsv_device_check.cu"
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
                        "-o", str(exe), str(src)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = {}
    for line in r.stdout.splitlines():
        kind, val, kept = line.split()
        res[kind] = float(val)
        assert kept == "b_unchanged=1", line
    assert set(res) == {"dominant", "zerodiag", "small"}, r.stdout
    assert res["dominant"] < 1e-14 and res["small"] < 1e-14, res
    assert res["zerodiag"] < 1e-12, res
