"""Generates the golden fixtures that pin the CPU oracle to the reference.

Three steps, run where each can run:

1. ``inputs <dir>`` (here, where the reference source tree is): writes the
   reference-format input directories of the pinned cases under <dir>:
     - ``channel``   : the 256x128 channel case (dx=dy=10 m, dt=2 s);
     - ``luy``       : the reference's own river mesh (Inputs/, 464x324) with
                       its boundary types spread to the 80-entry side-major
                       layout the kernels index (support_funcs.cpp:705-721);
     - ``sediment``  : a 128x64 channel with the sediment sweeps and the
                       erosion source on from t=0 (dx=dy=5 m).
2. ``run <dir> <out>`` (on the GPU box): runs oracle/_ref/hydist_ref_driver,
   the reference's own time step built from its sources, on each case and
   writes full-precision state files under <out>/<case>/.
3. ``collect <out>`` (here): turns the state files into compact fixtures
   tests/golden/ref_<case>.npz: a strided subsample of u, v, z (and FS for the
   sediment case) at each saved step, plus the full wet/dry mask.

``luy-inputs`` (here) writes tests/golden/luy_inputs.npz, the reference's river
inputs in the scenario layout (for the pinned river case without the tree).

``kat`` (here) writes tests/golden/khouot_kat.npz: the reference's shipped
Inputs/bandodosau.txt and the wet/dry mask its Onetime_init produced from it
(Outputs/khouot.txt, written by main.cpp:268-280).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from hydist_c_b200 import scenario as S  # noqa: E402

# the reference's Inputs/ directory, under the source tree named by
# HYDIST_REFERENCE_SRC (the cases that need it are skipped without it)
_SRC = os.environ.get("HYDIST_REFERENCE_SRC")
REF_INPUTS = Path(_SRC) / "Inputs" if _SRC else Path("HYDIST_REFERENCE_SRC-unset")
CASES = {
    "channel": dict(steps=[1, 2, 10, 100, 1800], stride=3, fields=["u", "v", "z"],
                    args=[]),
    "luy": dict(steps=[1, 10, 100, 600], stride=5, fields=["u", "v", "z"], args=[]),
    "sediment": dict(steps=[1, 2, 10, 100, 300], stride=3, fields=["u", "v", "z", "FS"],
                     args=["sediment_start=0", "bed_change_start=0", "dX=5", "Toe=0.2",
                           "Tod=0.1", "Mbochat=0.0001", "wss=0.0005", "fs0=fs0.bin"]),
    # the reference's own (FMA-contracted) build and the oracle separate by
    # O(1) between steps 700 and 1000 of this case, once cells dry: the
    # smoothing's exact-zero test (support_funcs.cpp:770) turns rounding
    # differences at still-water cells into visible ones. Steps 1 and 700
    # are the pinned ones.
    "wetdry": dict(steps=[1, 700], stride=1, fields=["u", "v", "z"], args=[]),
    # wind stress and Coriolis force on (Constant_Coeffs Windx/Windy and
    # CORIOLIS_FORCE, loader.cpp:75,81-82; zero in the shipped Load_coeffs)
    "windcor": dict(steps=[1, 10, 100, 300], stride=2, fields=["u", "v", "z"],
                    args=["Wind=10", "huonggio=30", "CORIOLIS=0.0001"]),
    # non-cohesive sediment source (source_nchs, sediment_transport.cpp:41-49)
    "noncoh": dict(steps=[1, 10, 100, 300], stride=3, fields=["u", "v", "z", "FS"],
                   args=["sediment_start=0", "bed_change_start=0", "dX=5", "Toe=0.2",
                         "Tod=0.1", "Mbochat=0.0001", "wss=0.0005", "fs0=fs0.bin",
                         "ketdinh=0"]),
    # the narrow-channel modes (-kd, -kn): no boundary update, the sweeps'
    # ranges of engine.cpp:77-80 / 190-193; a sloshing initial level
    "narrow_d": dict(steps=[1, 10, 100, 300], stride=2, fields=["u", "v", "z"],
                     args=["z0=z0.bin", "kenhhepd=1"]),
    "narrow_n": dict(steps=[1, 10, 100, 300], stride=2, fields=["u", "v", "z"],
                     args=["z0=z0.bin", "kenhhepng=1"]),
}
# the cases a command runs: all, or those named in HYDIST_FIXTURE_CASES
# (comma-separated)
_SEL = os.environ.get("HYDIST_FIXTURE_CASES")
SELECTED = [c for c in CASES if not _SEL or c in _SEL.split(",")]


def sediment_bundle():
    b = S.make_channel(N=128, M=64, seed=20265000, dx=5.0, dt=2.0, hours=1.0, sediment=True,
                       sediment_start=0.0)
    b["options"]["bed_change_start"] = 0.0
    return b


LUY_NPZ = Path(__file__).resolve().parent / "luy_inputs.npz"


def luy_bundle():
    """The reference's river inputs as a scenario dict (from its Inputs/, or
    from tests/golden/luy_inputs.npz, the copy `luy-inputs` writes)."""
    if not REF_INPUTS.exists() and LUY_NPZ.exists():
        z = np.load(LUY_NPZ)
        sc = {k: z[k] for k in z.files if k not in ("M", "N", "total_time", "bienQ")}
        sc.update(M=int(z["M"]), N=int(z["N"]), total_time=int(z["total_time"]),
                  bienQ=[int(v) for v in z["bienQ"]], FS0=None)
        return dict(scenario=sc, params={},
                    options=dict(sediment_start=1e12, bed_change_start=1e12),
                    meta=dict(name="luy"))
    h = np.loadtxt(REF_INPUTS / "bandodosau.txt")
    n = h.size
    hs = np.loadtxt(REF_INPUTS / "hsnham.txt").ravel()[:n].reshape(h.shape)
    vi = np.loadtxt(REF_INPUTS / "hsnhotroiA.txt").ravel()[:n].reshape(h.shape)
    fw = np.loadtxt(REF_INPUTS / "Fw_map.txt").ravel()[:n].reshape(h.shape)
    rd = lambda f: np.loadtxt(REF_INPUTS / f).ravel()
    bt4 = np.loadtxt(REF_INPUTS / "boundary_type.txt").astype(np.int32).ravel()
    bt = np.zeros(80, np.int32)
    bt[:4] = bt4
    for s in range(4):
        bt[s * 20] = bt4[s]
    T = rd("bienduoi.txt").size
    sc = dict(M=h.shape[1] - 3, N=h.shape[0] - 3, total_time=T, h=h, hsnham=hs, visco=vi, Fw=fw,
              bc_up=rd("bientren.txt")[:T], bc_down=rd("bienphai.txt")[:T],
              bc_left=rd("bientrai.txt")[:T], bc_right=rd("bienduoi.txt")[:T],
              CC_up=rd("FS_bientren.txt")[:T], CC_down=rd("FS_bienduoi.txt")[:T],
              CC_left=rd("FS_bientrai.txt")[:T], CC_right=rd("FS_bienphai.txt")[:T],
              boundary_type=bt, bienQ=[int(bt[k] == 2) for k in range(4)], FS0=None)
    return dict(scenario=sc, params={}, options=dict(sediment_start=1e12, bed_change_start=1e12),
                meta=dict(name="luy"))


def wetdry_bundle():
    """A 64x32 basin: water level at the left end (i = 2), closed far end
    (dry rows past i = 61), a 0.25 m shelf with a 0.12 m patch near the far
    end, and a level swinging 0 -> -0.3 -> +0.3 m over two hours, so that
    cells dry and re-wet (Reset_states_vertical, support_funcs.cpp:142-188)."""
    b = S.make_channel(N=64, M=32, seed=21, dx=10.0, dt=2.0, hours=2.0)
    sc = b["scenario"]
    h = sc["h"]
    h[61:, :] = 0.0
    h[40:61, 3:31] = 0.25
    h[46:56, 10:22] = 0.12
    bt = np.zeros(80, np.int32)
    bt[40] = 1  # left side: water level
    sc["boundary_type"] = bt
    sc["bienQ"] = [0, 0, 0, 0]
    sc["bc_left"] = np.array([0.0, -0.3, 0.3, 0.3, 0.3])
    sc["total_time"] = 5
    for k in ("bc_up", "bc_down", "bc_right", "CC_up", "CC_down", "CC_left", "CC_right"):
        sc[k] = np.zeros(5)
    return b


def windcor_bundle():
    b = S.make_channel(N=128, M=64, seed=20265100, dx=10.0, dt=2.0, hours=1.0)
    b["params"] = dict(b["params"], Wind=10.0, huonggio=30.0, CORIOLIS_FORCE=1e-4)
    return b


def noncoh_bundle():
    b = sediment_bundle()
    b["options"] = dict(b["options"], ketdinh=0)
    return b


def narrow_bundle(kind):
    """A 96x48 channel at rest with a sloshing water level (0.05 m times a
    half cosine along x and a quarter along y), in the narrow-channel mode
    -kd (kind "d") or -kn ("n")."""
    b = S.make_channel(N=96, M=48, seed=20265200, dx=10.0, dt=2.0, hours=1.0)
    sc = b["scenario"]
    H, W = sc["h"].shape
    ii = np.arange(H, dtype=np.float64)[:, None]
    jj = np.arange(W, dtype=np.float64)[None, :]
    sc["z0"] = 0.05 * np.cos(np.pi * (ii - 2) / (H - 5)) * (1 + 0.25 * np.cos(0.5 * np.pi * jj / W))
    b["options"] = dict(b["options"], kenhhepd=int(kind == "d"), kenhhepng=int(kind == "n"))
    return b


def bundle(case):
    if case == "windcor":
        return windcor_bundle()
    if case == "noncoh":
        return noncoh_bundle()
    if case in ("narrow_d", "narrow_n"):
        return narrow_bundle(case[-1])
    if case == "channel":
        return S.config0()
    if case == "wetdry":
        return wetdry_bundle()
    if case == "sediment":
        return sediment_bundle()
    if case == "luy":
        return luy_bundle()
    raise KeyError(case)


def write_luy_inputs(d: Path):
    """Copy the reference's river inputs with an 80-entry boundary_type."""
    d.mkdir(parents=True, exist_ok=True)
    for f in REF_INPUTS.glob("*.txt"):
        if f.name == "boundary_type.txt":
            continue
        (d / f.name).write_bytes(f.read_bytes())
    bt = luy_bundle()["scenario"]["boundary_type"]
    (d / "boundary_type.txt").write_text("".join(f"{int(v)}\n" for v in bt))


def cmd_inputs(root):
    root = Path(root)
    for case in SELECTED:
        d = root / case
        if case == "luy":
            write_luy_inputs(d)
        else:
            b = bundle(case)
            S.write_reference_inputs(b["scenario"], d)
            for key, name in (("FS0", "fs0.bin"), ("z0", "z0.bin")):
                if b["scenario"].get(key) is not None:
                    np.ascontiguousarray(b["scenario"][key], dtype="<f8").tofile(d / name)
    print("inputs written under", root)


def cmd_run(root, out):
    root, out = Path(root), Path(out)
    drv = ROOT / "oracle" / "_ref" / "hydist_ref_driver"
    for case in SELECTED:
        spec = CASES[case]
        o = out / case
        o.mkdir(parents=True, exist_ok=True)
        args = [a.replace("fs0=fs0.bin", f"fs0={root / case / 'fs0.bin'}")
                 .replace("z0=z0.bin", f"z0={root / case / 'z0.bin'}") for a in spec["args"]]
        cmd = [str(drv), str(root / case) + "/", str(o), ",".join(map(str, spec["steps"]))] + args
        # the reference prints t every half-step (engine.cpp:67) and, on an
        # open water-level first end, one line per thread per half-step
        # (UVZSolver_multithread.cpp:137): stdout is discarded
        with open(os.devnull, "w") as f:
            r = subprocess.run(cmd, stdout=f, stderr=subprocess.PIPE, text=True)
        print(case, r.returncode, r.stderr[-2000:])
        if r.returncode != 0:
            raise SystemExit(r.returncode)


PACK_FIELDS = {"channel": ["u", "v", "z", "FS", "H_moi", "t_u", "t_v", "t_z", "khouot"],
               "luy": ["u", "v", "z", "khouot"],
               "wetdry": ["u", "v", "z", "H_moi", "t_u", "t_v", "t_z", "Htdu", "Htdv", "khouot"],
               "sediment": ["u", "v", "z", "FS", "tFS", "H_moi", "VTH", "Kx", "Ky", "khouot"],
               "windcor": ["u", "v", "z", "khouot"],
               "noncoh": ["u", "v", "z", "FS", "khouot"],
               "narrow_d": ["u", "v", "z", "khouot"],
               "narrow_n": ["u", "v", "z", "khouot"]}


def cmd_pack(out):
    """On the GPU box: full-precision state files -> one npz per case (the
    raw files are removed so that the results fit the return channel)."""
    from oracle.oracle import read_ref_state
    out = Path(out)
    for case in SELECTED:
        spec = CASES[case]
        arrs = {}
        for st in spec["steps"]:
            p = out / case / f"state_{st}.bin"
            r = read_ref_state(p)
            for f in PACK_FIELDS[case]:
                a = r["fields"][f]
                arrs[f"{f}_{st}"] = a.astype(np.int8) if f == "khouot" else a
            arrs[f"t_{st}"] = np.float64(r["t"])
            p.unlink()
        np.savez_compressed(out / f"full_{case}.npz", **arrs)
        print("packed", case)


def cmd_collect(out):
    out = Path(out)
    for case in SELECTED:
        spec = CASES[case]
        arrs = {}
        meta = dict(case=case, steps=spec["steps"], stride=spec["stride"], fields=spec["fields"])
        s = spec["stride"]
        full = np.load(out / f"full_{case}.npz")
        for st in spec["steps"]:
            for f in spec["fields"]:
                arrs[f"{f}_{st}"] = full[f"{f}_{st}"][::s, ::s].copy()
            arrs[f"khouot_{st}"] = full[f"khouot_{st}"].astype(np.int8)
            arrs[f"t_{st}"] = full[f"t_{st}"]
        np.savez_compressed(ROOT / "tests" / "golden" / f"ref_{case}.npz", meta=json.dumps(meta),
                            **arrs)
        print("wrote", case)


def cmd_luy_inputs():
    """tests/golden/luy_inputs.npz: the reference's river inputs (Inputs/) in
    the scenario layout, so that the pinned river case runs without the
    reference tree."""
    sc = luy_bundle()["scenario"]
    arrs = {k: np.asarray(v) for k, v in sc.items() if isinstance(v, np.ndarray)}
    np.savez_compressed(LUY_NPZ, **arrs, M=sc["M"], N=sc["N"], total_time=sc["total_time"],
                        bienQ=np.asarray(sc["bienQ"], dtype=np.int32))


def cmd_kat():
    h = np.loadtxt(REF_INPUTS / "bandodosau.txt")
    k = np.loadtxt(REF_INPUTS.parent / "Outputs" / "khouot.txt").astype(np.int8)
    np.savez_compressed(ROOT / "tests" / "golden" / "khouot_kat.npz", h=h, khouot=k)


if __name__ == "__main__":
    cmd = sys.argv[1]
    if cmd == "kat":
        cmd_kat()
    elif cmd == "inputs":
        cmd_inputs(sys.argv[2])
    elif cmd == "run":
        cmd_run(sys.argv[2], sys.argv[3])
    elif cmd == "pack":
        cmd_pack(sys.argv[2])
    elif cmd == "collect":
        cmd_collect(sys.argv[2])
    elif cmd == "luy-inputs":
        cmd_luy_inputs()
