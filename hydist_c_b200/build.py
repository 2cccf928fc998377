"""Builds the CUDA library libhydist_b200.so in-tree with nvcc for sm_100a.

    python -m hydist_c_b200.build [--force]

The sources are compiled as separate translation units and linked into one
shared object with a C ABI (include/hydist_capi.h). Nothing is JIT-compiled
at import time; the product fails loudly if the library is missing.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libhydist_b200.so"
SOURCES = ["engine.cu", "hydro.cu", "sweep.cu", "sediment.cu", "tridiag.cu", "compat.cu", "server.cu",
           "uvz_compat.cu"]
HEADERS = ["common.cuh", "hydro.cuh", "assembly.cuh", "linesolve.cuh", "partsolve.cuh", "sediment_cell.cuh",
           "explicit.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-v"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (Path(c).exists() or c == "nvcc"):
            return c
    return "nvcc"


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    nvcc = _nvcc()
    hdrs = [CSRC / h for h in HEADERS] + [ROOT / "include" / h for h in (
        "hydist_capi.h", "hydist_compat.h", "hydist_uvz_compat.h", "hydist_gtsv_device.cuh")]
    objs = []
    logs = []
    for s in SOURCES:
        src = CSRC / s
        o = OBJ / (src.stem + ".o")
        objs.append(o)
        if force or _stale(o, [src] + hdrs):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(o)]
            r = subprocess.run(cmd, capture_output=True, text=True)
            logs.append(f"== {s}\n{r.stdout}{r.stderr}")
            if r.returncode != 0:
                raise RuntimeError("nvcc failed on %s:\n%s%s" % (s, r.stdout, r.stderr))
    if force or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
        os.replace(tmp, LIB)
    if logs:
        (OBJ / "ptxas.log").write_text("\n".join(logs))
        if verbose:
            print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
