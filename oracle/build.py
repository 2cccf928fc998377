"""TEST INFRASTRUCTURE: builds the CPU oracle and, where the reference source
tree is given, the reference driver.

The reference source tree is named by the caller (the ``src`` argument) or by
the environment variable HYDIST_REFERENCE_SRC (``reference_src()``); nothing
here assumes where it lies.

* ``build_oracle()`` compiles hydist_oracle.cpp into
  ``oracle/_build/libhydist_oracle.so`` (g++, FP64, no fused multiply-add).
* ``build_reference(src)`` compiles the reference's own CUDA sources where
  they lie (``src``; nothing is copied) with nvcc for sm_100a, links them
  with ``ref_driver.cu`` (our driver, which calls the reference's set-up
  functions and Hydraulic_Calculation and dumps the state in binary) and
  writes ``oracle/_ref/hydist_ref_driver``. It also builds
  ``oracle/_ref/hydist_ref_tridiag``, which runs the reference's device
  tridiag() on batched systems, and ``oracle/_ref/hydist_ref_main_b200``:
  the reference's own main.cpp, loader.cpp and set-up kernels linked against
  this repository's library in place of the reference's engine.cpp (the
  drop-in check of tests/test_compat.py), and
  ``oracle/_ref/hydist_ref_driver_uvz_b200``: the driver with the reference's
  own engine.cpp, support_funcs.cpp, loader.cpp and sediment_transport.cpp
  but this library's UVZSolver kernels in place of UVZSolver_multithread.cpp
  and gtsv.cpp (the kernel-level drop-in check of tests/test_uvz_compat.py).
  Outputs go to oracle/_ref/ only.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
REF_OUT = HERE / "_ref"
ORACLE_SO = BUILD / "libhydist_oracle.so"
REF_DRIVER = REF_OUT / "hydist_ref_driver"
REF_TRIDIAG = REF_OUT / "hydist_ref_tridiag"
# the reference's own main.cpp + loader.cpp + set-up kernels, linked against
# this repository's library in place of engine.cpp (the drop-in check)
REF_MAIN_B200 = REF_OUT / "hydist_ref_main_b200"
# the driver on the reference's engine with this library's UVZSolver kernels
REF_DRIVER_UVZ = REF_OUT / "hydist_ref_driver_uvz_b200"
PRODUCT_DIR = HERE.parent / "hydist_c_b200"
REF_SOURCES = ["engine.cpp", "support_funcs.cpp", "UVZSolver_multithread.cpp", "loader.cpp",
               "sediment_transport.cpp", "gtsv.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
    return r


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_oracle(force=False) -> Path:
    BUILD.mkdir(exist_ok=True)
    src = HERE / "hydist_oracle.cpp"
    deps = [src, HERE / "hydist_oracle.h", HERE.parent / "include" / "hydist_capi.h"]
    if force or _stale(ORACLE_SO, deps):
        tmp = ORACLE_SO.with_suffix(".so.tmp")
        _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
              "-fPIC", "-shared", "-o", str(tmp), str(src)])
        os.replace(tmp, ORACLE_SO)
    return ORACLE_SO


def reference_src():
    """The reference source tree named by HYDIST_REFERENCE_SRC, or None."""
    p = os.environ.get("HYDIST_REFERENCE_SRC")
    return Path(p) if p else None


def build_reference(src, force=False):
    """Compile the reference CUDA sources from ``src`` into oracle/_ref."""
    src = Path(src)
    if not (src / "engine.cpp").exists():
        return None
    if shutil.which("nvcc") is None:
        return None
    REF_OUT.mkdir(exist_ok=True)
    objdir = REF_OUT / "obj"
    objdir.mkdir(exist_ok=True)
    drv = HERE / "ref_driver.cu"
    tri = HERE / "ref_tridiag.cu"
    deps = [drv, tri] + [src / s for s in REF_SOURCES]
    if not force and not _stale(REF_DRIVER, deps) and not _stale(REF_TRIDIAG, deps):
        if not REF_MAIN_B200.exists():
            build_reference_main_on_library(src)
        if not REF_DRIVER_UVZ.exists():
            build_reference_engine_on_library_kernels(src)
        return REF_DRIVER
    objs = []
    for s in REF_SOURCES:
        o = objdir / (Path(s).stem + ".o")
        _run(["nvcc", "-std=c++11", f"-I{src}", "-x", "cu", *ARCH, "-O3", "-w", "-dc",
              str(src / s), "-o", str(o)])
        objs.append(str(o))
    d_o = objdir / "ref_driver.o"
    _run(["nvcc", "-std=c++14", f"-I{src}", "-x", "cu", *ARCH, "-O3", "-w", "-dc", str(drv),
          "-o", str(d_o)])
    _run(["nvcc", *ARCH, *objs, str(d_o), "-o", str(REF_DRIVER)])
    t_o = objdir / "ref_tridiag.o"
    _run(["nvcc", "-std=c++14", f"-I{src}", "-x", "cu", *ARCH, "-O3", "-w", "-dc", str(tri),
          "-o", str(t_o)])
    _run(["nvcc", *ARCH, str(objdir / "UVZSolver_multithread.o"), str(objdir / "support_funcs.o"),
          str(objdir / "gtsv.o"), str(t_o), "-o", str(REF_TRIDIAG)])
    build_reference_main_on_library(src)
    build_reference_engine_on_library_kernels(src)
    return REF_DRIVER


def build_reference_engine_on_library_kernels(src):
    """Link ref_driver.cu and the reference's engine.cpp, support_funcs.cpp,
    loader.cpp and sediment_transport.cpp (objects from build_reference) with
    libhydist_b200.so for the UVZSolver kernels (include/hydist_uvz_compat.h):
    the reference's engine launches this library's kernels unchanged."""
    src = Path(src)
    lib = PRODUCT_DIR / "libhydist_b200.so"
    objdir = REF_OUT / "obj"
    names = ["ref_driver.o", "engine.o", "support_funcs.o", "loader.o", "sediment_transport.o"]
    objs = [objdir / n for n in names]
    if not lib.exists() or not all(o.exists() for o in objs):
        return None
    # -cudart shared: the engine's launches of the library's kernels pass
    # their configuration through the CUDA runtime, which must be the
    # library's (the shared one), not a static copy in the executable
    _run(["nvcc", *ARCH, "-cudart", "shared", *map(str, objs), f"-L{PRODUCT_DIR}", "-lhydist_b200",
          "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../../hydist_c_b200", "-o", str(REF_DRIVER_UVZ)])
    return REF_DRIVER_UVZ


def build_reference_main_on_library(src):
    """Link the reference's main.cpp, loader.cpp and support_funcs.cpp (its
    set-up kernels) with libhydist_b200.so instead of engine.cpp: the
    library's Hydraulic_Calculation / update_boundary_at_t / synch_and_check
    (include/hydist_compat.h) must satisfy the reference's own main unchanged.
    The executable finds the library through an rpath relative to itself."""
    src = Path(src)
    lib = PRODUCT_DIR / "libhydist_b200.so"
    if not (src / "main.cpp").exists() or not lib.exists():
        return None
    objdir = REF_OUT / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    objs = []
    for s in ("main.cpp", "loader.cpp", "support_funcs.cpp"):
        o = objdir / (Path(s).stem + ".o")
        if _stale(o, [src / s]):
            _run(["nvcc", "-std=c++11", f"-I{src}", "-x", "cu", *ARCH, "-O3", "-w", "-dc",
                  str(src / s), "-o", str(o)])
        objs.append(str(o))
    _run(["nvcc", *ARCH, *objs, f"-L{PRODUCT_DIR}", "-lhydist_b200",
          "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../../hydist_c_b200", "-o", str(REF_MAIN_B200)])
    return REF_MAIN_B200


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    if "--ref" in sys.argv:
        src = reference_src()
        if src is None:
            sys.exit("set HYDIST_REFERENCE_SRC to the reference source tree")
        print(build_reference(src, force="--force" in sys.argv))
