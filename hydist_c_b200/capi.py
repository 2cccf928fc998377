"""ctypes mirror of include/hydist_capi.h and the loader of the CUDA library.

The structs below have the exact layout of the C header. ``load_library()``
opens the in-tree ``libhydist_b200.so`` (built by ``hydist_c_b200.build``) and
raises if it is missing: there is no CPU fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

SEGMENT_LIMIT = 20

HYDIST_OK = 0
STATUS_NAMES = {
    0: "HYDIST_OK", -1: "HYDIST_ERR_ARG", -2: "HYDIST_ERR_CUDA", -3: "HYDIST_ERR_OOM",
    -4: "HYDIST_ERR_SEGMENTS", -5: "HYDIST_ERR_STATE", -6: "HYDIST_ERR_BUDGET",
    -7: "HYDIST_ERR_TIMEOUT", -8: "HYDIST_ERR_NONFINITE", -9: "HYDIST_ERR_NODEVICE",
}

FIELDS = {
    "u": 0, "v": 1, "z": 2, "FS": 3, "tFS": 4, "H_moi": 5, "khouot": 6, "dH": 7,
    "Htdu": 8, "Htdv": 9, "t_u": 10, "t_v": 11, "t_z": 12, "Kx1": 13, "Ky1": 14,
    "VTH": 15, "Kx": 16, "Ky": 17, "h": 18, "htaiz": 19, "Qbx": 20, "Qby": 21,
}

FP64 = 0
FP32_REFINE = 1
FP32 = 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class HydistParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "dX", "dY", "dT", "NANGDAY", "H_TINH", "heso", "mu_mn", "NDnen",
        "Tod", "Toe", "hstoe", "ghtoe", "Mbochat", "ro", "ros",
        "dm", "d90", "muy", "Dorong", "Sx", "CORIOLIS_FORCE", "g",
        "Wind", "huonggio", "wss", "Ks")]


class HydistOptions(C.Structure):
    _fields_ = [("t_start", C.c_double), ("sediment_start", C.c_double),
                ("bed_change_start", C.c_double), ("ketdinh", C.c_int32),
                ("bed_change", C.c_int32), ("precision", C.c_int32),
                ("kenhhepd", C.c_int32), ("kenhhepng", C.c_int32),
                ("channel_wave", C.c_int32), ("reset_horizontal", C.c_int32),
                ("bed_feedback", C.c_int32), ("reserved", C.c_int32)]


class HydistScenario(C.Structure):
    _fields_ = [("M", C.c_int32), ("N", C.c_int32), ("total_time", C.c_int32),
                ("n_boundary_type", C.c_int32),
                ("h", _dp), ("hsnham", _dp), ("visco", _dp), ("Fw", _dp),
                ("bc_up", _dp), ("bc_down", _dp), ("bc_left", _dp), ("bc_right", _dp),
                ("CC_up", _dp), ("CC_down", _dp), ("CC_left", _dp), ("CC_right", _dp),
                ("boundary_type", _ip), ("bienQ", C.c_int32 * 4), ("FS0", _dp), ("z0", _dp)]


_vp = C.c_void_p
EXTERNAL_READONLY = ("h", "hsnham", "visco", "Fw", "htaiz", "htaiz_bd", "Kx1", "Ky1", "Tsxw", "Tsyw",
                     "bc_up", "bc_down", "bc_left", "bc_right", "CC_up", "CC_down", "CC_left",
                     "CC_right", "boundary_type")
EXTERNAL_STATE = ("u", "v", "z", "t_u", "t_v", "t_z", "H_moi", "Htdu", "Htdv", "FS", "tFS", "VTH",
                  "Kx", "Ky", "dH", "Qbx", "Qby", "khouot", "daui", "cuoii", "moci", "dauj",
                  "cuoij", "mocj", "ubt", "ubp", "vbt", "vbd")


class HydistExternal(C.Structure):
    """Caller-owned device arrays (include/hydist_capi.h); pointers as ints."""
    _fields_ = ([("M", C.c_int32), ("N", C.c_int32), ("total_time", C.c_int32),
                 ("bienQ", C.c_int32 * 4)] +
                [(k, _vp) for k in EXTERNAL_READONLY + EXTERNAL_STATE])


def default_params() -> HydistParams:
    """Reference constants of Load_coeffs (loader.cpp:4-87)."""
    p = HydistParams()
    p.dX, p.dY, p.dT = 10.0, 10.0, 2.0
    p.NANGDAY, p.H_TINH, p.heso, p.mu_mn = 0.0, 0.02, 0.94, 0.2
    p.NDnen = 0.0
    p.Tod, p.Toe, p.hstoe, p.ghtoe, p.Mbochat = 0.06, 0.15, 0.0, 3.0, 0.00001
    p.ro, p.ros = 1000.0, 2000.0
    p.dm, p.d90, p.muy, p.Dorong, p.Sx = 0.00001, 0.002, 1.01e-06, 0.5, 2.0
    p.CORIOLIS_FORCE, p.g = 0.0, 9.81
    p.Wind, p.huonggio = 0.0, 0.0
    p.wss, p.Ks = -1.0, -1.0
    return p


def default_options() -> HydistOptions:
    """Options as main.cpp:49-53 defaults them."""
    o = HydistOptions()
    o.t_start = 0.0
    o.sediment_start = 20 * 3600.0
    o.bed_change_start = 500 * 3600.0
    o.ketdinh = 1
    o.bed_change = 0
    o.precision = FP64
    return o


def _ptr(a, ctype=C.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


class ScenarioStruct:
    """Keeps the numpy arrays of a scenario alive while a HydistScenario
    struct points into them."""

    def __init__(self, sc: dict):
        self.arrays = {}
        for k in ("h", "hsnham", "visco", "Fw", "bc_up", "bc_down", "bc_left", "bc_right",
                  "CC_up", "CC_down", "CC_left", "CC_right"):
            self.arrays[k] = np.ascontiguousarray(sc[k], dtype=np.float64)
        self.arrays["boundary_type"] = np.ascontiguousarray(sc["boundary_type"], dtype=np.int32)
        for k in ("FS0", "z0"):
            a = sc.get(k)
            self.arrays[k] = None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        s = HydistScenario()
        s.M, s.N, s.total_time = int(sc["M"]), int(sc["N"]), int(sc["total_time"])
        s.n_boundary_type = int(self.arrays["boundary_type"].size)
        for k in ("h", "hsnham", "visco", "Fw", "bc_up", "bc_down", "bc_left", "bc_right",
                  "CC_up", "CC_down", "CC_left", "CC_right"):
            setattr(s, k, _ptr(self.arrays[k]))
        s.boundary_type = _ptr(self.arrays["boundary_type"], C.c_int32)
        for k in range(4):
            s.bienQ[k] = int(sc["bienQ"][k])
        s.FS0 = _ptr(self.arrays["FS0"])
        s.z0 = _ptr(self.arrays["z0"])
        self.struct = s


def params_from_dict(d: dict) -> HydistParams:
    p = default_params()
    for k, v in d.items():
        setattr(p, k, float(v))
    return p


def options_from_dict(d: dict) -> HydistOptions:
    o = default_options()
    for k, v in d.items():
        setattr(o, k, type(getattr(o, k))(v))
    return o


_PKG_DIR = Path(__file__).resolve().parent
LIB_NAME = "libhydist_b200.so"


def library_path() -> Path:
    return _PKG_DIR / LIB_NAME


_lib = None


def load_library():
    """Open the CUDA library; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not path.exists():
        raise RuntimeError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `python -m hydist_c_b200.build`; the package has no CPU fallback")
    lib = C.CDLL(str(path))
    _declare(lib)
    _lib = lib
    return lib


def _declare(lib):
    vp = C.c_void_p
    lib.hydist_last_error.restype = C.c_char_p
    lib.hydist_version.restype = C.c_char_p
    lib.hydist_params_default.argtypes = [C.POINTER(HydistParams)]
    lib.hydist_options_default.argtypes = [C.POINTER(HydistOptions)]
    lib.hydist_bienq_from_boundary_type.argtypes = [_ip, C.c_int32, _ip]
    lib.hydist_create.argtypes = [C.POINTER(HydistScenario), C.POINTER(HydistParams),
                                  C.POINTER(HydistOptions), C.c_int, C.POINTER(vp)]
    lib.hydist_destroy.argtypes = [vp]
    lib.hydist_step.argtypes = [vp, C.c_int32]
    lib.hydist_step_graph.argtypes = [vp, C.c_int32]
    lib.hydist_sync.argtypes = [vp]
    lib.hydist_get_time.argtypes = [vp, _dp]
    lib.hydist_set_time.argtypes = [vp, C.c_double]
    lib.hydist_download.argtypes = [vp, C.c_int32, vp]
    lib.hydist_upload.argtypes = [vp, C.c_int32, vp]
    lib.hydist_mass.argtypes = [vp, _dp]
    lib.hydist_stream.argtypes = [vp]
    lib.hydist_stream.restype = vp
    lib.hydist_step_traced.argtypes = [vp, C.POINTER(C.c_float)]
    lib.hydist_step_traced_sweeps.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    lib.hydist_kernel_launches.argtypes = [vp, C.POINTER(C.c_int64)]
    lib.hydist_create_phases.argtypes = [vp, C.POINTER(C.c_double)]
    lib.hydist_gtsv_batched.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int32, C.c_int32,
                                        C.c_int32, vp]
    lib.hydist_gtsv_batched_noalloc.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int32,
                                                C.c_int32, C.c_int32, vp]
    lib.hydist_gtsv_batched_refine.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int32, C.c_int32,
                                               vp]
    lib.hydist_gtsv_autotune.argtypes = [C.c_int32, vp, _ip]
    lib.hydist_create_external.argtypes = [C.POINTER(HydistExternal), C.POINTER(HydistParams),
                                           C.POINTER(HydistOptions), C.c_int, C.POINTER(vp)]
    lib.hydist_half_step.argtypes = [vp, C.c_int32]
    lib.hydist_ensemble_create.argtypes = [C.POINTER(vp), C.c_int32, C.POINTER(vp)]
    lib.hydist_ensemble_step.argtypes = [vp, C.c_int32]
    lib.hydist_ensemble_batched.argtypes = [vp, C.c_int32]
    lib.hydist_ensemble_sync.argtypes = [vp]
    lib.hydist_ensemble_destroy.argtypes = [vp]
    lib.hydist_ensemble_stream.argtypes = [vp]
    lib.hydist_ensemble_stream.restype = vp
    lib.hydist_checkpoint_save.argtypes = [vp, C.c_char_p]
    lib.hydist_checkpoint_load.argtypes = [vp, C.c_char_p]
    lib.hydist_scenario_bytes.argtypes = [C.c_int32, C.c_int32]
    lib.hydist_scenario_bytes.restype = C.c_int64
    lib.hydist_server_create.argtypes = [C.c_int, C.c_uint64, C.c_int32, C.POINTER(vp)]
    lib.hydist_server_destroy.argtypes = [vp]
    lib.hydist_server_submit.argtypes = [vp, C.POINTER(HydistScenario), C.POINTER(HydistParams),
                                         C.POINTER(HydistOptions), C.c_int32, C.POINTER(C.c_int64)]
    lib.hydist_server_round.argtypes = [vp, C.POINTER(C.c_int64), C.c_int32, _ip]
    lib.hydist_server_status.argtypes = [vp, C.c_int64, _ip, _ip]
    lib.hydist_server_counts.argtypes = [vp, _ip, _ip, C.POINTER(C.c_uint64)]
    lib.hydist_server_handle.argtypes = [vp, C.c_int64]
    lib.hydist_server_handle.restype = vp
    lib.hydist_server_release.argtypes = [vp, C.c_int64]
    lib.hydist_update_boundary.argtypes = [vp, C.c_double]
    lib.hydist_gtsv_band_bounds.argtypes = [_ip]


class HydistError(RuntimeError):
    pass


def check(lib, status: int, what: str):
    if status != HYDIST_OK:
        msg = lib.hydist_last_error()
        msg = msg.decode() if msg else ""
        raise HydistError(f"{what} failed: {STATUS_NAMES.get(status, status)}: {msg}")


EXPORTED_SYMBOLS = [
    "hydist_params_default", "hydist_options_default", "hydist_bienq_from_boundary_type",
    "hydist_last_error", "hydist_version", "hydist_create", "hydist_destroy", "hydist_step",
    "hydist_sync", "hydist_get_time", "hydist_set_time", "hydist_download", "hydist_upload", "hydist_mass",
    "hydist_step_graph", "hydist_stream", "hydist_gtsv_batched", "hydist_step_traced",
    "hydist_kernel_launches", "hydist_gtsv_batched_noalloc", "hydist_step_traced_sweeps",
    "hydist_gtsv_autotune", "hydist_gtsv_band_bounds", "hydist_create_external",
    "hydist_half_step", "hydist_update_boundary", "hydist_ensemble_create",
    "hydist_ensemble_step", "hydist_ensemble_sync", "hydist_ensemble_destroy",
    "hydist_ensemble_stream", "hydist_scenario_bytes", "hydist_server_create",
    "hydist_server_destroy", "hydist_server_submit", "hydist_server_round",
    "hydist_server_status", "hydist_server_counts", "hydist_server_handle",
    "hydist_server_release", "hydist_checkpoint_save", "hydist_checkpoint_load",
    "hydist_create_phases", "hydist_gtsv_batched_refine", "hydist_ensemble_batched",
]
GTSV_AUTO, GTSV_THOMAS, GTSV_PARTITION, GTSV_WARP, GTSV_PARTITION_512, GTSV_PARTITION_128, \
    GTSV_PIVOT = 0, 1, 2, 3, 4, 5, 6
GTSV_BANDS = 7

PHASES = ["boundary_x", "sweep_x", "explicit_v", "commit_x", "sediment_x",
          "boundary_y", "sweep_y", "explicit_u", "commit_y", "sediment_y"]
# the line-solver launches hydist_step_traced_sweeps times one by one
SWEEPS = ["line_solve_hydro_x", "line_solve_hydro_y", "line_solve_conc_x", "line_solve_conc_y"]
