"""hydist_c_b200 -- B200 (sm_100a) implementation of the Hydist_C ADI time step.

Python mirror of the reference's entry points for this path, over the C ABI
of ``libhydist_b200.so`` (include/hydist_capi.h):

=======================================  =====================================
reference (Hydist_C)                     here
=======================================  =====================================
main.cpp:138-304 set-up sequence         ``Simulation(bundle)``
Hydraulic_Calculation (engine.cpp:41)    ``Simulation.hydraulic_calculation``
one pass of its time loop                ``Simulation.step`` / ``step_graph``
synch_and_check (engine.cpp:13)          ``Simulation.sync``
save_result / save_FS (loader.cpp:397)   ``Simulation.download``
tridiag / gtsv_spike_partial_diag_pivot  ``gtsv_batched``
=======================================  =====================================

Errors are raised as :class:`HydistError`; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi, scenario
from .capi import FIELDS, FP32, FP32_REFINE, FP64, HydistError

__all__ = ["Simulation", "Ensemble", "Server", "gtsv_batched", "HydistError", "scenario", "FP64", "FP32", "FP32_REFINE",
           "FIELDS", "library"]


def library():
    return capi.load_library()


class Simulation:
    """One scenario resident on a GPU (the reference's Argument_Pointers,
    Array_Pointers and Constant_Coeffs of one run, engine.h:39-78)."""

    def __init__(self, bundle: dict, device: int = 0, precision: int | None = None):
        lib = capi.load_library()
        sc = bundle["scenario"]
        self.M, self.N = int(sc["M"]), int(sc["N"])
        self.shape = (self.N + 3, self.M + 3)
        self._ss = capi.ScenarioStruct(sc)
        self._p = capi.params_from_dict(bundle.get("params", {}))
        opts = dict(bundle.get("options", {}))
        if precision is not None:
            opts["precision"] = int(precision)
        self._o = capi.options_from_dict(opts)
        h = C.c_void_p()
        st = lib.hydist_create(C.byref(self._ss.struct), C.byref(self._p), C.byref(self._o),
                               int(device), C.byref(h))
        capi.check(lib, st, "hydist_create")
        self._h = h
        self._lib = lib
        self.dT = float(self._p.dT)

    # -- lifecycle
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.hydist_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- time stepping
    def step(self, n: int = 1):
        capi.check(self._lib, self._lib.hydist_step(self._h, int(n)), "hydist_step")

    def step_graph(self, n: int = 1):
        capi.check(self._lib, self._lib.hydist_step_graph(self._h, int(n)), "hydist_step_graph")

    def hydraulic_calculation(self, Tmax: float, graph: bool = False):
        """Advance while t < Tmax, one full step (two half-steps) at a time,
        as the while-loop of Hydraulic_Calculation (engine.cpp:65)."""
        n = 0
        t = self.t
        while t < int(Tmax):
            t += self.dT
            n += 1
        if n:
            (self.step_graph if graph else self.step)(n)
        return n

    def sync(self):
        capi.check(self._lib, self._lib.hydist_sync(self._h), "hydist_sync")

    def half_step(self, half: int):
        """One half of a step (0: x sweep half, 1: y sweep half); halves
        alternate starting with 0."""
        capi.check(self._lib, self._lib.hydist_half_step(self._h, int(half)), "hydist_half_step")

    def step_traced(self) -> dict:
        """One full step with per-phase device times (ms)."""
        ms = (C.c_float * len(capi.PHASES))()
        capi.check(self._lib, self._lib.hydist_step_traced(self._h, ms), "hydist_step_traced")
        return dict(zip(capi.PHASES, [float(x) for x in ms]))

    def step_traced_sweeps(self):
        """One full step with per-phase device times and the device time of
        each line-solver launch (ms): (phases, sweeps)."""
        ms = (C.c_float * len(capi.PHASES))()
        sw = (C.c_float * len(capi.SWEEPS))()
        capi.check(self._lib, self._lib.hydist_step_traced_sweeps(self._h, ms, sw),
                   "hydist_step_traced_sweeps")
        return (dict(zip(capi.PHASES, [float(x) for x in ms])),
                dict(zip(capi.SWEEPS, [float(x) for x in sw])))

    @property
    def kernel_launches(self) -> int:
        v = C.c_int64()
        capi.check(self._lib, self._lib.hydist_kernel_launches(self._h, C.byref(v)),
                   "hydist_kernel_launches")
        return int(v.value)

    @property
    def t(self) -> float:
        v = C.c_double()
        capi.check(self._lib, self._lib.hydist_get_time(self._h, C.byref(v)), "hydist_get_time")
        return v.value

    @t.setter
    def t(self, value: float):
        capi.check(self._lib, self._lib.hydist_set_time(self._h, float(value)), "hydist_set_time")

    @property
    def stream(self) -> int:
        return int(self._lib.hydist_stream(self._h) or 0)

    # -- fields
    def download(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """A field as a (N+3, M+3) array; `out` (C-contiguous, of that shape
        and the field's dtype, e.g. in pinned memory) receives it if given."""
        f = FIELDS[name]
        dt = np.int32 if name == "khouot" else np.float64
        if out is None:
            out = np.empty(self.shape, dtype=dt)
        elif out.shape != self.shape or out.dtype != dt or not out.flags.c_contiguous:
            raise ValueError(f"{name}: out must be a C-contiguous {dt.__name__} array of shape "
                             f"{self.shape}")
        capi.check(self._lib, self._lib.hydist_download(self._h, f, out.ctypes.data),
                   "hydist_download")
        return out

    def upload(self, name: str, arr):
        f = FIELDS[name]
        a = np.ascontiguousarray(arr, dtype=np.int32 if name == "khouot" else np.float64)
        if a.shape != self.shape:
            raise ValueError(f"{name}: expected shape {self.shape}, got {a.shape}")
        capi.check(self._lib, self._lib.hydist_upload(self._h, f, a.ctypes.data), "hydist_upload")

    def save(self, path):
        """Checkpoint the state and time to a file (hydist_checkpoint_save)."""
        capi.check(self._lib, self._lib.hydist_checkpoint_save(self._h, str(path).encode()),
                   "hydist_checkpoint_save")

    def load(self, path):
        """Restore a checkpoint of this scenario (hydist_checkpoint_load)."""
        capi.check(self._lib, self._lib.hydist_checkpoint_load(self._h, str(path).encode()),
                   "hydist_checkpoint_load")

    def create_phases(self) -> dict:
        """Host time of this handle's creation by part (ms)."""
        ms = (C.c_double * 4)()
        capi.check(self._lib, self._lib.hydist_create_phases(self._h, ms), "hydist_create_phases")
        return dict(zip(("alloc_ms", "inputs_ms", "setup_ms", "total_ms"), list(ms)))

    def mass(self) -> float:
        v = C.c_double()
        capi.check(self._lib, self._lib.hydist_mass(self._h, C.byref(v)), "hydist_mass")
        return v.value


class Ensemble:
    """Scenarios stepped together by one graph launch per step
    (hydist_ensemble_*). The members stay usable as Simulations."""

    def __init__(self, members):
        self._lib = capi.load_library()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m._h.value for m in self.members])
        e = C.c_void_p()
        capi.check(self._lib, self._lib.hydist_ensemble_create(arr, len(self.members), C.byref(e)),
                   "hydist_ensemble_create")
        self._e = e

    def step(self, n: int = 1):
        capi.check(self._lib, self._lib.hydist_ensemble_step(self._e, int(n)), "hydist_ensemble_step")

    def batched(self, enable: bool = True):
        """Batch the members' launches (the default where they allow it) or
        step them by their own launches (hydist_ensemble_batched)."""
        capi.check(self._lib, self._lib.hydist_ensemble_batched(self._e, int(bool(enable))),
                   "hydist_ensemble_batched")

    def sync(self):
        capi.check(self._lib, self._lib.hydist_ensemble_sync(self._e), "hydist_ensemble_sync")

    @property
    def stream(self) -> int:
        """The cudaStream_t the ensemble's graphs run on."""
        return self._lib.hydist_ensemble_stream(self._e)

    def close(self):
        if getattr(self, "_e", None) is not None and self._e.value:
            self._lib.hydist_ensemble_destroy(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous batching of scenario solves on one device
    (hydist_server_*): submit requests at any time, run rounds, collect
    finished requests."""

    QUEUED, ACTIVE, DONE = 0, 1, 2

    def __init__(self, budget_bytes: int, steps_per_round: int = 50, device: int = 0):
        self._lib = capi.load_library()
        s = C.c_void_p()
        capi.check(self._lib, self._lib.hydist_server_create(int(device), int(budget_bytes),
                                                             int(steps_per_round), C.byref(s)),
                   "hydist_server_create")
        self._s = s
        self._shape = {}

    @staticmethod
    def scenario_bytes(M: int, N: int) -> int:
        return int(capi.load_library().hydist_scenario_bytes(int(M), int(N)))

    def submit(self, bundle: dict, nsteps: int) -> int:
        sc = bundle["scenario"]
        ss = capi.ScenarioStruct(sc)
        p = capi.params_from_dict(bundle.get("params", {}))
        o = capi.options_from_dict(bundle.get("options", {}))
        rid = C.c_int64()
        capi.check(self._lib, self._lib.hydist_server_submit(self._s, C.byref(ss.struct), C.byref(p),
                                                             C.byref(o), int(nsteps), C.byref(rid)),
                   "hydist_server_submit")
        self._shape[rid.value] = (int(sc["N"]) + 3, int(sc["M"]) + 3)
        return rid.value

    def round(self) -> list:
        """One scheduling round; returns the ids finished in it."""
        cap = 4096
        done = (C.c_int64 * cap)()
        nd = C.c_int32()
        capi.check(self._lib, self._lib.hydist_server_round(self._s, done, cap, C.byref(nd)),
                   "hydist_server_round")
        return [done[i] for i in range(min(nd.value, cap))]

    def status(self, rid: int):
        st, k = C.c_int32(), C.c_int32()
        capi.check(self._lib, self._lib.hydist_server_status(self._s, int(rid), C.byref(st), C.byref(k)),
                   "hydist_server_status")
        return st.value, k.value

    def counts(self):
        q, a, b = C.c_int32(), C.c_int32(), C.c_uint64()
        capi.check(self._lib, self._lib.hydist_server_counts(self._s, C.byref(q), C.byref(a), C.byref(b)),
                   "hydist_server_counts")
        return q.value, a.value, b.value

    def download(self, rid: int, name: str) -> np.ndarray:
        h = self._lib.hydist_server_handle(self._s, int(rid))
        if not h:
            raise capi.HydistError(f"request {rid} is not finished")
        out = np.empty(self._shape[rid], dtype=np.int32 if name == "khouot" else np.float64)
        capi.check(self._lib, self._lib.hydist_download(C.c_void_p(h), FIELDS[name], out.ctypes.data),
                   "hydist_download")
        return out

    def release(self, rid: int):
        capi.check(self._lib, self._lib.hydist_server_release(self._s, int(rid)), "hydist_server_release")
        self._shape.pop(rid, None)

    def close(self):
        if getattr(self, "_s", None) is not None and self._s.value:
            self._lib.hydist_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gtsv_batched(dl, d, du, b, offsets, lengths, algo: int = 0, x=None, stream=None,
                 refine: bool = False):
    """Solve a packed batch of tridiagonal systems on the GPU.

    Arguments are CUDA tensors (torch) of one dtype (float64 or float32);
    offsets/lengths are int32 tensors. Returns x. algo (enum HydistGtsvAlgo):
    0 autotuned per length band, 1 Thomas, 2 / 4 / 5 the CTA partition
    solver on 256 / 512 / 128 threads, 3 the warp partition solver, 6
    Gaussian elimination with diagonal pivoting (for systems that are not
    diagonally dominant; the others do not pivot). refine (float64 only):
    solve in FP32 and refine once with the FP64 residual
    (hydist_gtsv_batched_refine).
    """
    import torch

    lib = capi.load_library()
    if d.dtype == torch.float64:
        dt = 0
    elif d.dtype == torch.float32:
        dt = 1
    else:
        raise TypeError("float64 or float32 expected")
    for t in (dl, d, du, b):
        if not (t.is_cuda and t.is_contiguous() and t.dtype == d.dtype):
            raise ValueError("dl, d, du, b must be contiguous CUDA tensors of one dtype")
    if x is None:
        x = torch.empty_like(d)
    offsets = offsets.to(device=d.device, dtype=torch.int32).contiguous()
    lengths = lengths.to(device=d.device, dtype=torch.int32).contiguous()
    if stream is None:
        stream = torch.cuda.current_stream(d.device).cuda_stream
    if refine:
        if dt != 0:
            raise TypeError("refine takes float64 systems")
        st = lib.hydist_gtsv_batched_refine(dl.data_ptr(), d.data_ptr(), du.data_ptr(),
                                            b.data_ptr(), x.data_ptr(), offsets.data_ptr(),
                                            lengths.data_ptr(), int(offsets.numel()), int(algo),
                                            C.c_void_p(stream))
        capi.check(lib, st, "hydist_gtsv_batched_refine")
        return x
    st = lib.hydist_gtsv_batched(dl.data_ptr(), d.data_ptr(), du.data_ptr(), b.data_ptr(),
                                 x.data_ptr(), offsets.data_ptr(), lengths.data_ptr(),
                                 int(offsets.numel()), dt, int(algo), C.c_void_p(stream))
    capi.check(lib, st, "hydist_gtsv_batched")
    return x
