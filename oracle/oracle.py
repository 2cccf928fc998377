"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the FP64 CPU oracle.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import struct
from pathlib import Path

import numpy as np

from hydist_c_b200 import capi
from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build_oracle()
        L = C.CDLL(str(path))
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_create.argtypes = [C.POINTER(capi.HydistScenario), C.POINTER(capi.HydistParams),
                                    C.POINTER(capi.HydistOptions), C.c_int]
        L.oracle_create.restype = vp
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_race_mode.argtypes = [vp, C.c_int]
        L.oracle_step.argtypes = [vp, C.c_int]
        L.oracle_time.argtypes = [vp]
        L.oracle_time.restype = C.c_double
        L.oracle_set_time.argtypes = [vp, C.c_double]
        L.oracle_rescan_segments.argtypes = [vp]
        L.oracle_get.argtypes = [vp, C.c_int, vp]
        L.oracle_set.argtypes = [vp, C.c_int, vp]
        L.oracle_get_segments.argtypes = [vp, C.c_int, ip, ip, ip]
        L.oracle_get_boundary.argtypes = [vp, dp, dp, dp, dp, dp, dp]
        L.oracle_thomas.argtypes = [C.c_int, dp, dp, dp, dp, dp]
        L.oracle_thomas_batched.argtypes = [dp, dp, dp, dp, dp, ip, ip, C.c_int, C.c_int]
        _lib = L
    return _lib


class OracleSim:
    """One scenario advanced by the CPU oracle."""

    def __init__(self, bundle: dict, nthreads: int = 1, race_new: int = 1):
        L = lib()
        sc = bundle["scenario"]
        self.M, self.N = int(sc["M"]), int(sc["N"])
        self.shape = (self.N + 3, self.M + 3)
        self._ss = capi.ScenarioStruct(sc)
        self._p = capi.params_from_dict(bundle.get("params", {}))
        self._o = capi.options_from_dict(bundle.get("options", {}))
        h = L.oracle_create(C.byref(self._ss.struct), C.byref(self._p), C.byref(self._o),
                            int(nthreads))
        if not h:
            raise RuntimeError("oracle_create: " + L.oracle_last_error().decode())
        self._h = h
        L.oracle_set_race_mode(h, int(race_new))

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    __del__ = close

    def step(self, n=1):
        st = lib().oracle_step(self._h, int(n))
        if st != 0:
            raise RuntimeError("oracle_step: " + lib().oracle_last_error().decode())

    @property
    def t(self):
        return lib().oracle_time(self._h)

    @t.setter
    def t(self, value):
        lib().oracle_set_time(self._h, float(value))

    def load_state(self, fields: dict):
        """Set the given fields (name -> array; the mask as "khouot") and
        rebuild the segment tables from the mask."""
        for name, arr in fields.items():
            self.set(name, arr)
        st = lib().oracle_rescan_segments(self._h)
        if st != 0:
            raise RuntimeError("oracle_rescan_segments: " + lib().oracle_last_error().decode())

    def get(self, name):
        f = capi.FIELDS[name]
        if name == "khouot":
            out = np.empty(self.shape, dtype=np.int32)
        else:
            out = np.empty(self.shape, dtype=np.float64)
        lib().oracle_get(self._h, f, out.ctypes.data)
        return out

    def set(self, name, arr):
        f = capi.FIELDS[name]
        dt = np.int32 if name == "khouot" else np.float64
        a = np.ascontiguousarray(arr, dtype=dt)
        assert a.shape == self.shape
        lib().oracle_set(self._h, f, a.ctypes.data)

    def segments(self, kind):
        n = (self.N + 3) if kind == 0 else (self.M + 3)
        dau = np.zeros(n * capi.SEGMENT_LIMIT, np.int32)
        cuoi = np.zeros_like(dau)
        moc = np.zeros(n, np.int32)
        ip = C.POINTER(C.c_int32)
        lib().oracle_get_segments(self._h, kind, dau.ctypes.data_as(ip), cuoi.ctypes.data_as(ip),
                                  moc.ctypes.data_as(ip))
        return dau.reshape(n, -1), cuoi.reshape(n, -1), moc

    def boundary(self):
        M, N = self.M, self.N
        ubt, ubp = np.zeros(M + 3), np.zeros(M + 3)
        vbt, vbd = np.zeros(N + 3), np.zeros(N + 3)
        hi = np.zeros(2 * (M + N + 6))
        hmax = np.zeros(4)
        dp = C.POINTER(C.c_double)
        lib().oracle_get_boundary(self._h, *(a.ctypes.data_as(dp) for a in (ubt, ubp, vbt, vbd, hi, hmax)))
        return dict(ubt=ubt, ubp=ubp, vbt=vbt, vbd=vbd, hi=hi, hmax=hmax)


def thomas(dl, d, du, b):
    n = len(d)
    x = np.zeros(n)
    dp = C.POINTER(C.c_double)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dl, d, du, b)]
    lib().oracle_thomas(n, *(a.ctypes.data_as(dp) for a in arrs), x.ctypes.data_as(dp))
    return x


def thomas_batched(dl, d, du, b, offsets, lengths, nthreads=1):
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dl, d, du, b)]
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    ln = np.ascontiguousarray(lengths, dtype=np.int32)
    x = np.zeros(len(arrs[1]))
    lib().oracle_thomas_batched(*(a.ctypes.data_as(dp) for a in arrs), x.ctypes.data_as(dp),
                                off.ctypes.data_as(ip), ln.ctypes.data_as(ip), len(off), int(nthreads))
    return x


REF_FIELDS = ["u", "v", "z", "FS", "H_moi", "t_u", "t_v", "t_z", "Htdu", "Htdv", "khouot", "tFS",
              "VTH", "Kx", "Ky"]


def read_ref_state(path):
    """Read a state file written by ref_driver.cu."""
    raw = Path(path).read_bytes()
    N, M, steps, nf = struct.unpack_from("<4i", raw, 0)
    (t,) = struct.unpack_from("<d", raw, 16)
    n = (N + 3) * (M + 3)
    arr = np.frombuffer(raw, dtype="<f8", offset=24, count=nf * n).reshape(nf, N + 3, M + 3)
    out = {name: arr[k].copy() for k, name in enumerate(REF_FIELDS[:nf])}
    out["khouot"] = out["khouot"].astype(np.int32)
    return dict(N=N, M=M, steps=steps, t=t, fields=out)
