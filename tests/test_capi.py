"""CPU checks of the C ABI: the library loads without a GPU and exports every
function include/hydist_capi.h declares; argument errors come back as status
codes, not crashes."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared(header):
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hydist_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(hyd):
    lib = hyd.library()
    names = _declared("hydist_capi.h")
    assert "hydist_create" in names and "hydist_gtsv_batched" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_lists_every_export(hyd):
    from hydist_c_b200 import capi
    assert sorted(capi.EXPORTED_SYMBOLS) == _declared("hydist_capi.h")


def test_params_default_match_reference(hyd):
    from hydist_c_b200 import capi
    lib = hyd.library()
    p = capi.HydistParams()
    lib.hydist_params_default(C.byref(p))
    q = capi.default_params()
    for name, _ in capi.HydistParams._fields_:
        assert getattr(p, name) == getattr(q, name), name


def test_bienq_from_boundary_type(hyd):
    lib = hyd.library()
    bt = np.zeros(80, np.int32)
    bt[0], bt[2], bt[3] = 2, 2, 1
    out = (C.c_int32 * 4)()
    lib.hydist_bienq_from_boundary_type(bt.ctypes.data_as(C.POINTER(C.c_int32)), 80, out)
    assert list(out) == [1, 0, 1, 0]


def test_create_rejects_bad_arguments(hyd):
    from hydist_c_b200 import capi, scenario
    lib = hyd.library()
    h = C.c_void_p()
    st = lib.hydist_create(None, None, None, 0, C.byref(h))
    assert st == -1
    b = scenario.make_channel(N=16, M=12)
    ss = capi.ScenarioStruct(b["scenario"])
    ss.struct.M = 2
    p, o = capi.default_params(), capi.default_options()
    assert lib.hydist_create(C.byref(ss.struct), C.byref(p), C.byref(o), 0, C.byref(h)) == -1
    assert b"4x4" in lib.hydist_last_error()


def test_null_handle_is_an_error(hyd):
    lib = hyd.library()
    assert lib.hydist_step(None, 1) == -1
    assert lib.hydist_sync(None) == -1
    assert lib.hydist_destroy(None) == 0
    assert lib.hydist_gtsv_batched(None, None, None, None, None, None, None, 0, 0, 0, None) == -1
