"""Errors the time step reports from the device, made on the host (no GPU
fault is involved): a line with more wet segments than the segment tables
hold (HYDIST_ERR_SEGMENTS, the reference's 20-per-line limit, engine.h:12),
and a NaN planted in an uploaded field, which the commits' canary reports at
the next synchronisation (HYDIST_ERR_NONFINITE)."""
import numpy as np
import pytest

from hydist_c_b200 import scenario as S

pytestmark = pytest.mark.gpu


def _comb_depths(h, row, period=4):
    """Node depths that make cell row `row` alternate 3 wet cells and 1 dry
    cell: a cell is dry when its four corner nodes are at NANGDAY (0), so a
    pair of zero node columns in node rows row-1 and row dries one cell of
    that row and no other."""
    W = h.shape[1]
    for j0 in range(4, W - 3, period):
        h[row - 1:row + 1, j0 - 1:j0 + 1] = 0.0
    return h


def test_segment_overflow_at_create(hyd):
    b = S.make_channel(N=40, M=120, seed=3)
    _comb_depths(b["scenario"]["h"], 20)
    with pytest.raises(hyd.HydistError, match="HYDIST_ERR_SEGMENTS"):
        hyd.Simulation(b)


def test_segment_overflow_from_uploaded_mask(hyd):
    b = S.make_channel(N=40, M=120, seed=3)
    sim = hyd.Simulation(b)
    sim.step(2)
    sim.sync()
    k = sim.download("khouot")
    k[20, 4:k.shape[1] - 3:4] = 1  # 26 wet runs in row 20
    sim.upload("khouot", k)
    with pytest.raises(hyd.HydistError, match="HYDIST_ERR_SEGMENTS"):
        sim.sync()
    sim.close()


def test_nan_in_state_is_reported(hyd):
    b = S.make_channel(N=48, M=24, seed=5)
    sim = hyd.Simulation(b)
    sim.step(3)
    sim.sync()  # finite so far: no error
    u = sim.download("u")
    u[20, 12] = np.nan
    sim.upload("u", u)
    sim.step(1)
    with pytest.raises(hyd.HydistError, match="HYDIST_ERR_NONFINITE"):
        sim.sync()
    sim.close()


def test_inf_in_concentration_is_reported(hyd):
    b = S.make_channel(N=48, M=24, seed=6, sediment=True, sediment_start=0.0)
    sim = hyd.Simulation(b)
    sim.step(2)
    sim.sync()
    fs = sim.download("FS")
    fs[24, 12] = np.inf
    sim.upload("FS", fs)
    sim.step(1)
    with pytest.raises(hyd.HydistError, match="HYDIST_ERR_NONFINITE"):
        sim.sync()
    sim.close()
