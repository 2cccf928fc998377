"""The wet-run scan of Find_Calculation_limits_* (support_funcs.cpp:260-288)
restated as a fixed-trip loop and as the per-cell run-start/run-end flags of
hydro.cu (run_flags / k_runs_flags, each cell deciding alone, starts and ends
then sorted per line): all formulations produce the same segment tables on
random masks, including runs that touch the line's end and the dropped run
starting at lim-1."""
import numpy as np


def scan_reference(K, lim):
    """The reference's while-loop, as in the oracle."""
    dau, cuoi = [], []
    start = 2
    while start < lim:
        if K[start] != 0:
            while K[start] and start < lim:
                start += 1
        if start + 1 == lim:
            start = lim
        if K[start] == 0 and start + 1 < lim:
            dau.append(start)
            end = start
            while K[end] == 0 and end < lim:
                end += 1
            if K[end] != 0 and end <= lim:
                cuoi.append(end - 1)
                start = end
            else:
                cuoi.append(lim)
                start = lim
    return dau, cuoi


def scan_runs(K, lim):
    dau, cuoi = [], []
    s, inside = 0, False
    for p in range(2, lim + 1):
        wet = K[p] == 0
        if wet and not inside:
            inside, s = True, p
        elif not wet and inside:
            inside = False
            if s <= lim - 2:
                dau.append(s)
                cuoi.append(p - 1)
    if inside and s <= lim - 2:
        dau.append(s)
        cuoi.append(lim)
    return dau, cuoi


def scan_flags(K, lim):
    """hydro.cu run_flags: a cell starts a run if it is wet, its left
    neighbour dry (or it is position 2) and it lies at or before lim-2; it
    ends one if it is wet, its right neighbour dry (or it is lim) and the run
    it ends starts at or before lim-2."""
    wet = lambda p: K[p] == 0
    dau, cuoi = [], []
    for p in range(2, lim + 1):
        if not wet(p):
            continue
        if (p == 2 or not wet(p - 1)) and p <= lim - 2:
            dau.append(p)
        ok = True
        if p == lim - 1:
            ok = wet(lim - 2)
        elif p == lim:
            ok = wet(lim - 1) and wet(lim - 2)
        if (p == lim or not wet(p + 1)) and ok:
            cuoi.append(p)
    return sorted(dau), sorted(cuoi)


def test_scan_formulations_agree():
    rng = np.random.default_rng(0)
    for trial in range(4000):
        lim = int(rng.integers(4, 40))
        p_dry = rng.uniform(0.0, 0.6)
        K = np.where(rng.uniform(size=lim + 3) < p_dry, rng.choice([1, 2], size=lim + 3), 0)
        ref = scan_reference(K, lim)
        assert ref == scan_runs(K, lim), (K.tolist(), lim)
        assert ref == scan_flags(K, lim), (K.tolist(), lim)


def test_scan_edge_cases():
    lim = 10
    K = np.zeros(lim + 3, int)
    K[lim - 2] = 2  # a wet run starting at lim-1 is dropped
    assert scan_reference(K, lim) == scan_runs(K, lim) == scan_flags(K, lim) == ([2], [lim - 3])
    K = np.zeros(lim + 3, int)
    assert scan_runs(K, lim) == scan_flags(K, lim) == ([2], [lim])
