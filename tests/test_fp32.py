"""The FP32 forms (HYDIST_FP32_REFINE, and HYDIST_FP32 without the refinement
pass): FP32 fields, assembly and solves, FP64 water level, bed and mass. After one simulated hour of the 256x128 channel it
must stay within the stated tolerances of the FP64 form (which is itself
pinned to the oracle within 1e-6 over the same hour): max |dz| <= 1e-4 m,
relative difference of the water volume <= 1e-6, relative L2 of u and v
<= 1e-3; and a sediment case within 1e-3 relative L2 of FS."""
import numpy as np
import pytest

from hydist_c_b200 import scenario as S

pytestmark = pytest.mark.gpu


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("form", ["FP32_REFINE", "FP32"])
def test_fp32_one_hour_channel(hyd, form):
    b = S.config0()
    s64 = hyd.Simulation(b, precision=hyd.FP64)
    s32 = hyd.Simulation(b, precision=getattr(hyd, form))
    s64.step(1800)
    s32.step(1800)
    z64, z32 = s64.download("z"), s32.download("z")
    dz = float(np.abs(z32 - z64).max())
    assert dz <= 1e-4, dz
    m64, m32 = s64.mass(), s32.mass()
    assert abs(m32 - m64) / abs(m64) <= 1e-6, (m32, m64)
    for f in ("u", "v"):
        assert _rel_l2(s32.download(f), s64.download(f)) <= 1e-3, f
    assert np.array_equal(s32.download("khouot"), s64.download("khouot"))
    s64.close()
    s32.close()


@pytest.mark.parametrize("form", ["FP32_REFINE", "FP32"])
def test_fp32_sediment(hyd, form):
    b = S.make_channel(N=128, M=64, seed=20260500, dx=10.0, dt=2.0, hours=1.0, sediment=True,
                       sediment_start=20.0)
    s64 = hyd.Simulation(b, precision=hyd.FP64)
    s32 = hyd.Simulation(b, precision=getattr(hyd, form))
    s64.step(300)
    s32.step(300)
    assert _rel_l2(s32.download("FS"), s64.download("FS")) <= 1e-3
    assert float(np.abs(s32.download("z") - s64.download("z")).max()) <= 1e-4
    s64.close()
    s32.close()


def _volume(orc, N, M, dx, dy):
    k, ht, z = orc.get("khouot"), orc.get("htaiz"), orc.get("z")
    sl = (slice(2, N + 1), slice(2, M + 1))
    return float(np.sum(np.where(k[sl] == 0, ht[sl] + z[sl], 0.0))) * dx * dy


@pytest.mark.parametrize("form", ["FP32_REFINE", "FP32"])
def test_fp32_one_hour_against_oracle(hyd, oracle_mod, form):
    """The stated tolerances against the FP64 CPU oracle itself: after one
    simulated hour of the 256x128 channel, max |dz| <= 1e-4 m, the device's
    water volume within 1e-6 of the oracle's, relative L2 of u and v <= 1e-3,
    the same wet/dry mask; and after one hour of a sediment channel with the
    bed change (sediment from 600 s), the concentration and the bed change
    within 1e-3 relative L2."""
    b = S.config0()
    sim = hyd.Simulation(b, precision=getattr(hyd, form))
    orc = oracle_mod.OracleSim(b, nthreads=8)
    sim.step(1800)
    orc.step(1800)
    sim.sync()
    assert float(np.abs(sim.download("z") - orc.get("z")).max()) <= 1e-4
    N, M = b["scenario"]["N"], b["scenario"]["M"]
    vol = _volume(orc, N, M, 10.0, 10.0)
    assert abs(sim.mass() - vol) / abs(vol) <= 1e-6
    for f in ("u", "v"):
        assert _rel_l2(sim.download(f), orc.get(f)) <= 1e-3, f
    assert np.array_equal(sim.download("khouot"), orc.get("khouot"))
    sim.close()
    orc.close()
    b = S.make_channel(N=128, M=64, seed=20260501, dx=10.0, dt=2.0, hours=1.0, sediment=True,
                       sediment_start=600.0)
    b["options"]["bed_change"] = 1
    sim = hyd.Simulation(b, precision=getattr(hyd, form))
    orc = oracle_mod.OracleSim(b, nthreads=8)
    sim.step(1800)
    orc.step(1800)
    sim.sync()
    assert float(np.abs(sim.download("z") - orc.get("z")).max()) <= 1e-4
    for f in ("FS", "dH"):
        assert _rel_l2(sim.download(f), orc.get(f)) <= 1e-3, f
    sim.close()
    orc.close()
