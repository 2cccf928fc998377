"""Ensembles (hydist_ensemble_*): scenarios stepped together by one graph
launch per step must give each member exactly what it gives alone, through
the start of the sediment sweeps (a new graph pattern) and with members on
different phases."""
import numpy as np
import pytest


def _member(k, sed_start):
    from hydist_c_b200 import scenario as S
    return S.make_channel(N=64, M=32, seed=20266000 + k, dx=10.0, dt=2.0, hours=1.0,
                          sediment=True, sediment_start=sed_start)


@pytest.mark.gpu
def test_ensemble_equals_members_alone(hyd):
    # member 2 starts its sediment sweeps later: the patterns differ per member
    starts = [20.0, 20.0, 40.0]
    alone = []
    for k, s0 in enumerate(starts):
        sim = hyd.Simulation(_member(k, s0))
        sim.step(30)
        alone.append({f: sim.download(f) for f in ("u", "v", "z", "FS")})
        sim.close()
    mix = [hyd.Simulation(_member(k, s0)) for k, s0 in enumerate(starts)]
    ens = hyd.Ensemble(mix)
    ens.step(12)
    ens.step(18)
    ens.sync()
    for k, sim in enumerate(mix):
        assert sim.t == pytest.approx(60.0)
        for f, ref in alone[k].items():
            np.testing.assert_array_equal(sim.download(f), ref, err_msg=f"member {k} {f}")
    # members remain usable alone after the ensemble steps
    mix[0].step(1)
    ens.close()
    for sim in mix:
        sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["FP64", "FP32_REFINE"])
def test_batched_ensemble_launches_once_per_kernel(hyd, precision):
    """Members of one mesh size in the same phase share every launch (one
    launch per kernel of the step for the whole batch), with each member's
    result bitwise what it is alone; the same ensemble stepped by per-member
    launches gives the same."""
    prec = getattr(hyd, precision)
    members = [_member(k, 10.0) for k in range(4)]
    alone = []
    for b in members:
        sim = hyd.Simulation(b, precision=prec)
        sim.step(16)
        alone.append({f: sim.download(f) for f in ("u", "v", "z", "FS")})
        sim.close()
    mix = [hyd.Simulation(b, precision=prec) for b in members]
    ens = hyd.Ensemble(mix)
    n0 = mix[0].kernel_launches
    ens.step(8)
    ens.sync()
    per_step_batched = (mix[0].kernel_launches - n0) / 8
    ens.batched(False)
    n1 = mix[0].kernel_launches
    ens.step(8)
    ens.sync()
    per_step_members = (mix[0].kernel_launches - n1) / 8
    for k, sim in enumerate(mix):
        for f, ref in alone[k].items():
            np.testing.assert_array_equal(sim.download(f), ref, err_msg=f"member {k} {f}")
    # the batch's steps launch as many kernels as one member's steps alone
    solo = hyd.Simulation(members[0], precision=prec)
    l0 = solo.kernel_launches
    solo.step(8)
    l1 = solo.kernel_launches
    solo.step(8)
    assert per_step_batched == (l1 - l0) / 8
    assert per_step_members == 4 * (solo.kernel_launches - l1) / 8
    ens.close()
    for sim in mix + [solo]:
        sim.close()
