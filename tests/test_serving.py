"""Serving (hydist_server_*): continuous batching. Requests of different mesh
sizes and horizons, one of them arriving while the others run, under a
budget that holds two at a time: each result must equal the same scenario
solved alone, bit for bit; a scenario larger than the budget is refused."""
import numpy as np
import pytest


def _req(k, N, M):
    from hydist_c_b200 import scenario as S
    return S.make_channel(N=N, M=M, seed=20267000 + k, dx=10.0, dt=2.0, hours=1.0,
                          sediment=True, sediment_start=20.0)


def test_scenario_bytes_grow_with_the_mesh(hyd):
    from hydist_c_b200 import Server
    a, b, c = Server.scenario_bytes(128, 64), Server.scenario_bytes(256, 128), Server.scenario_bytes(2048, 1024)
    assert 0 < a <= b < c
    assert c > 30 * 2051 * 1027 * 8  # at least the 30 mesh-sized arrays


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix(hyd):
    from hydist_c_b200 import Server
    specs = [(0, 64, 32, 37), (1, 48, 24, 80), (2, 64, 32, 55)]
    alone = {}
    for k, N, M, n in specs:
        sim = hyd.Simulation(_req(k, N, M))
        sim.step(n)
        alone[k] = {f: sim.download(f) for f in ("u", "v", "z", "FS")}
        sim.close()
    budget = 2 * Server.scenario_bytes(32, 64) + 1
    srv = Server(budget, steps_per_round=16)
    ids = {srv.submit(_req(0, 64, 32), 37): 0, srv.submit(_req(1, 48, 24), 80): 1}
    results = {}

    def collect(done):
        for rid in done:
            k = ids[rid]
            results[k] = {f: srv.download(rid, f) for f in ("u", "v", "z", "FS")}
            srv.release(rid)

    collect(srv.round())
    q, a, _ = srv.counts()
    assert a == 2 and q == 0
    ids[srv.submit(_req(2, 64, 32), 55)] = 2  # arrives while two are running
    q, a, _ = srv.counts()
    assert q == 1  # the budget holds two: it waits for a slot
    for _ in range(20):
        collect(srv.round())
        if len(results) == 3:
            break
    assert sorted(results) == [0, 1, 2]
    for k, res in results.items():
        for f, ref in alone[k].items():
            np.testing.assert_array_equal(res[f], ref, err_msg=f"request {k} {f}")
    srv.close()
    # a scenario that does not fit the budget at all is refused at submit
    tiny = Server(1 << 20, steps_per_round=16)
    with pytest.raises(hyd.HydistError, match="BUDGET"):
        tiny.submit(_req(3, 64, 32), 10)
    tiny.close()
