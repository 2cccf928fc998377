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


@pytest.mark.gpu
def test_same_size_requests_step_as_one_batch(hyd):
    """Requests of one mesh size admitted together and advancing alike are
    stepped as one batch (one launch per kernel for all of them: the batch's
    launches are counted once, on its first member); each result agrees with
    its scenario solved alone to rounding (the batched kernels are separately
    compiled variants of the same arithmetic)."""
    import ctypes as C
    from hydist_c_b200 import Server, capi
    n = 40
    alone = {}
    for k in range(3):
        sim = hyd.Simulation(_req(10 + k, 64, 32))
        sim.step(n)
        alone[k] = {f: sim.download(f) for f in ("u", "v", "z", "FS")}
        solo_launches = sim.kernel_launches
        sim.close()
    srv = Server(8 * Server.scenario_bytes(32, 64), steps_per_round=20)
    ids = {srv.submit(_req(10 + k, 64, 32), n): k for k in range(3)}
    results, launches = {}, {}
    lib = capi.load_library()
    for _ in range(10):
        for rid in srv.round():
            k = ids[rid]
            results[k] = {f: srv.download(rid, f) for f in ("u", "v", "z", "FS")}
            v = C.c_int64()
            capi.check(lib, lib.hydist_kernel_launches(C.c_void_p(lib.hydist_server_handle(srv._s, rid)),
                                                       C.byref(v)), "hydist_kernel_launches")
            launches[k] = v.value
        if len(results) == 3:
            break
    assert sorted(results) == [0, 1, 2]
    for k, res in results.items():
        for f, ref in alone[k].items():
            scale = max(float(np.abs(ref).max()), 1e-30)
            d = float(np.abs(res[f] - ref).max()) / scale
            assert d <= 1e-11, (k, f, d)
    # the three requests' steps launched about as many kernels as one
    # request's alone (each handle's own set-up launches aside), not three
    # times as many
    assert sum(launches.values()) < 2 * solo_launches, (launches, solo_launches)
    srv.close()
