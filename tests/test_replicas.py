"""The N > 1 path on CPU: world-size-2 process groups over gloo.

bench.py --gpus N runs one replica per rank (hydist_c_b200/replicas.py):
rank r solves its own seeded scenario, and the only collectives are the
barrier and the max / sum over ranks of the timed region. Here each rank
advances its replica with the oracle (the CPU restatement; no GPU), and the
parent checks that rank r's result is the solo result for rank r's seed,
that the replicas differ, and that the reductions are right. A second test
has one rank leave before the barrier: the other must end with an error
within the process group's timeout, not hang.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica_bundle(rank):
    from hydist_c_b200 import scenario as S
    from hydist_c_b200.replicas import replica_seed
    return S.make_channel(N=40, M=20, seed=replica_seed(1234, rank), dx=10.0, dt=2.0, hours=1.0)


def _replica_checksum(rank, steps=3):
    from oracle import oracle as O
    o = O.OracleSim(_replica_bundle(rank), nthreads=1)
    o.step(steps)
    z = o.get("z")
    return float(np.sum(np.abs(z))), float(np.sum(z * z))


def _worker(rank, ws, port, out_dir, mode):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    from hydist_c_b200 import replicas as R
    r, _, n = R.init("gloo", timeout_s=10)
    res = {"rank": r}
    try:
        if mode == "leave" and r == 1:
            os._exit(0)  # this rank is gone before the barrier
        R.barrier(n)
        if mode == "run":
            res["checksum"] = _replica_checksum(r)
            res["max"] = R.max_over_ranks(10.0 + r, n)
            res["sum"] = R.sum_over_ranks(1.0, n)
            R.barrier(n)
            R.finish(n)
        res["ok"] = True
    except Exception as e:  # the rank left behind by a peer that exited
        res["error"] = type(e).__name__
    np.save(os.path.join(out_dir, f"rank{r}.npy"), np.array([repr(res)]))


def _spawn(mode, tmp_path, ws=2):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, ws, port, str(tmp_path), mode)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert not p.is_alive(), "a rank hung"
    out = {}
    for r in range(ws):
        f = tmp_path / f"rank{r}.npy"
        if f.exists():
            out[r] = eval(str(np.load(f)[0]))
    return out


def test_two_replicas_over_gloo(tmp_path):
    out = _spawn("run", tmp_path)
    assert sorted(out) == [0, 1]
    for r in (0, 1):
        assert out[r]["ok"]
        assert out[r]["max"] == 11.0
        assert out[r]["sum"] == 2.0
        assert out[r]["checksum"] == pytest.approx(_replica_checksum(r), rel=0, abs=0)
    assert out[0]["checksum"] != out[1]["checksum"]


def test_rank_left_behind_errors_instead_of_hanging(tmp_path):
    out = _spawn("leave", tmp_path)
    assert 1 not in out
    assert "error" in out[0], out[0]
