"""Checkpoint / resume (hydist_checkpoint_*): stop after some steps, save,
restore into a fresh handle of the same scenario, step on -- bit-identical
to the uninterrupted run, through the sediment start and wetting/drying. A
checkpoint of another mesh size or a foreign file is refused."""
import numpy as np
import pytest


def _bundle(N=64, M=32):
    from hydist_c_b200 import scenario as S
    return S.make_channel(N=N, M=M, seed=20268000, dx=10.0, dt=2.0, hours=1.0,
                          sediment=True, sediment_start=30.0)


@pytest.mark.gpu
def test_resume_is_bit_identical(hyd, tmp_path):
    ref = hyd.Simulation(_bundle())
    ref.step(40)
    want = {f: ref.download(f) for f in ("u", "v", "z", "FS", "khouot", "H_moi")}
    ref.close()
    a = hyd.Simulation(_bundle())
    a.step(17)
    ck = tmp_path / "state.ck"
    a.save(ck)
    a.close()
    b = hyd.Simulation(_bundle())
    b.load(ck)
    assert b.t == pytest.approx(34.0)
    b.step(23)
    for f, w in want.items():
        np.testing.assert_array_equal(b.download(f), w, err_msg=f)
    with pytest.raises(hyd.HydistError, match="mesh size"):
        c = hyd.Simulation(_bundle(N=48, M=24))
        c.load(ck)
    bad = tmp_path / "bad.ck"
    bad.write_bytes(b"not a checkpoint" * 8)
    with pytest.raises(hyd.HydistError, match="format"):
        b.load(bad)
    # a truncated file (valid header, body cut short) and one with trailing
    # bytes are refused before anything is uploaded: the handle's state and
    # time stay as they were
    raw = ck.read_bytes()
    before = {f: b.download(f) for f in ("u", "z", "khouot")}
    t_before = b.t
    for name, data in (("cut.ck", raw[:len(raw) - 1000]), ("long.ck", raw + b"\0" * 8)):
        p = tmp_path / name
        p.write_bytes(data)
        with pytest.raises(hyd.HydistError, match="size"):
            b.load(p)
        assert b.t == t_before
        for f, w in before.items():
            np.testing.assert_array_equal(b.download(f), w, err_msg=f)
    b.close()
