"""hydist_gtsv_batched_noalloc: the allocation-free batched Thomas solve.

Its results are compared with the FP64 CPU oracle's batched Thomas and with
hydist_gtsv_batched (the allocating entry point, autotuned solver choice) on
two consecutive calls; the second call must leave the device's free memory
unchanged. The file name sorts last so that the GPU
tests also run it after every other test has used the device.
"""
import ctypes as C

import numpy as np
import pytest

MAX_ROWS = 1 << 20


def _packed_batch(seed, nsys, max_len):
    """Diagonally dominant systems with ragged lengths (0, 1 and 2 included)."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(1, max_len + 1, size=nsys).astype(np.int32)
    lengths[:3] = [0, 1, 2]
    offsets = np.zeros(nsys, np.int32)
    offsets[1:] = np.cumsum(lengths[:-1])
    rows = int(lengths.sum())
    a = rng.uniform(-1, 1, rows)
    c = rng.uniform(-1, 1, rows)
    d = np.abs(a) + np.abs(c) + rng.uniform(0.1, 1.0, rows)
    b = rng.standard_normal(rows)
    return a, d, c, b, offsets, lengths, rows


def _call(lib, t, offs, lens, x, rows, stream):
    dl, d, du, b = t
    dt = 0 if d.dtype.itemsize == 8 else 1
    return lib.hydist_gtsv_batched_noalloc(dl.data_ptr(), d.data_ptr(), du.data_ptr(), b.data_ptr(),
                                           x.data_ptr(), offs.data_ptr(), lens.data_ptr(),
                                           int(offs.numel()), int(rows), dt, C.c_void_p(stream))


def test_noalloc_rejects_rows_beyond_limit(hyd):
    from hydist_c_b200 import capi
    lib = hyd.library()
    buf = np.zeros(4)
    p = buf.ctypes.data
    st = lib.hydist_gtsv_batched_noalloc(p, p, p, p, p, p, p, 1, MAX_ROWS + 1, 0, None)
    assert capi.STATUS_NAMES[st] == "HYDIST_ERR_BUDGET"
    assert b"HYDIST_GTSV_NOALLOC_MAX_ROWS" in lib.hydist_last_error()
    for st in (lib.hydist_gtsv_batched_noalloc(None, p, p, p, p, p, p, 1, 4, 0, None),
               lib.hydist_gtsv_batched_noalloc(p, p, p, p, p, p, p, 1, 4, 7, None)):
        assert capi.STATUS_NAMES[st] == "HYDIST_ERR_ARG"


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,rtol", [("float64", 1e-12), ("float32", 2e-5)])
def test_noalloc_matches_oracle_and_gtsv_batched(hyd, oracle_mod, dtype, rtol):
    import torch
    from hydist_c_b200 import capi
    lib = hyd.library()
    dev = torch.device("cuda:0")
    tdt = getattr(torch, dtype)
    a, d, c, b, offs, lens, rows = _packed_batch(7, 3000, 300)
    assert rows <= MAX_ROWS
    # the oracle solves the systems as the device sees them (rounded to the
    # call's type first)
    t = [torch.from_numpy(v).to(dev, tdt).contiguous() for v in (a, d, c, b)]
    host = [v.double().cpu().numpy() for v in t]
    ref = torch.from_numpy(oracle_mod.thomas_batched(*host, offs, lens)).to(dev, tdt)
    o = torch.from_numpy(offs).to(dev)
    n = torch.from_numpy(lens).to(dev)
    alloc = hyd.gtsv_batched(*t, o, n, algo=capi.GTSV_AUTO)
    torch.cuda.synchronize()
    scale0 = torch.clamp(ref.abs(), min=1.0)
    assert ((alloc - ref).abs() / scale0).max().item() <= rtol
    stream = torch.cuda.current_stream(dev).cuda_stream
    outs = [torch.zeros(rows, dtype=tdt, device=dev) for _ in range(2)]
    scale = torch.clamp(ref.abs(), min=1.0)
    free = []
    for x in outs:
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info(dev)[0]
        st = _call(lib, t, o, n, x, rows, stream)
        capi.check(lib, st, "hydist_gtsv_batched_noalloc")
        torch.cuda.synchronize()
        free.append((before, torch.cuda.mem_get_info(dev)[0]))
        err = ((x - ref).abs() / scale).max().item()
        assert err <= rtol, err
        # both are within rtol of the FP64 solution
        err = ((x - alloc).abs() / scale).max().item()
        assert err <= 2 * rtol, err
    # the second call allocated nothing on the device (the first one may
    # load the library's kernels and their fixed scratch)
    assert free[1][0] == free[1][1]
    x = outs[1]
    # residual of the solution itself (first rows of each system ignore dl,
    # last rows ignore du)
    xs = x.double().cpu().numpy()
    for s in range(3, 60):
        i0, m = offs[s], lens[s]
        A, D, Cc, B, X = a[i0:i0 + m], d[i0:i0 + m], c[i0:i0 + m], b[i0:i0 + m], xs[i0:i0 + m]
        r = D * X - B
        r[1:] += A[1:] * X[:-1]
        r[:-1] += Cc[:-1] * X[1:]
        assert np.abs(r).max() <= (1e-10 if dtype == "float64" else 1e-3)


@pytest.mark.gpu
def test_noalloc_leaves_systems_outside_rows_unsolved(hyd, oracle_mod):
    import torch
    from hydist_c_b200 import capi
    lib = hyd.library()
    dev = torch.device("cuda:0")
    a, d, c, b, offs, lens, rows = _packed_batch(11, 64, 40)
    t = [torch.from_numpy(v).to(dev).contiguous() for v in (a, d, c, b)]
    o = torch.from_numpy(offs).to(dev)
    n = torch.from_numpy(lens).to(dev)
    ref = torch.from_numpy(oracle_mod.thomas_batched(a, d, c, b, offs, lens)).to(dev)
    cut = int(offs[-1]) + 1  # the last system crosses the declared rows
    x = torch.zeros(rows, dtype=torch.float64, device=dev)
    st = _call(lib, t, o, n, x, cut, torch.cuda.current_stream(dev).cuda_stream)
    capi.check(lib, st, "hydist_gtsv_batched_noalloc")
    torch.cuda.synchronize()
    last = int(offs[-1])
    assert torch.all(x[last:] == 0)
    assert torch.allclose(x[:last], ref[:last], rtol=1e-12, atol=1e-12)
