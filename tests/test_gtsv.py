"""The batched tridiagonal solvers (hydist_gtsv_batched): every solver and
the autotuned choice against the oracle's FP64 Thomas on the same packed
batch, with the edge cases of the packed format (empty, 1-, 2- and 3-row
systems, lengths at every band boundary, systems longer than a CTA's shared
memory), in FP64 and FP32."""
import ctypes as C

import numpy as np
import pytest

from hydist_c_b200 import capi

# band boundaries and their neighbours, plus systems beyond the CTA solver
EDGE_LENGTHS = [0, 1, 2, 3, 4, 31, 32, 33, 127, 128, 129, 511, 512, 513, 2047, 2048, 2049,
                4095, 4096, 4097, 6144, 6145, 9000]
ALGOS = [capi.GTSV_AUTO, capi.GTSV_THOMAS, capi.GTSV_PARTITION, capi.GTSV_WARP,
         capi.GTSV_PARTITION_512, capi.GTSV_PARTITION_128]


def _batch(seed, nsys=600):
    from hydist_c_b200 import scenario as S
    rng = np.random.default_rng(seed)
    lens = np.concatenate([EDGE_LENGTHS, np.exp(rng.uniform(0, np.log(4096), nsys)).astype(int)])
    rng.shuffle(lens)
    return S.tridiag_batch(lengths=lens, seed=seed)


def test_band_bounds_exported(hyd):
    lib = hyd.library()
    hi = (C.c_int32 * capi.GTSV_BANDS)()
    assert lib.hydist_gtsv_band_bounds(hi) == 0
    hi = list(hi)
    assert hi == sorted(hi) and hi[0] == 32 and hi[-1] == 2**31 - 1


def test_oracle_batched_thomas_matches_dense_solve(oracle_mod):
    a, d, c, b, off, ln = _batch(5, nsys=20)
    x = oracle_mod.thomas_batched(a, d, c, b, off, ln)
    for s in range(len(ln)):
        n, o = ln[s], off[s]
        if n == 0 or n > 600:
            continue
        Am = np.diag(d[o:o + n]) + np.diag(a[o + 1:o + n], -1) + np.diag(c[o:o + n - 1], 1)
        np.testing.assert_allclose(x[o:o + n], np.linalg.solve(Am, b[o:o + n]), rtol=1e-10, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_gtsv_matches_oracle(hyd, oracle_mod, algo, dtype):
    import torch
    a, d, c, b, off, ln = _batch(11)
    ref = oracle_mod.thomas_batched(a, d, c, b, off, ln)
    dev = torch.device("cuda:0")
    tdt = getattr(torch, dtype)
    t = [torch.from_numpy(v).to(dev, tdt) for v in (a, d, c, b)]
    x = torch.full_like(t[1], float("nan"))
    hyd.gtsv_batched(*t, torch.from_numpy(off), torch.from_numpy(ln), algo=algo, x=x)
    torch.cuda.synchronize()
    xs = x.double().cpu().numpy()
    assert np.isfinite(xs).all()
    scale = np.maximum(np.abs(ref), 1.0)
    err = np.max(np.abs(xs - ref) / scale)
    # FP64: the partition method and Thomas differ by rounding only;
    # FP32: single-precision solves of systems with condition number O(10)
    assert err <= (1e-11 if dtype == "float64" else 2e-5), err


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [0, 1])
def test_autotune_then_auto(hyd, oracle_mod, dtype):
    import torch
    lib = hyd.library()
    table = (C.c_int32 * capi.GTSV_BANDS)()
    st = lib.hydist_gtsv_autotune(dtype, None, table)
    capi.check(lib, st, "hydist_gtsv_autotune")
    table = list(table)
    assert all(v in (capi.GTSV_THOMAS, capi.GTSV_PARTITION, capi.GTSV_WARP,
                    capi.GTSV_PARTITION_512, capi.GTSV_PARTITION_128) for v in table), table
    assert table[-1] == capi.GTSV_THOMAS  # the open band fits no shared memory
    a, d, c, b, off, ln = _batch(13, nsys=300)
    ref = oracle_mod.thomas_batched(a, d, c, b, off, ln)
    tdt = torch.float64 if dtype == 0 else torch.float32
    t = [torch.from_numpy(v).to("cuda", tdt) for v in (a, d, c, b)]
    for _ in range(2):  # two consecutive calls reuse the library's scratch
        x = hyd.gtsv_batched(*t, torch.from_numpy(off), torch.from_numpy(ln), algo=capi.GTSV_AUTO)
        torch.cuda.synchronize()
        err = np.max(np.abs(x.double().cpu().numpy() - ref) / np.maximum(np.abs(ref), 1.0))
        assert err <= (1e-11 if dtype == 0 else 2e-5), err


def _non_dominant_batch(seed, nsys=200, max_len=300):
    """Systems that are not diagonally dominant: half of them interleave
    continuity-like rows (a, 1, c) with |a|, |c| ~ U(0.8, 1.2) and weak
    momentum rows, as the ADI sweeps' interleaved (z, u) systems do at large
    time steps; the other half are random with a zero diagonal every third
    row (no Thomas step can take those)."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(2, max_len, nsys).astype(np.int32)
    off = np.zeros(nsys, np.int32)
    off[1:] = np.cumsum(lens[:-1])
    n = int(lens.sum())
    a = np.zeros(n)
    d = np.zeros(n)
    c = np.zeros(n)
    b = rng.standard_normal(n)
    for s in range(nsys):
        o, m = off[s], lens[s]
        q = np.arange(m)
        if s % 2 == 0:
            cont = q % 2 == 0
            a[o:o + m] = np.where(cont, rng.choice([-1, 1], m) * rng.uniform(0.8, 1.2, m),
                                  rng.uniform(-1, 1, m))
            c[o:o + m] = np.where(cont, rng.choice([-1, 1], m) * rng.uniform(0.8, 1.2, m),
                                  rng.uniform(-1, 1, m))
            d[o:o + m] = np.where(cont, 1.0, rng.uniform(-0.3, 0.3, m))
        else:
            a[o:o + m] = rng.uniform(-1, 1, m)
            c[o:o + m] = rng.uniform(-1, 1, m)
            d[o:o + m] = np.where(q % 3 == 0, 0.0, rng.uniform(-1, 1, m))
    return a, d, c, b, off, lens


def _dense(a, d, c, o, m):
    A = np.diag(d[o:o + m])
    if m > 1:
        A += np.diag(a[o + 1:o + m], -1) + np.diag(c[o:o + m - 1], 1)
    return A


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_pivot_solves_non_dominant_systems(hyd, dtype):
    """HYDIST_GTSV_PIVOT (diagonal pivoting) on systems the non-pivoting
    solvers cannot take: its backward error is at rounding level, and where
    the system is well conditioned its solution agrees with a dense LU solve
    with partial pivoting (numpy)."""
    import torch
    a, d, c, b, off, ln = _non_dominant_batch(21)
    tdt = getattr(torch, dtype)
    t = [torch.from_numpy(v).to("cuda", tdt) for v in (a, d, c, b)]
    x = hyd.gtsv_batched(*t, torch.from_numpy(off), torch.from_numpy(ln), algo=capi.GTSV_PIVOT)
    torch.cuda.synchronize()
    xs = x.double().cpu().numpy()
    assert np.isfinite(xs).all()
    host = [v.double().cpu().numpy() for v in t]  # the systems as the device saw them
    eps = 1e-13 if dtype == "float64" else 2e-5
    checked = 0
    for s in range(len(ln)):
        o, m = off[s], ln[s]
        A = _dense(host[0], host[1], host[2], o, m)
        xx = xs[o:o + m]
        bb = host[3][o:o + m]
        back = np.abs(A @ xx - bb).max() / (np.abs(A).sum(1).max() * np.abs(xx).max() + np.abs(bb).max())
        assert back <= eps * 10, (s, back)
        if dtype == "float64" and np.linalg.cond(A) < 1e6:
            ref = np.linalg.solve(A, bb)
            assert np.abs(xx - ref).max() <= 1e-8 * max(1.0, np.abs(ref).max()), s
            checked += 1
    assert dtype != "float64" or checked > len(ln) // 2


@pytest.mark.gpu
def test_thomas_breaks_where_pivot_does_not(hyd):
    """A zero leading diagonal: Thomas divides by it, the pivoting solver
    takes a 2x2 block."""
    import torch
    a = np.array([0.0, 1.0, 0.5])
    d = np.array([0.0, 2.0, 1.0])
    c = np.array([1.0, 0.5, 0.0])
    b = np.array([1.0, 2.0, 3.0])
    off, ln = np.array([0], np.int32), np.array([3], np.int32)
    t = [torch.from_numpy(v).cuda() for v in (a, d, c, b)]
    xt = hyd.gtsv_batched(*t, torch.from_numpy(off), torch.from_numpy(ln), algo=capi.GTSV_THOMAS)
    xp = hyd.gtsv_batched(*t, torch.from_numpy(off), torch.from_numpy(ln), algo=capi.GTSV_PIVOT)
    torch.cuda.synchronize()
    ref = np.linalg.solve(_dense(a, d, c, 0, 3), b)
    assert not np.isfinite(xt.cpu().numpy()).all()
    np.testing.assert_allclose(xp.cpu().numpy(), ref, rtol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("algo", [capi.GTSV_AUTO, capi.GTSV_THOMAS, capi.GTSV_PIVOT])
def test_fp32_refined_solve_reaches_fp64_accuracy(hyd, oracle_mod, algo):
    """hydist_gtsv_batched_refine: FP64 systems solved in FP32, one FP64
    residual, the correction in FP32: within 1e-12 of the FP64 oracle on the
    diagonally dominant batch (plain FP32 is at about 1e-6)."""
    import torch
    a, d, c, b, off, ln = _batch(17, nsys=600)
    ref = oracle_mod.thomas_batched(a, d, c, b, off, ln)
    t = [torch.from_numpy(v).cuda() for v in (a, d, c, b)]
    o, n = torch.from_numpy(off), torch.from_numpy(ln)
    for _ in range(2):  # the library's FP32 scratch is reused
        x = hyd.gtsv_batched(*t, o, n, algo=algo, refine=True)
        torch.cuda.synchronize()
        err = np.max(np.abs(x.cpu().numpy() - ref) / np.maximum(np.abs(ref), 1.0))
        assert err <= 1e-12, err
    x32 = hyd.gtsv_batched(*[v.float() for v in t], o, n, algo=algo)
    torch.cuda.synchronize()
    err32 = np.max(np.abs(x32.double().cpu().numpy() - ref) / np.maximum(np.abs(ref), 1.0))
    assert err32 > 1e-9  # what the refinement buys
