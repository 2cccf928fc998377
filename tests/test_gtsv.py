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
