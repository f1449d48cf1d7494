"""The no-allocation PCG entry point (pk_pcg_noalloc) against the allocating one (pk_pcg).

pk_pcg_noalloc exists for callers that may not allocate device memory while they
solve -- a game-engine plugin that solves inside its frame loop under a fixed memory
budget, or a host application that routes all device memory through its own pool.
They pass device buffers for the matrix, its transposed index, the rhs, the
preconditioner and the solution; the solver's working vectors live in a fixed array
inside the library.  This test calls it through the C ABI twice in a row (the second
call reuses the array the first one left behind) and compares both results with
pk_pcg on the same system, with the tolerances of the other PCG tests.  At the size
limit itself (32,768 rows, where the FP64 working vectors fill most of the array) it
also checks both calls against the FP64 oracle's PCG.  It also checks that a system
larger than the fixed array is refused without touching the GPU.

This file is collected last so that a failure here cannot hide the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
torch = pytest.importorskip("torch")

MAX_ROWS = 32768


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def random_spd_bsr(n, density, seed):
    rng = np.random.default_rng(seed)
    rows, cols = list(range(n)), list(range(n))
    for r in range(n):
        nb = rng.choice(np.arange(r + 1, n), size=min(n - r - 1, rng.poisson(density)), replace=False) if r + 1 < n else []
        rows += [r] * len(nb)
        cols += list(nb)
    rs, col = po.oracle_build_pattern(n, rows, cols)
    vals = np.zeros((len(col), 3, 3))
    rowsum = np.zeros(n)
    for r in range(n):
        for k in range(rs[r], rs[r + 1]):
            if col[k] != r:
                b = rng.normal(size=(3, 3))
                vals[k] = b
                rowsum[r] += np.abs(b).sum()
                rowsum[col[k]] += np.abs(b).sum()
    for r in range(n):
        a = rng.normal(size=(3, 3))
        vals[rs[r]] = (a @ a.T + (rowsum[r] + 4.0) * np.eye(3)).T
    minv = np.stack([np.linalg.inv(vals[rs[r]].T).T for r in range(n)])
    b = rng.normal(size=(n, 3))
    return rs, col, vals, minv, b


def banded_spd_bsr(n, seed):
    """A sparse SPD system of n rows built without per-row Python loops: every row couples
    to rows r+1, r+7 and r+61 (when they exist), diagonal blocks dominant."""
    rng = np.random.default_rng(seed)
    rows, cols = [np.arange(n)], [np.arange(n)]
    for off in (1, 7, 61):
        r = np.arange(n - off)
        rows.append(r)
        cols.append(r + off)
    rs, col = po.oracle_build_pattern(n, np.concatenate(rows), np.concatenate(cols))
    row_of = np.repeat(np.arange(n), np.diff(rs))
    vals = rng.normal(size=(len(col), 3, 3))
    off_sum = np.abs(vals).sum(axis=(1, 2))
    off_sum[col == row_of] = 0.0
    rowsum = np.bincount(row_of, off_sum, n) + np.bincount(col, off_sum, n)
    diag = rs[:-1]
    a = rng.normal(size=(n, 3, 3))
    d = a @ np.transpose(a, (0, 2, 1)) + (rowsum + 4.0)[:, None, None] * np.eye(3)
    vals[diag] = np.transpose(d, (0, 2, 1))
    minv = np.transpose(np.linalg.inv(d), (0, 2, 1))
    b = rng.normal(size=(n, 3))
    return rs, col, vals, minv, b


def allocating_pcg(prec, rs, col, vals, b, minv, max_it, tol):
    n = len(rs) - 1
    x = np.zeros((n, 3))
    res = L.PkCgResult()
    rc = L.PK.pk_pcg(0, prec, n, _ptr(np.ascontiguousarray(rs, np.int32)), _ptr(np.ascontiguousarray(col, np.int32)),
                     _ptr(np.ascontiguousarray(vals)), _ptr(np.ascontiguousarray(b)), _ptr(np.ascontiguousarray(minv)),
                     n, max_it, tol, _ptr(x), C.byref(res))
    assert rc == 0, L.last_error()
    return x, res


def noalloc_pcg(prec, rs, col, vals, b, minv, max_it, tol):
    """One call of pk_pcg_noalloc with every input and output in device memory."""
    n = len(rs) - 1
    lts = np.zeros(n + 1, np.int32)
    m = L.PK.pk_bsr_transpose_index(n, _ptr(np.ascontiguousarray(rs, np.int32)),
                                    _ptr(np.ascontiguousarray(col, np.int32)), _ptr(lts), None, None)
    ltr = np.zeros(max(m, 1), np.int32)
    ltb = np.zeros(max(m, 1), np.int32)
    L.PK.pk_bsr_transpose_index(n, _ptr(np.ascontiguousarray(rs, np.int32)), _ptr(np.ascontiguousarray(col, np.int32)),
                                _ptr(lts), _ptr(ltr), _ptr(ltb))
    real = torch.float64 if prec == L.PK_PREC_FP64 else torch.float32
    dev = "cuda:0"
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a)).to(device=dev, dtype=dt).contiguous()  # noqa: E731
    d_rs, d_col = t(rs, torch.int32), t(col, torch.int32)
    d_lts, d_ltr, d_ltb = t(lts, torch.int32), t(ltr, torch.int32), t(ltb, torch.int32)
    d_vals, d_b, d_minv = t(vals.reshape(-1), real), t(b.reshape(-1), real), t(minv.reshape(-1), real)
    d_x = torch.full((3 * n,), float("nan"), dtype=real, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    res = L.PkCgResult()
    rc = L.PK.pk_pcg_noalloc(prec, n, d_rs.data_ptr(), d_col.data_ptr(), d_vals.data_ptr(), d_lts.data_ptr(),
                             d_ltr.data_ptr(), d_ltb.data_ptr(), d_b.data_ptr(), d_minv.data_ptr(), max_it, tol,
                             d_x.data_ptr(), C.byref(res), stream)
    assert rc == 0, (L.PK.pk_pcg_noalloc_last_error() or b"").decode()
    torch.cuda.synchronize()
    return d_x.cpu().double().numpy().reshape(n, 3), res


@pytest.mark.parametrize("prec", [L.PK_PREC_FP32, L.PK_PREC_MIXED, L.PK_PREC_FP64])
@pytest.mark.parametrize("n,max_it", [(40, 200), (1500, 300), (1500, 6)])
def test_noalloc_matches_allocating_pcg_twice(prec, n, max_it):
    rs, col, vals, minv, b = random_spd_bsr(n, 4.0, seed=n + max_it)
    x_ref, r_ref = allocating_pcg(prec, rs, col, vals, b, minv, max_it, 1e-6)
    tol = 1e-10 if prec == L.PK_PREC_FP64 else 5e-5
    for _ in range(2):  # the second call starts from what the first one left in the array
        x, res = noalloc_pcg(prec, rs, col, vals, b, minv, max_it, 1e-6)
        assert res.have_solution == 1
        assert abs(res.iterations - r_ref.iterations) <= (1 if prec == L.PK_PREC_FP64 else 2)
        assert res.converged == r_ref.converged
        assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < tol


@pytest.mark.parametrize("prec", [L.PK_PREC_MIXED, L.PK_PREC_FP64])
def test_noalloc_at_the_row_limit_matches_allocating_pcg_and_oracle(prec):
    rs, col, vals, minv, b = banded_spd_bsr(MAX_ROWS, seed=7)
    max_it, tol_cg = 10, 1e-12  # stops at the iteration cap (the oracle needs 12 to converge)
    x_ref, r_ref = allocating_pcg(prec, rs, col, vals, b, minv, max_it, tol_cg)
    x_ora, s_ora = po.oracle_pcg(rs, col, vals, b, minv, max_it, tol_cg, "f64")
    tol = 1e-10 if prec == L.PK_PREC_FP64 else 5e-5
    for _ in range(2):
        x, res = noalloc_pcg(prec, rs, col, vals, b, minv, max_it, tol_cg)
        assert res.have_solution == 1
        assert res.iterations == r_ref.iterations == s_ora["iterations"] == max_it
        assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < tol
        assert np.linalg.norm(x - x_ora) / np.linalg.norm(x_ora) < tol


def test_noalloc_rejects_sizes_beyond_the_fixed_array():
    res = L.PkCgResult()
    dummy = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = L.PK.pk_pcg_noalloc(L.PK_PREC_FP32, MAX_ROWS + 1, dummy, dummy, dummy, dummy, dummy, dummy, dummy, dummy,
                             10, 1e-6, dummy, C.byref(res), None)
    assert rc == -5  # PK_ERR_UNSUPPORTED
    assert b"exceed" in (L.PK.pk_pcg_noalloc_last_error() or b"")
