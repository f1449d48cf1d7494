"""Kernel-level parity through the device C ABI (include/pkcuda.h) against the oracle.

* pk_bsr_multiply: the reference's SpMV known answers and random symmetric upper BSRs.
* pk_pcg: the reference's PCG known answers, failure semantics and random SPD systems,
  in FP32, mixed and FP64.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def gpu_multiply(row_start, col, values, x, precision):
    n = len(row_start) - 1
    rs = np.ascontiguousarray(row_start, np.int32)
    cl = np.ascontiguousarray(col, np.int32)
    vv = np.ascontiguousarray(values, np.float64)
    xx = np.ascontiguousarray(x, np.float64)
    y = np.zeros((n, 3))
    rc = L.PK.pk_bsr_multiply(0, precision, n, _ptr(rs), _ptr(cl), _ptr(vv), _ptr(xx), _ptr(y))
    assert rc == 0, L.last_error()
    return y


def gpu_pcg(row_start, col, values, b, minv, max_it, tol, precision):
    n = len(row_start) - 1
    rs = np.ascontiguousarray(row_start, np.int32)
    cl = np.ascontiguousarray(col, np.int32)
    vv = np.ascontiguousarray(values, np.float64)
    bb = np.ascontiguousarray(b, np.float64)
    mm = None if minv is None else np.ascontiguousarray(minv, np.float64)
    x = np.zeros((max(n, 1), 3))
    res = L.PkCgResult()
    rc = L.PK.pk_pcg(0, precision, n, _ptr(rs), _ptr(cl), _ptr(vv), _ptr(bb), _ptr(mm),
                     0 if mm is None else len(mm), max_it, tol, _ptr(x), C.byref(res))
    assert rc == 0, L.last_error()
    return (x[:n] if res.have_solution else None), res


def random_spd_bsr(n, density, seed, dominance=4.0):
    """Random symmetric positive definite BSR in canonical upper storage."""
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for r in range(n):
        rows.append(r)
        cols.append(r)
        for c in range(r + 1, n):
            if rng.random() < density:
                rows.append(r)
                cols.append(c)
    rs, col = po.oracle_build_pattern(n, rows, cols)
    nnz = len(col)
    vals = np.zeros((nnz, 3, 3))
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
        d = a @ a.T + (rowsum[r] + dominance) * np.eye(3)
        vals[rs[r]] = d.T
    return rs, col, vals


def block_jacobi(rs, col, vals):
    n = len(rs) - 1
    return np.stack([np.linalg.inv(vals[rs[r]].T).T for r in range(n)])


PRECISIONS = [(L.PK_PREC_FP32, "f32", 1e-5), (L.PK_PREC_MIXED, "f32", 1e-5), (L.PK_PREC_FP64, "f64", 1e-12)]


def test_device_present():
    assert L.device_count() >= 1


@pytest.mark.parametrize("prec,_o,_t", PRECISIONS)
def test_spmv_known_answers(golden_dir, prec, _o, _t):
    k = np.load(f"{golden_dir}/kat_bsr.npz")
    for c in ("a", "b"):
        y = gpu_multiply(k[f"{c}_row_start"], k[f"{c}_col"], k[f"{c}_values"], k[f"{c}_x"], prec)
        np.testing.assert_array_equal(y, k[f"{c}_y"])


@pytest.mark.parametrize("prec,oprec,tol", PRECISIONS)
@pytest.mark.parametrize("n,density", [(1, 0.0), (7, 0.5), (64, 0.1), (700, 0.01)])
def test_spmv_random(prec, oprec, tol, n, density):
    rs, col, vals = random_spd_bsr(n, density, seed=n)
    x = np.random.default_rng(1).normal(size=(n, 3))
    y = gpu_multiply(rs, col, vals, x, prec)
    ref = po.oracle_bsr_multiply(rs, col, vals, x, "f64")
    scale = np.abs(vals).max() * np.abs(x).max() * 20
    np.testing.assert_allclose(y, ref, rtol=0, atol=tol * scale)


@pytest.mark.parametrize("prec,_o,_t", PRECISIONS)
@pytest.mark.parametrize("case", ["c", "d", "e"])
def test_pcg_known_answers(golden_dir, prec, _o, _t, case):
    k = np.load(f"{golden_dir}/kat_bsr.npz")
    n = len(k[f"{case}_row_start"]) - 1
    minv = k[f"{case}_minv"] if f"{case}_minv" in k else np.stack([np.eye(3)] * n)
    max_it = {"c": 16, "d": 32, "e": 8}[case]
    x, res = gpu_pcg(k[f"{case}_row_start"], k[f"{case}_col"], k[f"{case}_values"], k[f"{case}_b"], minv, max_it,
                     1e-6, prec)
    assert x is not None
    np.testing.assert_allclose(x, k[f"{case}_x"], atol=1e-4)
    assert res.converged == int(k[f"{case}_conv"])
    if case == "e":
        # d.q <= 0 on the first iteration: x stays zero, zero completed iterations.
        np.testing.assert_array_equal(x, 0.0)
        assert res.iterations == 0


@pytest.mark.parametrize("prec", [L.PK_PREC_FP32, L.PK_PREC_MIXED, L.PK_PREC_FP64])
def test_pcg_invalid_settings_and_rhs(prec):
    rs, col = np.array([0, 1], np.int32), np.array([0], np.int32)
    vals = np.eye(3)[None]
    b = np.array([[1.0, 0, 0]])
    for max_it, tol in ((0, 1e-6), (8, 0.0), (8, np.inf)):
        x, res = gpu_pcg(rs, col, vals, b, np.eye(3)[None], max_it, tol, prec)
        assert x is None and res.converged == 0
    x, res = gpu_pcg(rs, col, vals, np.array([[np.nan, 0, 0]]), np.eye(3)[None], 8, 1e-6, prec)
    assert x is None and res.converged == 0
    # Preconditioner of the wrong size: x = 0, not converged (ApplyPreconditioner fails).
    x, res = gpu_pcg(rs, col, vals, b, None, 8, 1e-6, prec)
    np.testing.assert_array_equal(x, 0.0)
    assert res.converged == 0


@pytest.mark.parametrize("prec,oprec,tol", PRECISIONS)
@pytest.mark.parametrize("n,max_it", [(50, 200), (900, 400), (900, 7)])
def test_pcg_random_spd(prec, oprec, tol, n, max_it):
    rs, col, vals = random_spd_bsr(n, 6.0 / n, seed=3 + n)
    minv = block_jacobi(rs, col, vals)
    b = np.random.default_rng(5).normal(size=(n, 3))
    x, res = gpu_pcg(rs, col, vals, b, minv, max_it, 1e-6, prec)
    xo, ro = po.oracle_pcg(rs, col, vals, b, minv, max_it, 1e-6, "f64")
    assert x is not None
    assert abs(res.iterations - ro["iterations"]) <= (1 if prec == L.PK_PREC_FP64 else 2)
    rel = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    assert rel < (1e-10 if prec == L.PK_PREC_FP64 else 5e-5), rel
    if max_it >= 200:
        assert res.converged == 1
