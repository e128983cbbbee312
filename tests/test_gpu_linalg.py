"""Cholesky factor and SPD inverse kernels against NumPy (LAPACK) in FP64,
and the mixed-precision factor against the FP64 one."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _spd(n, seed, cond=1e3):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    ev = np.geomspace(1.0, cond, n)
    A = (Q * ev) @ Q.T
    return (A + A.T) / 2


def _run(fn, A, n, prec=0):
    import torch
    from pybrown_b200 import _lib
    ld = (n + 63) // 64 * 64
    dtype = torch.float64 if prec == 0 else torch.float32
    buf = torch.zeros((ld, ld), dtype=dtype, device="cuda")
    buf[:n, :n] = torch.tensor(A, dtype=dtype)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    if fn == "chol":
        _lib.call("pbg_dev_cholesky", buf.data_ptr(), n, ld, prec, info.data_ptr(), None)
    else:
        _lib.call("pbg_dev_spd_inverse", buf.data_ptr(), n, ld, info.data_ptr(), None)
    torch.cuda.synchronize()
    return buf[:n, :n].double().cpu().numpy(), int(info.item())


@pytest.mark.parametrize("n", [3, 64, 81, 192, 513, 1536])
def test_cholesky_fp64(n):
    A = _spd(n, n)
    L, info = _run("chol", A, n)
    assert info == 0
    ref = np.linalg.cholesky(A)
    # like LAPACK dpotrf, only the lower triangle is defined
    assert rel_err(np.tril(L), ref) <= 1e-12


@pytest.mark.parametrize("n", [3, 64, 81, 130, 192, 1000, 1536])
def test_spd_inverse_fp64(n):
    """inv(A) = X^T X with X = inv(L) formed inside the factorisation's task
    list (one tile row for n <= 64: no inverse tasks; up to 24 x 24 tiles)."""
    A = _spd(n, 100 + n)
    X, info = _run("inv", A, n)
    assert info == 0
    assert rel_err(X, np.linalg.inv(A)) <= 1e-11


def test_cholesky_not_spd_reports_pivot():
    n = 130
    A = _spd(n, 5)
    A[70, 70] = -1.0
    _, info = _run("chol", A, n)
    assert info > 0


# prec 1: FP32 chain (FP32 diagonal tiles); prec 2: FP64 diagonal tiles
@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("n", [3, 64, 192, 577, 768, 3072])
def test_cholesky_mixed(n, prec):
    A = _spd(n, 7, cond=1e2)
    L, info = _run("chol", A, n, prec=prec)
    assert info == 0
    assert rel_err(np.tril(L), np.linalg.cholesky(A)) <= 5e-5


@pytest.mark.parametrize("prec", [1, 2])
def test_cholesky_mixed_not_spd_reports_pivot(prec):
    n = 200
    A = _spd(n, 5)
    A[140, 140] = -1.0
    _, info = _run("chol", A, n, prec=prec)
    assert info > 0
