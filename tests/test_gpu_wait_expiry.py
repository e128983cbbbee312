"""Failure detection of the factorisation's device-wide waits, without a GPU
fault: the host drops one update task from the task list, so one wait can
never be satisfied; the wait gives up after a short poll limit, the launch
reports info = -1 with the barrier error bit, and the same context then
factors a matrix normally (pbg_selftest_wait_expiry).  A normal
factorisation through the public entry point follows as well."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PBG_DEV_ERR_BARRIER = 2


def test_wait_gives_up_and_the_context_stays_usable():
    import torch
    from pybrown_b200 import _lib
    info = ctypes.c_int(0)
    err = ctypes.c_uint(0)
    rc = _lib.lib.pbg_selftest_wait_expiry(4096, ctypes.byref(info), ctypes.byref(err))
    assert rc == 0, _lib.last_error()
    assert info.value == -1
    assert err.value & PBG_DEV_ERR_BARRIER
    rng = np.random.default_rng(0)
    n = 300
    X = rng.normal(size=(n, n))
    A = X @ X.T + n * np.eye(n)
    ld = 320
    M = torch.zeros((ld, ld), dtype=torch.float64, device="cuda")
    M[:n, :n] = torch.tensor(A, device="cuda")
    dinfo = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("pbg_dev_cholesky", M.data_ptr(), n, ld, 0, dinfo.data_ptr(), None)
    torch.cuda.synchronize()
    assert int(dinfo.item()) == 0
    L = np.tril(M[:n, :n].cpu().numpy())
    assert np.max(np.abs(L @ L.T - A)) / np.max(np.abs(A)) < 1e-12
