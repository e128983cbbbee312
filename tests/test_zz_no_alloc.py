"""The allocation-free Smith-Ewald entry point (pbg_dev_smith_matrix_noalloc).

It exists for callers that cannot allocate device memory: an application
whose memory manager has already taken all of it, or a step loop that must
not run into the device-wide synchronisation of cudaMalloc/cudaFree.  Its
scratch is one fixed array inside the library, shared by every call.

Checked through the C ABI against the allocating entry point
(pbg_dev_smith_matrix) on the same inputs, on two calls in a row (the second
call finds the first call's data in the shared array), at the tolerance of
the other FP64 tensor tests.  This file is collected last on purpose.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _config(seed, n, L, a_lo, a_hi):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 3))
    radii = np.zeros(n)
    k = 0
    while k < n:
        a = rng.uniform(a_lo, a_hi)
        p = rng.uniform(-L / 2, L / 2, size=3)
        if k:
            d = pos[:k] - p
            d -= L * np.round(d / L)
            if np.any(np.sqrt((d * d).sum(1)) <= radii[:k] + a):
                continue
        pos[k], radii[k] = p, a
        k += 1
    return pos, radii


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    from pybrown_b200 import _lib
    n_beads, L = 300, 900.0
    alpha, m_max, n_max = math.sqrt(math.pi), 2, 4
    n = 3 * n_beads
    cases = [_config(11, n_beads, L, 10.0, 40.0), _config(12, n_beads, L, 10.0, 40.0)]
    # FP64 at the FP64 tensor tolerance; the mixed (FP32) output at the FP32
    # level the mixed-precision tests use
    for prec, dtype, tol in ((0, torch.float64, TOL), (1, torch.float32, 1e-6)):
        for pos, radii in cases:  # two calls in a row, different inputs
            dpos = torch.tensor(pos.reshape(-1), dtype=torch.float64, device="cuda")
            drad = torch.tensor(radii, dtype=torch.float64, device="cuda")
            ref = torch.zeros(n * n, dtype=dtype, device="cuda")
            out = torch.full((n * n,), float("nan"), dtype=dtype, device="cuda")
            _lib.call("pbg_dev_smith_matrix", dpos.data_ptr(), drad.data_ptr(), n_beads, L, alpha, m_max, n_max,
                      1.0, prec, ref.data_ptr(), n, None)
            _lib.call("pbg_dev_smith_matrix_noalloc", dpos.data_ptr(), drad.data_ptr(), n_beads, L, alpha, m_max,
                      n_max, 1.0, prec, out.data_ptr(), n, None)
            torch.cuda.synchronize()
            r = ref.double().cpu().numpy()
            o = out.double().cpu().numpy()
            assert np.all(np.isfinite(o))
            assert _rel(o, r) <= tol, (prec, _rel(o, r))


def test_noalloc_rejects_oversized_input():
    import torch
    from pybrown_b200 import _lib
    n_beads = 5000  # 5000 beads x 64 half-vectors x 16 bytes > 4 MiB of phase tables
    pos = torch.zeros(3 * n_beads, dtype=torch.float64, device="cuda")
    rad = torch.ones(n_beads, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _lib.lib.pbg_dev_smith_matrix_noalloc(pos.data_ptr(), rad.data_ptr(), n_beads, 1e4, math.sqrt(math.pi),
                                               2, 4, 1.0, 0, out.data_ptr(), 3 * n_beads, None)
    assert rc == -2  # PBG_ERR_ARG
    assert "fixed scratch" in _lib.last_error()
