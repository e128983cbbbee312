"""The allocation-free Smith-Ewald entry point (pbg_dev_smith_matrix_noalloc).

It exists for callers that cannot allocate device memory: an application
whose memory manager has already taken all of it, or a step loop that must
not run into the device-wide synchronisation of cudaMalloc/cudaFree.  Its
scratch is one fixed array inside the library, shared by every call.

Checked through the C ABI against the allocating entry point
(pbg_dev_smith_matrix) on the same inputs, on calls in a row whose lattice
sizes differ (a larger call, then a smaller one, then a larger one again), so
stale tables left in the shared array by the previous call would show.  Both
entry points run the same kernels on the same tables, so the outputs must be
identical bit for bit.  This file is collected last on purpose.
"""
import math

import numpy as np
import pytest

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


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_in_a_row():
    import torch
    from pybrown_b200 import _lib
    n_beads, L = 300, 900.0
    alpha = math.sqrt(math.pi)
    n = 3 * n_beads
    # (config seed, ewald_real, ewald_imag): larger, smaller, larger again
    calls = [(11, 2, 4), (12, 1, 2), (13, 3, 5)]
    for prec, dtype in ((0, torch.float64), (1, torch.float32)):
        for seed, m_max, n_max in calls:
            pos, radii = _config(seed, n_beads, L, 10.0, 40.0)
            dpos = torch.tensor(pos.reshape(-1), dtype=torch.float64, device="cuda")
            drad = torch.tensor(radii, dtype=torch.float64, device="cuda")
            ref = torch.zeros(n * n, dtype=dtype, device="cuda")
            out = torch.full((n * n,), float("nan"), dtype=dtype, device="cuda")
            _lib.call("pbg_dev_smith_matrix", dpos.data_ptr(), drad.data_ptr(), n_beads, L, alpha, m_max, n_max,
                      1.0, prec, ref.data_ptr(), n, None)
            _lib.call("pbg_dev_smith_matrix_noalloc", dpos.data_ptr(), drad.data_ptr(), n_beads, L, alpha, m_max,
                      n_max, 1.0, prec, out.data_ptr(), n, None)
            torch.cuda.synchronize()
            r = ref.cpu().numpy()
            o = out.cpu().numpy()
            assert np.all(np.isfinite(o))
            assert np.array_equal(o, r), (prec, m_max, n_max, _rel(o.astype(np.float64), r.astype(np.float64)))


@pytest.mark.gpu
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


def test_noalloc_rejects_huge_lattice_before_building_tables():
    """An oversized ewald_real / ewald_imag is refused from the closed-form
    lattice counts at once, before any table is built or any CUDA call is
    made (so this runs without a GPU too)."""
    import ctypes
    import time
    from pybrown_b200 import _lib
    for m_max, n_max in ((1000, 4), (2, 1000), (100000, 100000), (2**31 - 1, 4)):
        t0 = time.perf_counter()
        rc = _lib.lib.pbg_dev_smith_matrix_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), 64,
                                                   ctypes.c_double(750.0), ctypes.c_double(math.sqrt(math.pi)),
                                                   m_max, n_max, ctypes.c_double(1.0), 0, ctypes.c_void_p(16),
                                                   192, None)
        assert rc == -2, (m_max, n_max, rc)
        assert "fixed scratch" in _lib.last_error()
        assert time.perf_counter() - t0 < 0.5
