"""GPU tensors through the reference ABI (pybrown_b200.diffusion / .bead, i.e.
the C exports of libpybrown_b200) against the reference's outputs
(tests/golden) and the CPU oracle.  Bar: relative error <= 1e-10 (FP64)."""
import math

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
CASES = ("grid27", "poly20", "rand33")
TOL = 1e-10


def _beads(pos, radii):
    from pybrown_b200.bead import Bead
    return [Bead(p, float(a)) for p, a in zip(pos, radii)]


@pytest.mark.parametrize("case", CASES)
def test_pointer_matrix_golden(tensors, case):
    from pybrown_b200.bead import compute_pointer_pbc_matrix
    got = compute_pointer_pbc_matrix(_beads(tensors[f"{case}/pos"], tensors[f"{case}/radii"]),
                                     float(tensors[f"{case}/L"]))
    assert np.array_equal(got, tensors[f"{case}/rij"])


def test_pointer_ties_golden(tensors):
    from pybrown_b200.bead import compute_pointer_pbc_matrix
    pos = tensors["pbc/pos"]
    got = compute_pointer_pbc_matrix(_beads(pos, np.ones(len(pos))), float(tensors["pbc/L"]))
    assert np.array_equal(got, tensors["pbc/rij"])


@pytest.mark.parametrize("case", CASES)
def test_rpy_golden(tensors, case):
    from pybrown_b200.diffusion import RPY_M_matrix
    got = RPY_M_matrix(_beads(tensors[f"{case}/pos"], tensors[f"{case}/radii"]), tensors[f"{case}/rij"])
    assert rel_err(got, tensors[f"{case}/rpy"]) <= TOL


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("mn", [(0, 0), (1, 1), (2, 4), (3, 3)])
def test_smith_golden(tensors, case, mn):
    from pybrown_b200.diffusion import RPY_Smith_M_matrix
    m, n = mn
    got = RPY_Smith_M_matrix(_beads(tensors[f"{case}/pos"], tensors[f"{case}/radii"]), tensors[f"{case}/rij"],
                             float(tensors[f"{case}/L"]), math.sqrt(math.pi), m, n)
    assert rel_err(got, tensors[f"{case}/smith_m{m}_n{n}"]) <= TOL
    assert np.array_equal(got, got.T)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("cutoff", [1.0, 10.0])
@pytest.mark.parametrize("cich", [True, False])
def test_lubrication_golden(tensors, case, cutoff, cich):
    from pybrown_b200.diffusion import JO_R_lubrication_correction_matrix
    got = JO_R_lubrication_correction_matrix(_beads(tensors[f"{case}/pos"], tensors[f"{case}/radii"]),
                                             tensors[f"{case}/rij"], cutoff, cich)
    assert rel_err(got, tensors[f"{case}/lub_c{cutoff:g}_{int(cich)}"]) <= TOL


def test_jo2b_golden(tensors):
    from pybrown_b200.bead import Bead
    from pybrown_b200.diffusion import JO_2B_R_matrix
    for row, ref in zip(tensors["jo2b/in"], tensors["jo2b/out"]):
        got = JO_2B_R_matrix(Bead(np.zeros(3), row[0]), Bead(row[2:5], row[1]))
        assert rel_err(got, ref) <= TOL


def test_overlaps_golden(tensors):
    from pybrown_b200.bead import check_overlaps
    L = float(tensors["overlap/L"])
    for p, r, t, flag in zip(tensors["overlap/pos"], tensors["overlap/radii"], tensors["overlap/thr"],
                             tensors["overlap/flag"]):
        b = _beads(p, r)
        assert check_overlaps(b, L, float(t), np.zeros((len(b), len(b)), np.int32)) == bool(flag)


def test_overlaps_bonded_pairs_skipped():
    from pybrown_b200.bead import check_overlaps
    b = _beads([[0, 0, 0], [1.5, 0, 0], [5, 5, 5]], [1.0, 1.0, 1.0])
    conn = np.zeros((3, 3), np.int32)
    assert check_overlaps(b, 20.0, 0.0, conn)
    conn[0, 1] = conn[1, 0] = 1
    assert not check_overlaps(b, 20.0, 0.0, conn)


def _random_config(seed, N, L, amin, amax, gap=0.0):
    rng = np.random.default_rng(seed)
    pos, radii = [], []
    while len(pos) < N:
        a = rng.uniform(amin, amax)
        p = rng.uniform(-L / 2, L / 2, size=3)
        ok = True
        for q, b in zip(pos, radii):
            d = p - q
            d -= L * np.round(d / L)
            if np.linalg.norm(d) <= a + b + gap:
                ok = False
                break
        if ok:
            pos.append(p)
            radii.append(a)
    return np.array(pos), np.array(radii)


@pytest.mark.parametrize("N,L,amin,amax", [(64, 750.0, 20.0, 20.0), (150, 400.0, 10.0, 40.0), (200, 60.0, 1.0, 2.5)])
def test_smith_vs_oracle_random(oracle_lib, N, L, amin, amax):
    from pybrown_b200.diffusion import RPY_Smith_M_matrix
    pos, radii = _random_config(N, N, L, amin, amax)
    rij = oracle_lib.pointers(pos, L)
    ref = oracle_lib.smith(radii, rij, L, math.sqrt(math.pi), 2, 4)
    got = RPY_Smith_M_matrix(_beads(pos, radii), rij, L, math.sqrt(math.pi), 2, 4)
    assert rel_err(got, ref) <= TOL


def test_lubrication_vs_oracle_dense(oracle_lib):
    from pybrown_b200.diffusion import JO_R_lubrication_correction_matrix
    # volume fraction ~0.25, minimum gap 0.05: many pairs inside the cutoff
    pos, radii = _random_config(7, 120, 19.5, 1.0, 2.0, gap=0.05)
    rij = oracle_lib.pointers(pos, 19.5)
    for cich in (True, False):
        ref = oracle_lib.lubrication(radii, rij, 0.5, cich)
        got = JO_R_lubrication_correction_matrix(_beads(pos, radii), rij, 0.5, cich)
        off_diagonal_blocks = np.count_nonzero(ref) - np.count_nonzero(np.kron(np.eye(120), np.ones((3, 3))) * ref)
        assert off_diagonal_blocks >= 9 * 60  # at least 30 lubricated pairs
        assert rel_err(got, ref) <= TOL


def test_device_smith_mixed_precision(oracle_lib):
    """FP32 Ewald build (mixed path) against the FP64 oracle."""
    import torch
    from pybrown_b200 import _lib
    N, L = 256, 1500.0
    pos, radii = _random_config(3, N, L, 10.0, 40.0)
    rij = oracle_lib.pointers(pos, L)
    ref = oracle_lib.smith(radii, rij, L, math.sqrt(math.pi), 2, 4)
    n = 3 * N
    for prec, dtype, tol in ((0, torch.float64, TOL), (1, torch.float32, 2e-6)):
        M = torch.zeros(n * n, dtype=dtype, device="cuda")
        dpos = torch.tensor(pos.reshape(-1), dtype=torch.float64, device="cuda")
        drad = torch.tensor(radii, dtype=torch.float64, device="cuda")
        _lib.call("pbg_dev_smith_matrix", dpos.data_ptr(), drad.data_ptr(), N, L, math.sqrt(math.pi), 2, 4, 1.0,
                  prec, M.data_ptr(), n, None)
        torch.cuda.synchronize()
        got = M.double().cpu().numpy().reshape(n, n)
        assert rel_err(got, ref) <= tol, prec
