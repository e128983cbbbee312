"""The CPU oracle (oracle/pybrown_oracle.c + oracle/oracle.py) against the
reference's own outputs (tests/golden/*.npz, made by tests/golden/make_golden.py
from the reference compiled here) and the known-answer values of the
reference's HYDROLIB / BD_BOX tests.  No GPU."""
import json
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

CASES = ("grid27", "poly20", "rand33")


@pytest.mark.parametrize("case", CASES)
def test_pointer_matrix(oracle_lib, tensors, case):
    got = oracle_lib.pointers(tensors[f"{case}/pos"], float(tensors[f"{case}/L"]))
    assert np.array_equal(got, tensors[f"{case}/rij"])


def test_pointer_ties(oracle_lib, tensors):
    got = oracle_lib.pointers(tensors["pbc/pos"], float(tensors["pbc/L"]))
    assert np.array_equal(got, tensors["pbc/rij"])


@pytest.mark.parametrize("case", CASES)
def test_rpy(oracle_lib, tensors, case):
    got = oracle_lib.rpy(tensors[f"{case}/radii"], tensors[f"{case}/rij"])
    assert rel_err(got, tensors[f"{case}/rpy"]) <= 1e-14


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("mn", [(0, 0), (1, 1), (2, 4), (3, 3)])
def test_smith(oracle_lib, tensors, case, mn):
    m, n = mn
    got = oracle_lib.smith(tensors[f"{case}/radii"], tensors[f"{case}/rij"], float(tensors[f"{case}/L"]),
                           math.sqrt(math.pi), m, n)
    assert rel_err(got, tensors[f"{case}/smith_m{m}_n{n}"]) <= 1e-13


@pytest.mark.parametrize("case", CASES)
def test_smith_alpha(oracle_lib, tensors, case):
    got = oracle_lib.smith(tensors[f"{case}/radii"], tensors[f"{case}/rij"], float(tensors[f"{case}/L"]), 2.0, 2, 2)
    assert rel_err(got, tensors[f"{case}/smith_alpha2_m2_n2"]) <= 1e-13


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("cutoff", [1.0, 10.0])
@pytest.mark.parametrize("cich", [True, False])
def test_lubrication(oracle_lib, tensors, case, cutoff, cich):
    got = oracle_lib.lubrication(tensors[f"{case}/radii"], tensors[f"{case}/rij"], cutoff, cich)
    ref = tensors[f"{case}/lub_c{cutoff:g}_{int(cich)}"]
    assert rel_err(got, ref) <= 1e-12


def test_jo2b(oracle_lib, tensors):
    for row, ref in zip(tensors["jo2b/in"], tensors["jo2b/out"]):
        got = oracle_lib.jo2b(row[0], row[1], row[2:5])
        # 6x6 layout of diffusion.py:120-139 vs the 18-vector
        ref18 = [ref[0][0], ref[1][1], ref[2][2], ref[0][1], ref[0][2], ref[1][2],
                 ref[3][3], ref[4][4], ref[5][5], ref[3][4], ref[3][5], ref[4][5],
                 ref[3][0], ref[4][1], ref[5][2], ref[4][0], ref[5][0], ref[5][1]]
        assert rel_err(got, ref18) <= 1e-13


def test_overlaps(oracle_lib, tensors):
    L = float(tensors["overlap/L"])
    flags = [oracle_lib.overlaps(p, r, L, t) for p, r, t in
             zip(tensors["overlap/pos"], tensors["overlap/radii"], tensors["overlap/thr"])]
    assert np.array_equal(np.array(flags, dtype=np.int32), tensors["overlap/flag"])
    assert 0 < tensors["overlap/flag"].sum() < len(flags)  # both outcomes are exercised


def _oracle_box(oracle_lib, trajectories, name):
    from oracle.oracle import OracleBox
    inp = json.loads(str(trajectories[f"{name}/config"]))
    init = trajectories[f"{name}/init"]
    radii = np.full(len(init), float(trajectories[f"{name}/radius"]))
    return OracleBox(init, radii, inp, clib=oracle_lib), float(trajectories[f"{name}/dt"])


TRAJ = ("ermak_nohi", "ermak_rpy", "ermak_smith", "ermak_smith_force", "ermak_rpy_reject",
        "midpoint_smith_lub", "midpoint_lub_reject")


@pytest.mark.parametrize("name", TRAJ)
def test_oracle_box_trajectory(oracle_lib, trajectories, name):
    box, dt = _oracle_box(oracle_lib, trajectories, name)
    traj = trajectories[f"{name}/traj"]
    draws = trajectories[f"{name}/draws"]
    init = trajectories[f"{name}/init"]
    for k in range(len(traj)):
        box.propagate(dt)
        assert box.draw_count == draws[k]
        disp_ref = traj[k] - init
        assert rel_err(box.pos - init, disp_ref) <= 1e-10, k


def test_known_answers_hydrolib(oracle_lib):
    """test_diffusion_vs_hydrolib.py:63-231 at the reference's tolerances."""
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        ka = json.load(f)
    pos = np.array([[0.0, 0.0, 0.0], [3000.0, 0.0, 0.0]])
    rij = oracle_lib.pointers(pos, 1000000.0)
    R_inf = np.linalg.inv(oracle_lib.rpy(np.ones(2), rij))[1][1]
    tol = {"3": 0.001, "2.5": 0.001, "2.1": 0.002, "2.01": 0.005, "2.001": 0.005}
    for sep, rec in ka["hydrolib_2body"].items():
        s = float(sep)
        R18 = oracle_lib.jo2b(1.0, 1.0, [s, 0.0, 0.0])
        R = np.zeros((6, 6))
        R[0, 0], R[1, 1], R[2, 2] = R18[0:3]
        R[3, 3], R[4, 4], R[5, 5] = R18[6:9]
        R[0, 3] = R[3, 0] = R18[12]
        R[1, 4] = R[4, 1] = R18[13]
        R[2, 5] = R[5, 2] = R18[14]
        ref = np.array(rec["R"]) / ka["hydrolib_R_infty"]
        assert np.max(np.abs(R / R_inf - ref)) <= tol[sep], sep


def test_known_answers_bdbox(oracle_lib):
    """test_diffusion_vs_bdbox.py:37-151 (coupling/diagonal ratios, delta 1e-4)."""
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        ka = json.load(f)
    for rec in ka["bdbox"]:
        pos = np.array([b[0] for b in rec["beads"]])
        radii = np.array([b[1] for b in rec["beads"]])
        rij = oracle_lib.pointers(pos, rec["box_size"])
        M = oracle_lib.smith(radii, rij, rec["box_size"], math.sqrt(math.pi), 2, 2)
        diag1 = rec.get("D_bdbox_diag_e", rec.get("D_bdbox_diag_1"))
        assert abs(M[3][0] / M[0][0] - rec["D_bdbox_coupling_ee"] / diag1) <= 1e-4, rec["test"]
        assert abs(M[5][2] / M[0][0] - rec["D_bdbox_coupling_rr"] / diag1) <= 1e-4, rec["test"]
        if "D_bdbox_diag_2" in rec:
            assert abs(M[0][0] / M[3][3] - rec["D_bdbox_diag_1"] / rec["D_bdbox_diag_2"]) <= 1e-4
