"""Box.propagate on the GPU against the reference's own trajectories
(tests/golden/trajectories.npz) and against the CPU oracle on larger systems.
FP64 bar: displacement relative error <= 1e-10 and identical RNG draw counts
(every accept/reject decision agrees)."""
import json
import math

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TRAJ = ("ermak_nohi", "ermak_rpy", "ermak_smith", "ermak_smith_force", "ermak_rpy_reject",
        "midpoint_smith_lub", "midpoint_lub_reject")


def _box(init, radii, inp):
    from pybrown_b200.bead import Bead
    from pybrown_b200.box import Box
    beads = [Bead(np.array(p, float), float(a)) for p, a in zip(init, radii)]
    return Box(beads, dict(inp))


@pytest.mark.parametrize("name", TRAJ)
def test_box_matches_reference_trajectory(trajectories, name):
    inp = json.loads(str(trajectories[f"{name}/config"]))
    init = trajectories[f"{name}/init"]
    radii = np.full(len(init), float(trajectories[f"{name}/radius"]))
    dt = float(trajectories[f"{name}/dt"])
    box = _box(init, radii, inp)
    for k, (ref, draws) in enumerate(zip(trajectories[f"{name}/traj"], trajectories[f"{name}/draws"])):
        box.propagate(dt)
        pos = np.array([b.r for b in box.beads])
        assert box.draw_count == draws, k
        assert rel_err(pos - init, ref - init) <= 1e-10, k


def _config(seed, N, L, a_lo, a_hi, gap):
    rng = np.random.default_rng(seed)
    pos, radii = [], []
    while len(pos) < N:
        a = rng.uniform(a_lo, a_hi)
        p = rng.uniform(-L / 2, L / 2, size=3)
        good = True
        for q, b in zip(pos, radii):
            d = p - q
            d -= L * np.round(d / L)
            if np.linalg.norm(d) <= a + b + gap:
                good = False
                break
        if good:
            pos.append(p)
            radii.append(a)
    return np.array(pos), np.array(radii)


def _inp(**kw):
    d = {"box_length": 750.0, "T": 293.15, "viscosity": 0.01005, "seed": 0, "hydrodynamics": "rpy_smith",
         "ewald_alpha": math.sqrt(math.pi), "ewald_real": 2, "ewald_imag": 4, "propagation_scheme": "ermak",
         "immobile_labels": [], "check_overlaps": True, "overlap_treshold": 0.0, "max_move_attempts": 1000000,
         "external_force": [0.0, 0.0, 0.0], "energy_unit": "joule", "verbose": False, "debug": False,
         "lubrication_cutoff": 0.5, "cichocki_correction": True, "m_midpoint": 100,
         "lennard_jones_6": False, "lennard_jones_12": False, "custom_interactions": False}
    d.update(kw)
    return d


def test_box_vs_oracle_bd_hi_n64(oracle_lib):
    """The BD-with-HI workload at N=64 (radius 20, box 750, Smith m=2 n=4, dt=1)."""
    from oracle.oracle import OracleBox
    pos, radii = _config(0, 64, 750.0, 20.0, 20.0, 0.0)
    inp = _inp()
    box = _box(pos, radii, inp)
    ref = OracleBox(pos, radii, inp, clib=oracle_lib)
    for _ in range(25):
        box.propagate(1.0)
        ref.propagate(1.0)
        assert box.draw_count == ref.draw_count
    got = np.array([b.r for b in box.beads])
    assert rel_err(got - pos, ref.pos - pos) <= 1e-10
    assert rel_err(box.D, ref.D) <= 1e-10


def test_box_vs_oracle_stokesian(oracle_lib):
    """SD with lubrication and midpoint at a dense packing (phi ~ 0.3, gap >= 0.05 a)."""
    from oracle.oracle import OracleBox
    N, a = 48, 20.0
    L = (N * 4 * math.pi * a ** 3 / 3 / 0.30) ** (1 / 3)
    pos, radii = _config(5, N, L, a, a, 0.05 * a)
    inp = _inp(box_length=L, hydrodynamics="rpy_smith_lub", propagation_scheme="midpoint", lubrication_cutoff=0.5)
    box = _box(pos, radii, inp)
    ref = OracleBox(pos, radii, inp, clib=oracle_lib)
    for _ in range(5):
        box.propagate(0.1)
        ref.propagate(0.1)
        assert box.draw_count == ref.draw_count
    got = np.array([b.r for b in box.beads])
    assert rel_err(got - pos, ref.pos - pos) <= 1e-10
    assert rel_err(box.R, ref.R) <= 1e-10
    assert rel_err(box.D, ref.D) <= 1e-10


def test_box_mixed_precision_displacement(oracle_lib):
    """Mixed path (FP32 Ewald + FP32 Cholesky updates, FP64 positions): the
    displacement after 20 steps stays within 1e-5 of the FP64 oracle."""
    from oracle.oracle import OracleBox
    pos, radii = _config(1, 256, 1500.0 * (256 / 1024) ** (1 / 3), 10.0, 40.0, 0.0)
    L = 1500.0 * (256 / 1024) ** (1 / 3)
    inp = _inp(box_length=L, precision="mixed")
    box = _box(pos, radii, inp)
    ref_inp = dict(inp)
    ref_inp.pop("precision")
    ref = OracleBox(pos, radii, ref_inp, clib=oracle_lib)
    for _ in range(20):
        box.propagate(0.5)
        ref.propagate(0.5)
    got = np.array([b.r for b in box.beads])
    assert rel_err(got - pos, ref.pos - pos) <= 1e-5


def test_box_pickle_resume_bit_exact():
    """Restart files (output.py:72-84; test_box.py:53-119): resuming from a
    pickled Box reproduces the uninterrupted trajectory bit for bit."""
    import pickle
    pos, radii = _config(2, 27, 100.0, 2.0, 2.0, 0.5)
    box = _box(pos, radii, _inp(box_length=100.0, ewald_real=1, ewald_imag=2))
    for _ in range(4):
        box.propagate(1.0)
    blob = pickle.dumps(box)
    for _ in range(3):
        box.propagate(1.0)
    original = [b.r.copy() for b in box.beads]
    resumed = pickle.loads(blob)
    for _ in range(3):
        resumed.propagate(1.0)
    assert all(np.array_equal(o, r.r) for o, r in zip(original, resumed.beads))


# Bars of the mixed lubricated path (max-abs / max against the FP64 oracle).
# The FP32 far-field inverse sets them: cond(Mff) ~ 2e2 and cond(R) ~ 7e2 at
# phi = 0.3 turn FP32 rounding into ~1e-5 in Rff, D and B; the midpoint drift
# multiplies the difference of two solves by m/2 = 50.
MLUB_BARS = {"ermak": 5e-5, "midpoint": 5e-4}


@pytest.mark.parametrize("scheme", ["midpoint", "ermak"])
def test_box_mixed_lubrication(oracle_lib, scheme):
    """Mixed lubricated path (FP32 far-field mobility and its tensor-core
    inverse, FP64 near-field correction and R, the FP32 factor of the
    reversed R for the noise, FP64-refined solves for D F and the midpoint
    drift) against the FP64 oracle at a dense packing (phi 0.3, gap >= 0.05 a),
    with the rebuild flags of diff_freq / lub_freq / chol_freq exercised on
    the Ermak run."""
    from oracle.oracle import OracleBox
    N, a = 128, 20.0
    L = (N * 4 * math.pi * a ** 3 / 3 / 0.30) ** (1 / 3)
    pos, radii = _config(7, N, L, a, a, 0.05 * a)
    inp = _inp(box_length=L, hydrodynamics="rpy_smith_lub", propagation_scheme=scheme, lubrication_cutoff=0.5)
    box = _box(pos, radii, dict(inp, precision="mixed"))
    ref = OracleBox(pos, radii, inp, clib=oracle_lib)
    flags = [(True, True, True)] * 6
    if scheme == "ermak":
        flags = [(True, True, True), (False, True, True), (True, True, False), (False, False, True),
                 (True, True, True), (False, True, False)]
    for b_ff, b_nf, chol in flags:
        box.propagate(0.1, build_Dff=b_ff, build_Dnf=b_nf, cholesky=chol)
        ref.propagate(0.1, build_Dff=b_ff, build_Dnf=b_nf, cholesky=chol)
        assert box.draw_count == ref.draw_count
    got = np.array([b.r for b in box.beads])
    assert rel_err(got - pos, ref.pos - pos) <= MLUB_BARS[scheme]
    assert rel_err(box.R, ref.R) <= 1e-5
    assert rel_err(box.Rff, ref.Rff) <= 5e-5
    assert rel_err(box.D, ref.D) <= 1e-4
    assert rel_err(box.B, ref.B) <= 1e-4


def test_box_mixed_lubrication_odd_tile_count(oracle_lib):
    """Mixed SD at N=48: order 144 padded to 192, an odd number (3) of 64-wide
    tiles, so the tensor-core inverse's workspace offsets are not multiples of
    an even tile count."""
    from oracle.oracle import OracleBox
    N, a = 48, 20.0
    L = (N * 4 * math.pi * a ** 3 / 3 / 0.30) ** (1 / 3)
    pos, radii = _config(5, N, L, a, a, 0.05 * a)
    inp = _inp(box_length=L, hydrodynamics="rpy_smith_lub", propagation_scheme="midpoint", lubrication_cutoff=0.5)
    box = _box(pos, radii, dict(inp, precision="mixed"))
    ref = OracleBox(pos, radii, inp, clib=oracle_lib)
    for _ in range(3):
        box.propagate(0.1)
        ref.propagate(0.1)
        assert box.draw_count == ref.draw_count
    got = np.array([b.r for b in box.beads])
    assert rel_err(got - pos, ref.pos - pos) <= MLUB_BARS["midpoint"]
    assert rel_err(box.D, ref.D) <= 1e-4
    assert rel_err(box.B, ref.B) <= 1e-4


def test_box_vs_oracle_stokesian_n256(oracle_lib):
    """FP64 SD at N=256 (order 768, 12 tiles: every level of the tensor-core
    triangular inverse down to 8-tile blocks) against the oracle."""
    from oracle.oracle import OracleBox
    N, a = 256, 20.0
    L = (N * 4 * math.pi * a ** 3 / 3 / 0.30) ** (1 / 3)
    pos, radii = _config(11, N, L, a, a, 0.05 * a)
    inp = _inp(box_length=L, hydrodynamics="rpy_smith_lub", propagation_scheme="midpoint", lubrication_cutoff=0.5)
    box = _box(pos, radii, inp)
    ref = OracleBox(pos, radii, inp, clib=oracle_lib)
    for _ in range(2):
        box.propagate(0.1)
        ref.propagate(0.1)
        assert box.draw_count == ref.draw_count
    got = np.array([b.r for b in box.beads])
    assert rel_err(got - pos, ref.pos - pos) <= 1e-10
    assert rel_err(box.Rff, ref.Rff) <= 1e-10
    assert rel_err(box.D, ref.D) <= 1e-10
    assert rel_err(box.B, ref.B) <= 1e-10
