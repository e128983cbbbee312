"""Inter-bead forces and immobile beads on the GPU (Box with device
interactions) against the reference's own trajectories (tests/golden/forces.npz)
and against the oracle on a larger polymer system.  Bar: positions, Box.F and
Box.E within 1e-10 relative; identical RNG draw counts."""
import json
import math

import numpy as np
import pytest

from conftest import rel_err
from test_forces_oracle import CASES, custom_terms, fixture_case

pytestmark = pytest.mark.gpu


def _product_beads(beads):
    from pybrown_b200.bead import Bead
    out = []
    for b in beads:
        nb = Bead(np.array(b.r, float), b.a, label=b.label, hard_core_radius=b.hard_core_radius,
                  epsilon_LJ=b.epsilon_LJ, bead_id=b.bead_id)
        nb.bonded_with = list(b.bonded_with)
        nb.bonded_how = dict(b.bonded_how)
        nb.angled_with = [list(x) for x in b.angled_with]
        nb.angled_how = dict(b.angled_how)
        out.append(nb)
    return out


def _full_inp(inp):
    from pybrown_b200.bd import DEFAULTS
    d = dict(DEFAULTS)
    d.update(inp)
    return d


@pytest.mark.parametrize("name", CASES)
def test_box_forces_match_reference(forces_golden, name):
    from pybrown_b200.box import Box
    beads, inp = fixture_case(forces_golden, name)
    box = Box(_product_beads(beads), _full_inp(inp))
    init = np.array([b.r for b in box.beads])
    dt = float(forces_golden[f"{name}/dt"])
    for k in range(len(forces_golden[f"{name}/traj"])):
        box.propagate(dt)
        assert box.draw_count == forces_golden[f"{name}/draws"][k]
        got = np.array([b.r for b in box.beads])
        ref = forces_golden[f"{name}/traj"][k]
        assert rel_err(got - init, ref - init) <= 1e-10, k
        E = forces_golden[f"{name}/E"][k]
        assert abs(box.E - E) <= 1e-10 * abs(E), k
        assert rel_err(box.F, forces_golden[f"{name}/F"][k]) <= 1e-10, k


def _polymer_system(seed, chains, length, n_obstacles, L):
    """Chains of bonded beads (bond 4.2, angle 150 deg) with LJ between all
    beads and immobile obstacle beads bonded to some chain ends."""
    rng = np.random.default_rng(seed)

    class B:
        pass

    beads, bid = [], 1
    placed = []

    def free(p, a):
        for q, b in placed:
            d = p - q
            d -= L * np.round(d / L)
            if np.linalg.norm(d) <= a + b + 0.3:
                return False
        return True

    for c in range(chains):
        while True:
            start = rng.uniform(-L / 2, L / 2, 3)
            direction = rng.normal(size=3)
            direction /= np.linalg.norm(direction)
            pts = [start + 4.2 * i * direction + rng.normal(scale=0.2, size=3) for i in range(length)]
            if all(free(p, 2.0) for p in pts):
                break
        ids = []
        for p in pts:
            b = B()
            b.r, b.a, b.label, b.bead_id = p, 2.0, "P", bid
            b.hard_core_radius, b.epsilon_LJ = 1.9, 0.2 + 0.1 * (bid % 3)
            b.bonded_with, b.bonded_how, b.angled_with, b.angled_how = [], {}, [], {}
            beads.append(b)
            placed.append((p, 2.0))
            ids.append(bid)
            bid += 1
        for i in range(length - 1):
            beads[ids[i] - 1].bonded_with.append(ids[i + 1])
            beads[ids[i] - 1].bonded_how[ids[i + 1]] = [4.2, 5.0]
        for i in range(length - 2):
            beads[ids[i] - 1].angled_with.append([ids[i + 1], ids[i + 2]])
            beads[ids[i] - 1].angled_how[(ids[i + 1], ids[i + 2])] = [150.0, 2.0]
    obstacles = []
    while len(obstacles) < n_obstacles:
        p = rng.uniform(-L / 2, L / 2, 3)
        if free(p, 3.0):
            b = B()
            b.r, b.a, b.label, b.bead_id = p, 3.0, "OBS", 1000 + len(obstacles)
            b.hard_core_radius, b.epsilon_LJ = 2.5, 0.3
            b.bonded_with, b.bonded_how, b.angled_with, b.angled_how = [], {}, [], {}
            placed.append((p, 3.0))
            obstacles.append(b)
    # tether two chain ends to their nearest obstacles (both bond directions)
    for c, ob in zip((0, 1), obstacles[:2]):
        head = beads[c * length]
        d = ob.r - head.r
        d -= L * np.round(d / L)
        if c == 0:
            head.bonded_with.append(ob.bead_id)
            head.bonded_how[ob.bead_id] = [float(np.linalg.norm(d)), 1.0]
        else:
            ob.bonded_with.append(head.bead_id)
            ob.bonded_how[head.bead_id] = [float(np.linalg.norm(d)), 1.0]
    order = list(range(len(beads) + len(obstacles)))
    rng.shuffle(order)
    allb = beads + obstacles
    return [allb[i] for i in order]


@pytest.mark.parametrize("hydro", ["rpy", "rpy_smith"])
def test_box_polymer_vs_oracle(oracle_lib, hydro):
    """4 chains of 24 beads, LJ 6-12, bonds, angles, 16 immobile obstacles (kcal/mol)."""
    from oracle.oracle import OracleForceBox
    from pybrown_b200.box import Box
    L = 80.0
    beads = _polymer_system(3, 4, 24, 16, L)
    inp = _full_inp({"box_length": L, "T": 293.15, "viscosity": 0.01005, "seed": 4, "hydrodynamics": hydro,
                     "ewald_alpha": math.sqrt(math.pi), "ewald_real": 1, "ewald_imag": 2,
                     "immobile_labels": ["OBS"], "lennard_jones_6": True, "lennard_jones_12": True,
                     "lennard_jones_alpha": 4.0, "energy_unit": "kcal/mol"})
    box = Box(_product_beads(beads), dict(inp))
    ref = OracleForceBox(beads, inp, clib=oracle_lib)
    init = ref.positions_all()
    for _ in range(6):
        box.propagate(0.05)
        ref.propagate(0.05)
        assert box.draw_count == ref.draw_count
        assert rel_err(box.F, ref.F) <= 1e-10
        assert abs(box.E - ref.E) <= 1e-10 * abs(ref.E)
    def disp(x):
        d = x - init
        return d - L * np.round(d / L)  # beads that crossed the box edge

    got = np.array([b.r for b in box.beads])
    assert rel_err(disp(got), disp(ref.positions_all())) <= 1e-10
    assert len(box.mobile_beads) == 96 and len(box.immobile_beads) == 16


def test_force_and_energy_before_first_step():
    """box.py:644: F starts at zero and E at 0.0."""
    from pybrown_b200.box import Box
    beads = _polymer_system(5, 1, 6, 0, 60.0)
    inp = _full_inp({"box_length": 60.0, "T": 293.15, "viscosity": 0.01005, "seed": 0, "hydrodynamics": "rpy",
                     "lennard_jones_12": True})
    box = Box(_product_beads(beads), inp)
    assert box.E == 0.0
    assert not np.any(box.F)
