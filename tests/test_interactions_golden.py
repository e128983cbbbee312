"""Host force-field helpers of pybrown_b200.interactions against the
reference's own (CPU): tests/golden/interactions.json holds what the
reference's harmonic bond / angle and Lennard-Jones force and energy
functions and unit conversions returned for seeded beads
(tests/golden/make_golden_interactions.py).  Results must be identical."""
import json
import os

import numpy as np
import pytest

from pybrown_b200 import bead as B
from pybrown_b200 import interactions as I

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "interactions.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _beads(g):
    beads = [B.Bead(np.array(s["r"]), s["a"], hard_core_radius=s["hard_core_radius"], epsilon_LJ=s["epsilon_LJ"],
                    bead_id=s["id"]) for s in g["beads"]]
    for i, j, d, k in g["bonds"]:
        beads[i].bonded_with.append(beads[j].bead_id)
        beads[i].bonded_how[beads[j].bead_id] = [d, k]
    for i, j, k, th, kk in g["angles"]:
        beads[i].angled_with.append([beads[j].bead_id, beads[k].bead_id])
        beads[i].angled_how[(beads[j].bead_id, beads[k].bead_id)] = [th, kk]
    return beads


def test_lennard_jones_terms(golden):
    beads, L = _beads(golden), golden["L"]
    for t in golden["pairs"]:
        b1, b2, alpha = beads[t["i"]], beads[t["j"]], t["alpha"]
        p = B.pointer_pbc(b1, b2, L)
        assert I.LJ_6_attractive_force(b1, b2, p, alpha).tolist() == t["LJ_6_attractive_force"]
        assert I.LJ_6_attractive_energy(b1, b2, p, alpha) == t["LJ_6_attractive_energy"]
        assert I.LJ_12_repulsive_force(b1, b2, p, alpha).tolist() == t["LJ_12_repulsive_force"]
        assert I.LJ_12_repulsive_energy(b1, b2, p, alpha) == t["LJ_12_repulsive_energy"]
        assert I.LJ_6_12_force(b1, b2, p, alpha).tolist() == t["LJ_6_12_force"]
        assert I.LJ_6_12_energy(b1, b2, p, alpha) == t["LJ_6_12_energy"]


def test_harmonic_terms(golden):
    beads, L = _beads(golden), golden["L"]
    for t in golden["bond_terms"]:
        b1, b2 = beads[t["i"]], beads[t["j"]]
        p = B.pointer_pbc(b1, b2, L)
        assert I.harmonic_bond_force(b1, b2, p).tolist() == t["force"]
        assert I.harmonic_bond_energy(b1, b2, p) == t["energy"]
    for t in golden["angle_terms"]:
        b1, b2, b3 = beads[t["i"]], beads[t["j"]], beads[t["k"]]
        p12, p23 = B.pointer_pbc(b1, b2, L), B.pointer_pbc(b2, b3, L)
        assert I.harmonic_angle_force(b1, b2, b3, p12, p23, L).tolist() == t["force"]
        assert float(I.harmonic_angle_energy(b1, b2, b3, p12, p23, L)) == t["energy"]


def test_unit_conversions(golden):
    u = golden["units"]
    assert I.kcal_per_mole_to_joule(2.5) == u["kcal_per_mole_to_joule"]
    assert I.joule_to_kcal_per_mole(3.0e-21) == u["joule_to_kcal_per_mole"]
    assert I.eV_to_joule(0.75) == u["eV_to_joule"]
    assert I.joule_to_eV(1.0e-19) == u["joule_to_eV"]


def test_set_interactions_full_evaluation(golden):
    """set_interactions + compute_forces_and_energy over a bonded chain with
    angles and LJ 6-12, on the reference's pair vectors: same F and E."""
    beads = _beads(golden)
    full = golden["full"]
    rij = np.array(full["pointers"])
    F = np.zeros(3 * len(beads))
    E = 0.0
    inters = I.set_interactions(full["input"], beads)
    assert [(i.how_many_body, i.bonded) for i in inters] == [(2, False), (2, True), (3, True)]
    for inter in inters:
        E += inter.compute_forces_and_energy(beads, rij, F)
    assert F.tolist() == full["F"]
    assert E == full["E"]
