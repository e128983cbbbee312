"""Generate tests/golden/interactions.json from the reference's own
interactions module (src/bdsim/pyBrown/interactions.py:641-849).

    make -C oracle ref && python tests/golden/make_golden_interactions.py

Seeded bead pairs and triples (with bond and angle parameters and
Lennard-Jones radii and well depths) go through the reference's harmonic
bond / angle and LJ 6 / 12 / 6-12 force and energy functions, and the whole
host evaluation (set_interactions, then compute_forces_and_energy on the
reference's pair vectors) runs over the same beads; the results are stored
as JSON for tests/test_interactions_golden.py.
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import _import_reference  # noqa: E402

L = 40.0


def bead_specs():
    rng = np.random.default_rng(7)
    specs = []
    for k in range(6):
        specs.append({"id": k + 1, "r": rng.uniform(-6.0, 6.0, size=3).tolist(), "a": float(rng.uniform(0.8, 1.6)),
                      "hard_core_radius": float(rng.uniform(0.9, 1.4)), "epsilon_LJ": float(rng.uniform(0.1, 2.0))})
    return specs


def main():
    bead_mod, _, _ = _import_reference()
    from pyBrown import interactions as ref  # noqa: E402
    specs = bead_specs()
    beads = [bead_mod.Bead(np.array(s["r"]), s["a"], hard_core_radius=s["hard_core_radius"],
                           epsilon_LJ=s["epsilon_LJ"], bead_id=s["id"]) for s in specs]
    bonds = [(0, 1, 3.5, 12.0), (1, 2, 2.25, 7.5), (3, 4, 4.0, 3.0)]
    for i, j, d, k in bonds:
        beads[i].bonded_with.append(beads[j].bead_id)
        beads[i].bonded_how[beads[j].bead_id] = [d, k]
    angles = [(0, 1, 2, 120.0, 5.0), (2, 3, 4, 95.0, 2.5), (5, 0, 3, 150.0, 8.0)]
    for i, j, k, th, kk in angles:
        beads[i].angled_with.append([beads[j].bead_id, beads[k].bead_id])
        beads[i].angled_how[(beads[j].bead_id, beads[k].bead_id)] = [th, kk]
    out = {"L": L, "beads": specs, "bonds": bonds, "angles": angles, "pairs": [], "bond_terms": [],
           "angle_terms": []}
    alpha = 4.0
    for i in range(6):
        for j in range(i + 1, 6):
            p = bead_mod.pointer_pbc(beads[i], beads[j], L)
            out["pairs"].append({
                "i": i, "j": j, "alpha": alpha,
                "LJ_6_attractive_force": ref.LJ_6_attractive_force(beads[i], beads[j], p, alpha).tolist(),
                "LJ_6_attractive_energy": ref.LJ_6_attractive_energy(beads[i], beads[j], p, alpha),
                "LJ_12_repulsive_force": ref.LJ_12_repulsive_force(beads[i], beads[j], p, alpha).tolist(),
                "LJ_12_repulsive_energy": ref.LJ_12_repulsive_energy(beads[i], beads[j], p, alpha),
                "LJ_6_12_force": ref.LJ_6_12_force(beads[i], beads[j], p, alpha).tolist(),
                "LJ_6_12_energy": ref.LJ_6_12_energy(beads[i], beads[j], p, alpha)})
    for i, j, _, _ in bonds:
        p = bead_mod.pointer_pbc(beads[i], beads[j], L)
        out["bond_terms"].append({"i": i, "j": j,
                                  "force": ref.harmonic_bond_force(beads[i], beads[j], p).tolist(),
                                  "energy": ref.harmonic_bond_energy(beads[i], beads[j], p)})
    for i, j, k, _, _ in angles:
        p12 = bead_mod.pointer_pbc(beads[i], beads[j], L)
        p23 = bead_mod.pointer_pbc(beads[j], beads[k], L)
        out["angle_terms"].append({"i": i, "j": j, "k": k,
                                   "force": ref.harmonic_angle_force(beads[i], beads[j], beads[k], p12, p23,
                                                                     L).tolist(),
                                   "energy": float(ref.harmonic_angle_energy(beads[i], beads[j], beads[k], p12,
                                                                             p23, L))})
    out["units"] = {"kcal_per_mole_to_joule": ref.kcal_per_mole_to_joule(2.5),
                    "joule_to_kcal_per_mole": ref.joule_to_kcal_per_mole(3.0e-21),
                    "eV_to_joule": ref.eV_to_joule(0.75), "joule_to_eV": ref.joule_to_eV(1.0e-19)}
    # the whole host evaluation: set_interactions + compute_forces_and_energy
    # over a bonded chain with angles and LJ 6-12 (all beads mobile)
    inp = {"lennard_jones_6": True, "lennard_jones_12": True, "lennard_jones_alpha": alpha,
           "custom_interactions": False, "box_length": L}
    rij = np.asarray(bead_mod.compute_pointer_pbc_matrix(beads, L))
    F = np.zeros(3 * len(beads))
    E = 0.0
    for inter in ref.set_interactions(inp, beads):
        E += inter.compute_forces_and_energy(beads, rij, F)
    out["full"] = {"input": inp, "pointers": rij.tolist(), "F": F.tolist(), "E": E}
    assert math.isfinite(out["angle_terms"][0]["energy"])
    with open(os.path.join(HERE, "interactions.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "interactions.json"))


if __name__ == "__main__":
    main()
