"""Generate the force fixtures (forces.npz) from the reference itself.

Run where the reference tree and oracle/_ref/libpyBrown.so exist:

    make -C oracle ref && python tests/golden/make_golden_forces.py

Runs the reference's Box.propagate (src/bdsim/pyBrown/box.py) on small systems
with inter-bead forces and immobile beads and records, after each step, the
positions of all beads, the RNG draw count, Box.E and Box.F:

  forces_chain_rpy      -- bonded chain with angles, LJ 6-12, kcal/mol, and
                           immobile beads bonded and angled to the chain in
                           every pair-vector form of interactions.py:291-414
  forces_custom_smith   -- LJ 12, external force, the custom interactions of
                           custom_forces.py (1-body and 2-body), eV, rpy_smith
  forces_lj6_midpoint   -- LJ 6 and bonds under the midpoint scheme, joule

The external force is given as floats: the reference sums forces into an
array built from it (box.py:452-460), which is an integer array for [0, 0, 0].

Each case also stores the bead table (ids, labels, radii, LJ parameters,
bonds and angles) so the tests rebuild identical inputs without the reference.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import _import_reference, mock_input  # noqa: E402


def chain_rpy():
    mob = [[-7.0 + 2.3 * i, 0.3 * (i % 2), 0.0] for i in range(7)]
    imm = [[-7.0, 3.0, 0.0], [0.0, 3.2, 0.5], [4.0, -3.0, 0.0]]
    beads = []
    for i, c in enumerate(mob):
        beads.append(dict(id=i + 1, label="MOB", r=c, a=1.0, hc=1.0, eps=0.3))
    for k, c in enumerate(imm):
        beads.append(dict(id=100 + k, label="IMM", r=c, a=1.0, hc=1.1, eps=0.2))
    bonds = [[i, i + 1, 2.3, 40.0] for i in range(1, 7)]
    bonds += [[2, 100, 3.0, 20.0], [101, 4, 3.2, 25.0]]
    angles = [[i, i + 1, i + 2, 170.0, 8.0] for i in range(1, 6)]
    angles += [[1, 100, 101, 120.0, 5.0],   # mobile i, j and k immobile: p23 = P(i,k) - P(i,j)
               [101, 100, 3, 100.0, 6.0],   # immobile i and j, mobile k: p12 = P(i,k) - P(j,k)
               [102, 6, 101, 90.0, 4.0],    # immobile i, mobile j, immobile k
               [5, 101, 6, 110.0, 3.0]]     # mobile i, immobile j, mobile k
    inp = mock_input(hydrodynamics="rpy", lennard_jones_6=True, lennard_jones_12=True,
                     lennard_jones_alpha=4.0, energy_unit="kcal/mol", immobile_labels=["IMM"],
                     external_force=[0.0, 0.0, 0.0])
    # a bead order with the immobile beads interleaved
    order = [0, 1, 7, 2, 3, 8, 4, 5, 6, 9]
    return [beads[i] for i in order], bonds, angles, inp, 2e-3, 12


def custom_smith():
    beads = [dict(id=i + 1, label="A", r=[2.4 * (i % 3) - 2.4, 2.4 * (i // 3) - 1.2, 0.2 * i], a=1.0,
                  hc=1.0, eps=0.5) for i in range(6)]
    inp = mock_input(hydrodynamics="rpy_smith", ewald_real=1, ewald_imag=1, box_length=20.0,
                     lennard_jones_12=True, lennard_jones_alpha=2.0, energy_unit="eV",
                     external_force=[1e-3, 0.0, -2e-3], custom_interactions=True,
                     custom_interactions_filename=os.path.join(HERE, "custom_forces.py"),
                     auxiliary_custom_interactions_keywords={"tether_k": 2e-3, "soft_eps": 5e-3})
    return beads, [], [], inp, 1e-3, 10


def lj6_midpoint():
    beads = [dict(id=i + 1, label="B", r=[2.5 * (i % 2), 2.5 * (i // 2), 0.0], a=1.0, hc=0.9, eps=1e-21)
             for i in range(4)]
    bonds = [[1, 2, 2.5, 2e-20], [3, 4, 2.5, 2e-20]]
    inp = mock_input(hydrodynamics="rpy", propagation_scheme="midpoint", m_midpoint=10.0,
                     lennard_jones_6=True, lennard_jones_alpha=1.0, energy_unit="joule",
                     external_force=[0.0, 0.0, 0.0])
    return beads, bonds, [], inp, 1e-3, 8


def make_beads(bead_mod, table, bonds, angles):
    Bead = bead_mod.Bead
    beads = [Bead(np.array(t["r"], float), t["a"], label=t["label"], hard_core_radius=t["hc"],
                  epsilon_LJ=t["eps"], bead_id=t["id"]) for t in table]
    by_id = {b.bead_id: b for b in beads}
    for i1, i2, eq, k in bonds:   # input.py:145-156
        by_id[i1].bonded_with.append(i2)
        by_id[i1].bonded_how[i2] = [eq, k]
    for i1, i2, i3, eq, k in angles:   # input.py:158-170
        by_id[i1].angled_with.append([i2, i3])
        by_id[i1].angled_how[(i2, i3)] = [eq, k]
    return beads


def main():
    bead_mod, box_mod, _ = _import_reference()
    out = {}
    for name, fn in (("forces_chain_rpy", chain_rpy), ("forces_custom_smith", custom_smith),
                     ("forces_lj6_midpoint", lj6_midpoint)):
        table, bonds, angles, inp, dt, steps = fn()
        beads = make_beads(bead_mod, table, bonds, angles)
        b = box_mod.Box(beads, dict(inp))
        traj, draws, E, F = [], [], [], []
        for _ in range(steps):
            b.propagate(dt)
            traj.append(np.array([bb.r for bb in b.beads]))
            draws.append(b.draw_count)
            E.append(b.E)
            F.append(np.array(b.F, dtype=float))
        cfg = dict(inp)
        if "custom_interactions_filename" in cfg:
            cfg["custom_interactions_filename"] = "custom_forces.py"
        out[f"{name}/beads"] = np.array(json.dumps(table))
        out[f"{name}/bonds"] = np.array(json.dumps(bonds))
        out[f"{name}/angles"] = np.array(json.dumps(angles))
        out[f"{name}/config"] = np.array(json.dumps(cfg))
        out[f"{name}/dt"] = np.array(dt)
        out[f"{name}/traj"] = np.array(traj)
        out[f"{name}/draws"] = np.array(draws)
        out[f"{name}/E"] = np.array(E)
        out[f"{name}/F"] = np.array(F)
    path = os.path.join(HERE, "forces.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
