"""The oracle's restatement of the reference's inter-bead forces and immobile
beads (oracle.OracleForceBox) against trajectories of the reference itself
(tests/golden/forces.npz, made by tests/golden/make_golden_forces.py): every
step's positions, RNG draw count, energy Box.E and force Box.F."""
import importlib
import json
import os
import sys

import numpy as np
import pytest

from conftest import rel_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("forces_chain_rpy", "forces_custom_smith", "forces_lj6_midpoint")


class _Bead:
    def __init__(self, t):
        self.r = np.array(t["r"], dtype=float)
        self.a = t["a"]
        self.label = t["label"]
        self.bead_id = t["id"]
        self.hard_core_radius = t["hc"]
        self.epsilon_LJ = t["eps"]
        self.bonded_with, self.bonded_how, self.angled_with, self.angled_how = [], {}, [], {}


def fixture_case(data, name):
    """Beads, input and reference records of one case."""
    table = json.loads(str(data[f"{name}/beads"]))
    beads = [_Bead(t) for t in table]
    by_id = {b.bead_id: b for b in beads}
    for i1, i2, eq, k in json.loads(str(data[f"{name}/bonds"])):
        by_id[i1].bonded_with.append(i2)
        by_id[i1].bonded_how[i2] = [eq, k]
    for i1, i2, i3, eq, k in json.loads(str(data[f"{name}/angles"])):
        by_id[i1].angled_with.append([i2, i3])
        by_id[i1].angled_how[(i2, i3)] = [eq, k]
    inp = json.loads(str(data[f"{name}/config"]))
    if inp.get("custom_interactions"):
        inp["custom_interactions_filename"] = os.path.join(GOLDEN, inp["custom_interactions_filename"])
    return beads, inp


def custom_terms(inp):
    """(force, energy, aux, bonded, body) of the custom-interactions file."""
    if not inp.get("custom_interactions"):
        return []
    sys.path.insert(0, GOLDEN)
    try:
        mod = importlib.import_module("custom_forces")
    finally:
        sys.path.pop(0)
    aux = inp["auxiliary_custom_interactions_keywords"]
    out = []
    for name in sorted(n[:-6] for n in dir(mod) if n.endswith("energy") and not n.startswith("_")):
        out.append((getattr(mod, name + "force"), getattr(mod, name + "energy"), aux,
                    "bonded" in name.split("_"), int(name.split("_")[-2][:-1])))
    return out


@pytest.mark.parametrize("name", CASES)
def test_oracle_forces_match_reference(forces_golden, oracle_lib, name):
    from oracle.oracle import OracleForceBox
    beads, inp = fixture_case(forces_golden, name)
    box = OracleForceBox(beads, inp, clib=oracle_lib, custom=custom_terms(inp))
    init = box.positions_all()
    dt = float(forces_golden[f"{name}/dt"])
    for k in range(len(forces_golden[f"{name}/traj"])):
        box.propagate(dt)
        assert box.draw_count == forces_golden[f"{name}/draws"][k]
        ref = forces_golden[f"{name}/traj"][k]
        assert rel_err(box.positions_all() - init, ref - init) <= 1e-12, k
        assert abs(box.E - forces_golden[f"{name}/E"][k]) <= 1e-12 * abs(forces_golden[f"{name}/E"][k])
        assert rel_err(box.F, forces_golden[f"{name}/F"][k]) <= 1e-12
