"""Generate tests/golden/bead.json from the reference's own bead module.

Run in a container that has the reference tree and oracle/_ref built:

    make -C oracle ref && python tests/golden/make_golden_bead.py

Seeded beads in a periodic box (some pairs straddling the box edge) go
through the reference's pure-Python bead functions (src/bdsim/pyBrown/
bead.py: pointer, pointer_pbc, distance, distance_pbc, overlap, overlap_pbc,
build_connection_matrix, get_bead_with_id, Bead.translate, Bead.keep_in_box)
and the results are stored as JSON; tests/test_bead_golden.py only reads it.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import _import_reference  # noqa: E402

L = 30.0


def beads_input():
    rng = np.random.default_rng(42)
    pos = rng.uniform(-L / 2, L / 2, size=(8, 3))
    pos[1] = pos[0] + np.array([L - 1.5, 0.5, -0.25])  # straddles the box edge
    pos[1] -= L * np.round(pos[1] / L)
    radii = rng.uniform(0.5, 2.0, size=8)
    return pos, radii


def main():
    bead_mod, _, _ = _import_reference()
    pos, radii = beads_input()

    def make():
        bs = [bead_mod.Bead(p.copy(), float(a), bead_id=i + 1) for i, (p, a) in enumerate(zip(pos, radii))]
        bs[0].bonded_with.append(3)
        bs[2].bonded_with.append(5)
        bs[6].mobile = False
        bs[7].mobile = False
        return bs

    bs = make()
    out = {"L": L, "pos": pos.tolist(), "radii": radii.tolist(), "bonds": [[1, 3], [3, 5]], "immobile": [7, 8]}
    pairs = []
    for i in range(8):
        for j in range(8):
            if i == j:
                continue
            pairs.append({"i": i, "j": j,
                          "pointer": bead_mod.pointer(bs[i], bs[j]).tolist(),
                          "pointer_pbc": bead_mod.pointer_pbc(bs[i], bs[j], L).tolist(),
                          "distance": bead_mod.distance(bs[i], bs[j]),
                          "distance_pbc": bead_mod.distance_pbc(bs[i], bs[j], L),
                          "overlap": bool(bead_mod.overlap(bs[i], bs[j])),
                          "overlap_pbc": bool(bead_mod.overlap_pbc(bs[i], bs[j], L)),
                          "overlap_pbc_eps": bool(bead_mod.overlap_pbc(bs[i], bs[j], L, 25.0))})
    out["pairs"] = pairs
    out["connection_matrix"] = np.asarray(bead_mod.build_connection_matrix(bs)).astype(int).tolist()
    out["get_bead_with_id"] = [bead_mod.get_bead_with_id(bs, k) for k in (1, 5, 8, 99)]
    moved = make()
    shifts = np.array([[2.5 * L, -0.75 * L, 0.1], [-3.2 * L, 1.6 * L, -0.49 * L]])
    for b, sft in zip(moved[:2], shifts):
        b.translate(sft)
        b.keep_in_box(L)
    out["translate_shifts"] = shifts.tolist()
    out["kept_in_box"] = [b.r.tolist() for b in moved[:2]]
    with open(os.path.join(HERE, "bead.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "bead.json"))


if __name__ == "__main__":
    main()
