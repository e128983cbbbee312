"""pybrown_b200.bead's pure-Python functions against the reference's own
(CPU): tests/golden/bead.json holds what the reference's bead module returned
for seeded beads in a periodic box (tests/golden/make_golden_bead.py).
Floating-point results must be identical: the functions are restated with
the reference's evaluation order."""
import json
import os

import numpy as np
import pytest

from pybrown_b200 import bead as B

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bead.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _beads(g):
    bs = [B.Bead(np.array(p), float(a), bead_id=i + 1) for i, (p, a) in enumerate(zip(g["pos"], g["radii"]))]
    for i, j in g["bonds"]:
        bs[i - 1].bonded_with.append(j)
    for k in g["immobile"]:
        bs[k - 1].mobile = False
    return bs


def test_pair_functions(golden):
    bs, L = _beads(golden), golden["L"]
    for p in golden["pairs"]:
        b1, b2 = bs[p["i"]], bs[p["j"]]
        assert B.pointer(b1, b2).tolist() == p["pointer"]
        assert B.pointer_pbc(b1, b2, L).tolist() == p["pointer_pbc"]
        assert B.distance(b1, b2) == p["distance"]
        assert B.distance_pbc(b1, b2, L) == p["distance_pbc"]
        assert bool(B.overlap(b1, b2)) == p["overlap"]
        assert bool(B.overlap_pbc(b1, b2, L)) == p["overlap_pbc"]
        assert bool(B.overlap_pbc(b1, b2, L, 25.0)) == p["overlap_pbc_eps"]


def test_connection_matrix_ids_and_wrapping(golden):
    bs, L = _beads(golden), golden["L"]
    assert B.build_connection_matrix(bs).tolist() == golden["connection_matrix"]
    assert [B.get_bead_with_id(bs, k) for k in (1, 5, 8, 99)] == golden["get_bead_with_id"]
    for b, shift, ref in zip(bs[:2], golden["translate_shifts"], golden["kept_in_box"]):
        b.translate(np.array(shift))
        b.keep_in_box(L)
        assert b.r.tolist() == ref
