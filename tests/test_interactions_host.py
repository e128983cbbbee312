"""Host logic of the interactions module (no GPU): the device term lists
follow the reference's loop order and pair-vector forms
(interactions.py:185-414), and the host Interactions class used for custom
interactions adds the same forces as the oracle's restatement."""
import numpy as np

from test_forces_oracle import custom_terms, fixture_case


def _split(beads, inp):
    labels = inp.get("immobile_labels", [])
    for b in beads:
        b.mobile = b.label not in labels
    return [b for b in beads if b.mobile], [b for b in beads if not b.mobile]


def test_device_term_lists(forces_golden):
    from pybrown_b200 import _lib
    from pybrown_b200.interactions import DeviceInteractions
    beads, inp = fixture_case(forces_golden, "forces_chain_rpy")
    mob, imm = _split(beads, inp)
    d = DeviceInteractions(inp, mob, imm)
    N = len(mob)
    mid = {b.bead_id: i for i, b in enumerate(mob)}
    iid = {b.bead_id: N + i for i, b in enumerate(imm)}
    idx = {**mid, **iid}
    bonds = d.bonds.reshape(-1, 2).tolist()
    # each mobile bead's bond list in bead order, then the immobile beads' bonds to mobile beads
    expected = [(1, 2), (2, 3), (2, 100), (3, 4), (4, 5), (5, 6), (6, 7), (101, 4)]
    assert bonds == [[idx[a], idx[b]] for a, b in expected]
    ang = {tuple(a[:3]): a[3] for a in d.angles.reshape(-1, 4).tolist()}
    assert ang[(idx[1], idx[100], idx[101])] == _lib.ANGLE_P23_DIFF
    assert ang[(idx[101], idx[100], idx[3])] == _lib.ANGLE_P12_DIFF
    assert ang[(idx[102], idx[6], idx[101])] == _lib.ANGLE_DIRECT
    assert ang[(idx[5], idx[101], idx[6])] == _lib.ANGLE_DIRECT
    assert d.desc.lennard_jones == 612 and d.desc.n_angles == 9
    assert d.desc.unit_scale == 10 ** (-21) * 6.9477
    assert d.hc.tolist() == [b.hard_core_radius for b in mob + imm]


def test_no_interactions_is_inactive(forces_golden):
    from pybrown_b200.interactions import DeviceInteractions
    beads, inp = fixture_case(forces_golden, "forces_custom_smith")
    mob, imm = _split(beads, inp)
    inp = dict(inp, lennard_jones_12=False)
    assert not DeviceInteractions(inp, mob, imm).active


def test_host_custom_interactions_match_oracle(forces_golden, oracle_lib):
    from oracle.oracle import OracleForceBox
    from pybrown_b200.interactions import set_custom_interactions
    beads, inp = fixture_case(forces_golden, "forces_custom_smith")
    inp = dict(inp, lennard_jones_12=False, external_force=[0.0, 0.0, 0.0], energy_unit="joule")
    ref = OracleForceBox(beads, inp, clib=oracle_lib, custom=custom_terms(inp))
    ref._forces()
    mob, imm = _split(beads, inp)
    rij = oracle_lib.pointers(np.array([b.r for b in mob]), inp["box_length"])
    F = np.zeros(3 * len(mob))
    E = 0.0
    for it in set_custom_interactions(inp):
        E += it.compute_forces_and_energy(mobile_beads=mob, pointers_mobile=rij, F=F)
    assert np.allclose(F, ref.F, rtol=1e-14, atol=0)
    assert abs(E - ref.E) <= 1e-14 * abs(ref.E)
