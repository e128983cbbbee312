"""Beads and periodic geometry (drop-in for pyBrown.bead, src/bdsim/pyBrown/bead.py).

`Bead` keeps the reference's attributes.  The pair-vector matrix and the
overlap test run on the GPU through the reference ABI of libpybrown_b200
(pointer_pbc_matrix, check_overlaps); the small per-bead helpers are host code.
"""
import math

import numpy as np

from ._lib import dptr, iptr, lib

_radius_generation = [0]


def radius_generation():
    """Counter bumped whenever any Bead's radius is set (lets a Box skip
    re-reading every radius before each step)."""
    return _radius_generation[0]


class Bead:
    """Spherical bead (bead.py:30-213): centre `r`, hydrodynamic radius `a`,
    label, mobility, Lennard-Jones parameters and bond bookkeeping."""

    def __init__(self, coords, hydrodynamic_radius, label="XXX", hard_core_radius=None,
                 epsilon_LJ=0.0, mobile=True, bead_id=None):
        self.r = np.array(coords, dtype=float)
        self.a = hydrodynamic_radius
        self.label = label
        self.mobile = mobile
        self.hard_core_radius = hard_core_radius if hard_core_radius is not None else self.a
        self.epsilon_LJ = epsilon_LJ
        self.bead_id = bead_id
        self.bonded_with = []
        self.bonded_how = {}
        self.angled_with = []
        self.angled_how = {}

    @property
    def a(self):
        return self._a

    @a.setter
    def a(self, value):
        self._a = value
        _radius_generation[0] += 1

    def __setstate__(self, state):
        # pickles written before `a` became a property hold it as a plain attribute
        if "a" in state:
            state["_a"] = state.pop("a")
        self.__dict__.update(state)

    def translate(self, vector):
        """bead.py:92-101."""
        if self.mobile:
            self.r += vector

    def keep_in_box(self, box_length):
        """bead.py:170-183: wrap into [-L/2, L/2) by whole box lengths."""
        for i in range(3):
            while self.r[i] < -box_length / 2:
                self.r[i] += box_length
            while self.r[i] >= box_length / 2:
                self.r[i] -= box_length

    def is_there_bond_between(self, bead):
        return bead.bead_id in self.bonded_with or self.bead_id in bead.bonded_with

    def __str__(self):
        mobile_string = "mobile" if self.mobile else "immobile"
        return "{}: {}, radius = {}, {}".format(self.label, self.r, self.a, mobile_string)

    __repr__ = __str__

    def __eq__(self, p):
        if isinstance(p, Bead):
            return bool(np.all(self.r == p.r)) and self.a == p.a
        return False

    __hash__ = object.__hash__


def pointer(bead1, bead2):
    return bead2.r - bead1.r


def _min_image(x, box_size):
    # bead.py:239-244 / bead.c:44-73 while-loop semantics
    while x >= box_size / 2:
        x -= box_size
    while x <= -box_size / 2:
        x += box_size
    return x


def pointer_pbc(bead1, bead2, box_size):
    """Vector from bead1 to the closest replica of bead2 (bead.py:226-246)."""
    r = pointer(bead1, bead2)
    for i in range(3):
        r[i] = _min_image(r[i], box_size)
    return r


def distance(bead1, bead2):
    r = pointer(bead1, bead2)
    return math.sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2])


def distance_pbc(bead1, bead2, box_size):
    r = pointer_pbc(bead1, bead2, box_size)
    return math.sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2])


def overlap(bead1, bead2):
    return distance(bead1, bead2) <= bead1.a + bead2.a


def overlap_pbc(bead1, bead2, box_size, epsilon=0.0):
    return distance_pbc(bead1, bead2, box_size) <= bead1.a + bead2.a + epsilon


def positions_array(beads):
    return np.ascontiguousarray(np.array([b.r for b in beads], dtype=np.float64).reshape(-1))


def compute_pointer_pbc_matrix(beads, box_length):
    """bead.py:282-303: (N, N, 3) minimum-image pair vectors, rij[a][b] ~ r_b - r_a."""
    N = len(beads)
    pos = positions_array(beads)
    rij = np.zeros(3 * N * N, dtype=np.float64)
    lib.pointer_pbc_matrix(dptr(pos), N, float(box_length), dptr(rij))
    return rij.reshape(N, N, 3)


def compute_pointer_immobile_pbc_matrix(mobile_beads, immobile_beads, box_length):
    """bead.py:307-337."""
    n_mob, n_imm = len(mobile_beads), len(immobile_beads)
    pm = positions_array(mobile_beads) if n_mob else np.zeros(0)
    pi = positions_array(immobile_beads) if n_imm else np.zeros(0)
    out = np.zeros(3 * n_mob * n_imm, dtype=np.float64)
    lib.pointer_immobile_pbc_matrix(dptr(pm), dptr(pi), n_mob, n_imm, float(box_length), dptr(out))
    return out.reshape(n_mob, n_imm, 3)


def build_connection_matrix(beads):
    """bead.py:401-413: symmetric int32 matrix, 1 for bonded or both-immobile pairs."""
    n = len(beads)
    cm = np.zeros((n, n), dtype=np.int32)
    for i in range(n):
        for j in range(n):
            if beads[i].is_there_bond_between(beads[j]):
                cm[i][j] = cm[j][i] = 1
            if not (beads[i].mobile or beads[j].mobile):
                cm[i][j] = cm[j][i] = 1
    return cm


def check_overlaps(beads, box_length, overlap_treshold, connection_matrix):
    """bead.py:417-443: True if any non-bonded pair overlaps."""
    pos = positions_array(beads)
    radii = np.ascontiguousarray([b.a for b in beads], dtype=np.float64)
    conn = np.ascontiguousarray(connection_matrix, dtype=np.int32).ravel()
    flag = lib.check_overlaps(dptr(pos), dptr(radii), len(beads), float(box_length),
                              float(overlap_treshold), iptr(conn))
    return flag == 1


def get_bead_with_id(beads, bead_id):
    for i, b in enumerate(beads):
        if b.bead_id == bead_id:
            return i
    return None
