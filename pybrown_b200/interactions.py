"""Inter-bead interactions (drop-in for pyBrown.interactions,
src/bdsim/pyBrown/interactions.py).

The built-in interactions -- Lennard-Jones (lennard_jones_6 / _12), harmonic
bonds and harmonic angles from the .str file -- run on the device: `device_
interactions` turns the beads and the input into the pbg_interactions
descriptor of the C ABI (term lists in the order the reference's loops meet
them, interactions.py:185-414), and every pbg_step_begin evaluates them at the
step-start positions.  Custom interactions (a user's Python file,
interactions.py:591-637) are user code and stay on the host: `Interactions`
evaluates them with the reference's loops and the result joins the external
force.
"""
import ctypes
import importlib
import math
import os
import sys

import numpy as np

from . import _lib


def kcal_per_mole_to_joule(value):
    """interactions.py:823-825."""
    return 10 ** (-21) * 6.9477 * value


def joule_to_kcal_per_mole(value):
    """interactions.py:829-831."""
    return value / (10 ** (-21) * 6.9477)


def eV_to_joule(value):
    """interactions.py:835-837."""
    return 10 ** (-19) * 1.602176634 * value


def joule_to_eV(value):
    """interactions.py:841-843."""
    return value / (10 ** (-19) * 1.602176634)


def to_joule(F, energy_unit):
    """The unit conversion of Box._compute_forces (box.py:414-428)."""
    if energy_unit == "kcal/mol":
        return kcal_per_mole_to_joule(F)
    if energy_unit == "eV":
        return eV_to_joule(F)
    return F


def _index_by_id(beads):
    """get_bead_with_id (bead.py:447-453) as a table: first bead with each id."""
    table = {}
    for i, b in enumerate(beads):
        table.setdefault(b.bead_id, i)
    return table


class Interactions:
    """A force/energy function pair evaluated over the beads on the host
    (interactions.py:57-481); used for custom interactions."""

    def __init__(self, force_function, energy_function, auxiliary_force_parameters=None, bonded=False,
                 how_many_body=2):
        self.force = force_function
        self.energy = energy_function
        self.auxiliary_force_parameters = dict(auxiliary_force_parameters or {})
        self.bonded = bonded
        self.how_many_body = how_many_body

    def compute_forces_and_energy(self, mobile_beads, pointers_mobile, F, immobile_beads=(),
                                  pointers_mobile_immobile=()):
        """Adds this interaction's forces into F (3 per mobile bead) and
        returns its energy (interactions.py:109-165)."""
        assert len(F) == 3 * len(mobile_beads), "ERROR: invalid length of force vector"
        kind = (self.how_many_body, bool(self.bonded))
        args = (mobile_beads, list(immobile_beads), pointers_mobile, pointers_mobile_immobile, F)
        if kind == (1, False):
            return self._one_body(*args)
        if kind == (2, True):
            return self._two_body_bonded(*args)
        if kind == (2, False):
            return self._two_body_nonbonded(*args)
        if kind == (3, True):
            return self._three_body_bonded(*args)
        raise NotImplementedError("{}-body {} interactions are not implemented".format(
            self.how_many_body, "bonded" if self.bonded else "non-bonded"))

    def _f(self, *beads_and_pointers):
        return np.asarray(self.force(*beads_and_pointers, **self.auxiliary_force_parameters), dtype=float)

    def _e(self, *beads_and_pointers):
        return self.energy(*beads_and_pointers, **self.auxiliary_force_parameters)

    # interactions.py:169-181
    def _one_body(self, mob, imm, rij, rik, F):
        E = 0.0
        for i, b in enumerate(mob):
            F[3 * i:3 * i + 3] += self._f(b)
            E += self._e(b)
        return E

    # interactions.py:185-245
    def _two_body_bonded(self, mob, imm, rij, rik, F):
        E = 0.0
        mob_id, imm_id = _index_by_id(mob), _index_by_id(imm)
        for i, bi in enumerate(mob):
            for idx in bi.bonded_with:
                j = mob_id.get(idx)
                if j is not None:
                    p = rij[i][j]
                    f = self._f(bi, mob[j], p)
                    F[3 * i:3 * i + 3] += f
                    F[3 * j:3 * j + 3] -= f
                    E += self._e(bi, mob[j], p)
                else:
                    k = imm_id[idx]
                    p = rik[i][k]
                    F[3 * i:3 * i + 3] += self._f(bi, imm[k], p)
                    E += self._e(bi, imm[k], p)
        for k, bk in enumerate(imm):
            for idx in bk.bonded_with:
                j = mob_id.get(idx)
                if j is not None:
                    p = -rik[j][k]
                    F[3 * j:3 * j + 3] -= self._f(bk, mob[j], p)
                    E += self._e(bk, mob[j], p)
        return E

    # interactions.py:249-287
    def _two_body_nonbonded(self, mob, imm, rij, rik, F):
        E = 0.0
        for i in range(1, len(mob)):
            for j in range(i):
                p = rij[i][j]
                f = self._f(mob[i], mob[j], p)
                F[3 * i:3 * i + 3] += f
                F[3 * j:3 * j + 3] -= f
                E += self._e(mob[i], mob[j], p)
        for i in range(len(mob)):
            for k in range(len(imm)):
                p = rik[i][k]
                F[3 * i:3 * i + 3] += self._f(mob[i], imm[k], p)
                E += self._e(mob[i], imm[k], p)
        return E

    # interactions.py:291-414
    def _three_body_bonded(self, mob, imm, rij, rik, F):
        E = 0.0
        mob_id, imm_id = _index_by_id(mob), _index_by_id(imm)
        for i, bi in enumerate(mob):
            for idx1, idx2 in bi.angled_with:
                j, k = mob_id.get(idx1), mob_id.get(idx2)
                if j is not None:
                    bj, p12 = mob[j], rij[i][j]
                else:
                    j = imm_id[idx1]
                    bj, p12 = imm[j], rik[i][j]
                if k is not None:
                    bk = mob[k]
                    p23 = rij[j][k] if bj.mobile else -rik[k][j]
                else:
                    k = imm_id[idx2]
                    bk = imm[k]
                    p23 = rik[j][k] if bj.mobile else rik[i][k] - p12
                f = self._f(bi, bj, bk, p12, p23)
                F[3 * i:3 * i + 3] += f[:3]
                if bj.mobile:
                    F[3 * j:3 * j + 3] += f[3:6]
                if bk.mobile:
                    F[3 * k:3 * k + 3] += f[6:]
                E += self._e(bi, bj, bk, p12, p23)
        for i, bi in enumerate(imm):
            for idx1, idx2 in bi.angled_with:
                j, k = mob_id.get(idx1), mob_id.get(idx2)
                if j is None and k is None:
                    continue
                if j is not None and k is not None:
                    bj, bk = mob[j], mob[k]
                    p12, p23 = -rik[j][i], rij[j][k]
                elif j is not None:
                    bj = mob[j]
                    k = imm_id[idx2]
                    bk = imm[k]
                    p12, p23 = -rik[j][i], rik[j][k]
                else:
                    j = imm_id[idx1]
                    bj, bk = imm[j], mob[k]
                    p23 = -rik[k][j]
                    p12 = -rik[k][i] - p23
                f = self._f(bi, bj, bk, p12, p23)
                if bj.mobile:
                    F[3 * j:3 * j + 3] += f[3:6]
                if bk.mobile:
                    F[3 * k:3 * k + 3] += f[6:]
                E += self._e(bi, bj, bk, p12, p23)
        return E


def set_custom_interactions(input_data):
    """Loads the custom-interactions file (interactions.py:591-637): every
    pair of functions <name>_force / <name>_energy becomes one Interactions;
    "bonded" among the '_'-separated words of <name> makes it bonded and the
    word before the last, minus its final letter, is the body count."""
    if not input_data.get("custom_interactions"):
        return []
    filename = input_data["custom_interactions_filename"]
    location, modulename = os.path.split(filename)
    aux = input_data.get("auxiliary_custom_interactions_keywords", {})
    sys.path.append(location)
    try:
        module = importlib.import_module(modulename.split(".")[0])
    finally:
        sys.path.pop()
    energy = {n[:-6]: n for n in dir(module) if not n.startswith("_") and n.endswith("energy")}
    force = {n[:-5]: n for n in dir(module) if not n.startswith("_") and n.endswith("force")}
    assert len(energy) == len(force), "unequal number of energy and force functions in custom interactions file"
    assert energy.keys() == force.keys(), "different names of force and energy functions in custom interactions file"
    out = []
    for key in energy:
        bonded = "bonded" in key.split("_")
        how_many_body = int(key.split("_")[-2][:-1])
        out.append(Interactions(getattr(module, force[key]), getattr(module, energy[key]), aux,
                                bonded=bonded, how_many_body=how_many_body))
    return out


class DeviceInteractions:
    """The pbg_interactions descriptor of the built-in interactions of a box
    (interactions.py:483-589) and the arrays it points to."""

    def __init__(self, input_data, mobile_beads, immobile_beads):
        N = len(mobile_beads)
        beads = list(mobile_beads) + list(immobile_beads)
        mob_id, imm_id = _index_by_id(mobile_beads), _index_by_id(immobile_beads)
        lj = _lib.LJ[(bool(input_data.get("lennard_jones_6")), bool(input_data.get("lennard_jones_12")))]
        self.hc = np.ascontiguousarray([b.hard_core_radius for b in beads], dtype=np.float64)
        self.eps = np.ascontiguousarray([b.epsilon_LJ for b in beads], dtype=np.float64)
        bonds, bond_params, angles, angle_params = [], [], [], []
        # interactions.py:185-245: each listed bond once, force +f on the first
        # bead and -f on the second where they are mobile.
        for i, bi in enumerate(mobile_beads):
            for idx in bi.bonded_with:
                j = mob_id.get(idx)
                bonds.append((i, j if j is not None else N + imm_id[idx]))
                bond_params.append(bi.bonded_how[idx])
        for k, bk in enumerate(immobile_beads):
            for idx in bk.bonded_with:
                j = mob_id.get(idx)
                if j is not None:
                    bonds.append((N + k, j))
                    bond_params.append(bk.bonded_how[idx])
        # interactions.py:291-414 with the pair-vector form of each branch.
        for i, bi in enumerate(mobile_beads):
            for idx1, idx2 in bi.angled_with:
                j, k = mob_id.get(idx1), mob_id.get(idx2)
                jj = j if j is not None else N + imm_id[idx1]
                kk = k if k is not None else N + imm_id[idx2]
                form = _lib.ANGLE_P23_DIFF if (j is None and k is None) else _lib.ANGLE_DIRECT
                angles.append((i, jj, kk, form))
                angle_params.append(bi.angled_how[(idx1, idx2)])
        for m, bm in enumerate(immobile_beads):
            for idx1, idx2 in bm.angled_with:
                j, k = mob_id.get(idx1), mob_id.get(idx2)
                if j is None and k is None:
                    continue
                if j is not None and k is not None:
                    angles.append((N + m, j, k, _lib.ANGLE_DIRECT))
                elif j is not None:
                    angles.append((N + m, j, N + imm_id[idx2], _lib.ANGLE_DIRECT))
                else:
                    angles.append((N + m, N + imm_id[idx1], k, _lib.ANGLE_P12_DIFF))
                angle_params.append(bm.angled_how[(idx1, idx2)])
        self.bonds = np.ascontiguousarray(np.array(bonds, dtype=np.int32).reshape(-1))
        self.bond_params = np.ascontiguousarray(np.array(bond_params, dtype=np.float64).reshape(-1))
        self.angles = np.ascontiguousarray(np.array(angles, dtype=np.int32).reshape(-1))
        self.angle_params = np.ascontiguousarray(np.array(angle_params, dtype=np.float64).reshape(-1))
        self.active = bool(lj or bonds or angles)
        d = _lib.PbgInteractions()
        d.lennard_jones = lj
        d.lennard_jones_alpha = float(input_data.get("lennard_jones_alpha", 4.0)) if lj else 0.0
        d.hard_core_radius = self.hc.ctypes.data if lj else None
        d.epsilon_lj = self.eps.ctypes.data if lj else None
        d.n_bonds = len(bonds)
        d.bonds = self.bonds.ctypes.data if bonds else None
        d.bond_params = self.bond_params.ctypes.data if bonds else None
        d.n_angles = len(angles)
        d.angles = self.angles.ctypes.data if angles else None
        d.angle_params = self.angle_params.ctypes.data if angles else None
        d.unit_scale = float(to_joule(1.0, input_data.get("energy_unit", "joule")))
        self.desc = d

    def install(self, handle):
        _lib.call("pbg_set_interactions", handle, ctypes.byref(self.desc))
