"""Simulation box (drop-in for pyBrown.box.Box, src/bdsim/pyBrown/box.py).

`Box(beads, input_data).propagate(dt, build_Dff, build_Dnf, cholesky)` runs
one Brownian (Ermak-McCammon) or Stokesian (midpoint) step exactly as the
reference orders it (box.py:150-389), but every tensor lives in HBM inside a
`pbg_system` handle of libpybrown_b200 and every kernel is sm_100a code:
the RPY / Smith-Ewald tensor, the Jeffrey-Onishi lubrication correction, the
SPD inverses, the Cholesky factor, the matrix-vector products, the overlap
test and the wrap into the box.

The inter-bead forces of the reference (Lennard-Jones, harmonic bonds and
angles, interactions.py) are evaluated on the device at the start of each
step; immobile beads (immobile_labels) stay fixed and take part in the
overlap test and the forces, while D, B and the noise cover the mobile beads
only, as in the reference.

The host keeps what the reference keeps on the host: the RandomState noise
stream (drawn 3N at a time in the reference's order, box.py:393-399), the
accept/reject loop over move attempts, the Bead objects and custom
interactions (user Python code, evaluated with the reference's loops and
added to the external force).  The mobile beads' Bead.r arrays are views into
one (N, 3) array that is refreshed from the device after each step, so
`box.beads` always shows current positions.  Modify bead positions in place
(Bead.translate does) or call `sync_positions_from_beads()`.

Keywords beyond the reference's: "precision": "fp64" (default) or "mixed"
(FP32 Ewald tensor and Cholesky trailing updates, FP64 diagonal tiles and
position accumulation).
"""
import ctypes
import math

import numpy as np
from scipy.constants import Boltzmann

from . import _lib
from .bead import (Bead, build_connection_matrix, check_overlaps, compute_pointer_immobile_pbc_matrix,
                   compute_pointer_pbc_matrix, radius_generation)
from .interactions import DeviceInteractions, eV_to_joule, kcal_per_mole_to_joule, set_custom_interactions, to_joule

__all__ = ["Box", "eV_to_joule", "kcal_per_mole_to_joule"]

_OUT_OF_SCOPE = ("walls", "measure_flux", "measure_concentration", "external_force_region")


class Box:
    """Device-resident simulation box; see the module docstring."""

    def __init__(self, beads, input_data):
        self.beads = beads
        self.inp = input_data
        self.box_length = self.inp["box_length"]
        self._initialize_pseudorandom_number_generation()
        self._handle_bead_mobility()
        self._handle_bead_labels()
        self._set_physical_constants()
        self.hydrodynamics = self.inp["hydrodynamics"]
        if self.hydrodynamics not in _lib.HI:
            raise ValueError("unknown hydrodynamics {!r}".format(self.hydrodynamics))
        if self.hydrodynamics in ("rpy_smith", "rpy_smith_lub"):
            self.alpha = self.inp["ewald_alpha"]
            self.m_max = self.inp["ewald_real"]
            self.n_max = self.inp["ewald_imag"]
        if self.hydrodynamics in ("rpy_lub", "rpy_smith_lub"):
            self.lubrication_cutoff = self.inp["lubrication_cutoff"]
            self.cichocki_correction = self.inp["cichocki_correction"]
        self.propagation_scheme = self.inp["propagation_scheme"]
        if self.propagation_scheme == "midpoint":
            self.m_midpoint = self.inp["m_midpoint"]
            if self.hydrodynamics == "nohi":
                raise ValueError("the midpoint scheme needs hydrodynamic interactions")
        self.precision = self.inp.get("precision", "fp64")
        if self.precision not in _lib.PREC:
            raise ValueError("precision must be 'fp64' or 'mixed'")
        for key in _OUT_OF_SCOPE:
            if key in self.inp:
                raise NotImplementedError("keyword {!r} is outside the accelerated hot path".format(key))
        # box.py:731-733 (interactions.py:483-515): built-in terms on the device,
        # custom ones on the host.
        self.custom_interactions = set_custom_interactions(self.inp)
        self.interactions = list(self.custom_interactions)
        self._device_interactions = DeviceInteractions(self.inp, self.mobile_beads, self.immobile_beads)
        self.reactions = []
        self.end_simulation = False
        self.is_energy = "enr_write_freq" in self.inp
        self.is_flux = self.is_concentration = self.is_wall = False
        self._h = None
        self.E = 0.0

        self.overlaps = self.inp["check_overlaps"]
        self.connection_matrix = build_connection_matrix(self.beads)
        self._has_bonds = bool(self.connection_matrix.any())
        if self.overlaps:
            assert not self._check_overlaps(), "starting configuration contains overlaps"

        self.Fex = np.array(self.inp["external_force"], dtype=float)
        self.F = np.zeros(3 * len(self.mobile_beads))
        self._device_force = None
        self.N = None
        self._create_device_state()

    # ------------------------------------------------------------------ setup

    def _initialize_pseudorandom_number_generation(self):
        """box.py:621-629."""
        if self.inp["seed"] is None:
            self.seed = np.random.randint(2 ** 32 - 1)
        else:
            self.seed = self.inp["seed"]
        self.pseudorandom_number_generator = np.random.RandomState(self.seed)
        self.draw_count = 0

    def _set_physical_constants(self):
        """box.py:633-637."""
        self.T = self.inp["T"]
        self.kBT = Boltzmann * self.T
        self.viscosity = self.inp["viscosity"]

    def _handle_bead_mobility(self):
        """box.py:649-668."""
        self.immobile_labels = self.inp["immobile_labels"]
        for bead in self.beads:
            if bead.label in self.immobile_labels:
                bead.mobile = False
        self.mobile_beads = [b for b in self.beads if b.mobile]
        self.immobile_beads = [b for b in self.beads if not b.mobile]
        self.mobile_bead_indices = [i for i, b in enumerate(self.beads) if b.mobile]
        self.immobile_bead_indices = [i for i, b in enumerate(self.beads) if not b.mobile]

    def _handle_bead_labels(self):
        self.labels = []
        self.mobile_labels = []
        for bead in self.beads:
            if bead.label not in self.labels:
                self.labels.append(bead.label)
                if bead.mobile:
                    self.mobile_labels.append(bead.label)

    def _params(self):
        p = _lib.PbgParams()
        p.n_beads = len(self.mobile_beads)
        p.hydrodynamics = _lib.HI[self.hydrodynamics]
        p.precision = _lib.PREC[self.precision]
        p.propagation_scheme = _lib.SCHEME[self.propagation_scheme]
        p.box_length = float(self.box_length)
        p.kBT = float(self.kBT)
        p.viscosity = float(self.viscosity)
        p.ewald_alpha = float(getattr(self, "alpha", math.sqrt(math.pi)))
        p.ewald_real = int(getattr(self, "m_max", 0))
        p.ewald_imag = int(getattr(self, "n_max", 0))
        p.lubrication_cutoff = float(getattr(self, "lubrication_cutoff", 1.0))
        p.cichocki_correction = 1 if getattr(self, "cichocki_correction", True) else 0
        p.check_overlaps = 1 if self.overlaps else 0
        p.overlap_treshold = float(self.inp["overlap_treshold"])
        p.max_move_attempts = int(min(self.inp["max_move_attempts"], 2 ** 31 - 1))
        p.m_midpoint = float(getattr(self, "m_midpoint", 1.0))
        return p

    def _create_device_state(self, matrices=None):
        self._stream = None  # legacy default stream
        self._h = None
        self._device_force = None
        mob = self.mobile_beads
        N = len(mob)
        self._pos = np.ascontiguousarray(np.array([b.r for b in mob], dtype=np.float64).reshape(N, 3))
        for i, b in enumerate(mob):
            b.r = self._pos[i]
        self._radii = np.ascontiguousarray([b.a for b in mob], dtype=np.float64)
        self._pos_synced = self._pos.copy()  # positions the device holds
        self._radius_gen = radius_generation()
        self._own_beads = all(type(b) is Bead for b in mob)
        self._force_key = None
        if N == 0:
            return  # box.py:176: nothing moves
        handle = _lib.ctypes.c_void_p()
        params = self._params()
        _lib.call("pbg_create", _lib.ctypes.byref(params), _lib.ctypes.byref(handle))
        self._h = handle
        if self.inp.get("divergence_term"):
            # box.py:211-215: only the lubrication modes under Ermak use it;
            # the library ignores it elsewhere, as the reference does.
            _lib.call("pbg_set_divergence", self._h, 1)
        conn = np.asarray(self.connection_matrix, dtype=np.int32)
        mi, ii = self.mobile_bead_indices, self.immobile_bead_indices
        conn_mm = conn[np.ix_(mi, mi)]
        self._conn = np.ascontiguousarray(conn_mm) if conn_mm.any() else None
        _lib.call("pbg_set_state", self._h, self._pos.ctypes.data, self._radii.ctypes.data,
                  self._conn.ctypes.data if self._conn is not None else None, self._stream)
        if ii:
            pos_imm = np.ascontiguousarray([b.r for b in self.immobile_beads], dtype=np.float64).reshape(-1)
            radii_imm = np.ascontiguousarray([b.a for b in self.immobile_beads], dtype=np.float64)
            order = np.ascontiguousarray(mi + ii, dtype=np.int32)
            conn_mi = np.ascontiguousarray(conn[np.ix_(mi, ii)])
            _lib.call("pbg_set_immobile", self._h, len(ii), pos_imm.ctypes.data, radii_imm.ctypes.data,
                      order.ctypes.data, conn_mi.ctypes.data if conn_mi.any() else None, self._stream)
        if self._device_interactions.active:
            self._device_interactions.install(self._h)
        if matrices:
            for name, arr in matrices.items():
                arr = np.ascontiguousarray(arr, dtype=np.float64)
                _lib.call("pbg_set_matrix", self._h, _lib.MAT[name], arr.ctypes.data, self._stream)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib.pbg_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------------ step

    def propagate(self, dt, build_Dff=True, build_Dnf=True, cholesky=True):
        """One step (box.py:150-198) on the GPU."""
        if self._h is None:
            return
        self._upload_positions()
        self._compute_forces()
        h, st = self._h, self._stream
        _lib.call("pbg_step_begin", h, float(dt), int(bool(build_Dff)), int(bool(build_Dnf)),
                  int(bool(cholesky)), st)
        count_move_attempts = 0
        accepted = _lib.ctypes.c_int(0)
        while True:
            count_move_attempts += 1
            self._generate_random_vector()
            _lib.call("pbg_step_attempt", h, self.N.ctypes.data, _lib.ctypes.byref(accepted), st)
            if accepted.value:
                break
            assert count_move_attempts < self.inp["max_move_attempts"], \
                "maximal number of move attepts exceeded"
        self.last_move_attempts = count_move_attempts
        _lib.call("pbg_step_finish", h, self._pos.ctypes.data, st)
        self._pos_synced[...] = self._pos
        if self.inp["verbose"]:
            print("move attempts: {}".format(count_move_attempts))

    def _generate_random_vector(self):
        """box.py:393-399."""
        self.N = self.pseudorandom_number_generator.normal(0.0, 1.0, 3 * len(self.mobile_beads))
        self.draw_count += 3 * len(self.mobile_beads)

    def _prepare_external_force(self):
        """box.py:452-460."""
        self.F = np.tile(np.asarray(self.Fex, dtype=float), len(self.mobile_beads))

    def _compute_forces(self):
        """box.py:404-428.  The external force and the custom interactions are
        summed here; pbg_step_begin adds the built-in interactions."""
        self.E = 0.0
        if not self.custom_interactions:
            # the base force depends on Fex and the unit only: upload it when they change
            key = (np.asarray(self.Fex, dtype=float).tobytes(), self.inp["energy_unit"])
            if key == self._force_key:
                return
            self._force_key = key
        self._prepare_external_force()
        if self.custom_interactions:
            rij = compute_pointer_pbc_matrix(self.mobile_beads, self.box_length)
            rik = (compute_pointer_immobile_pbc_matrix(self.mobile_beads, self.immobile_beads, self.box_length)
                   if self.immobile_beads else [])
            F = self._F
            for interaction in self.custom_interactions:
                self._E_host += interaction.compute_forces_and_energy(
                    mobile_beads=self.mobile_beads, pointers_mobile=rij, F=F,
                    immobile_beads=self.immobile_beads, pointers_mobile_immobile=rik)
        self.F = to_joule(self._F, self.inp["energy_unit"])
        F = np.ascontiguousarray(self._F, dtype=np.float64)
        if self._device_force is None or not np.array_equal(F, self._device_force):
            _lib.call("pbg_set_force", self._h, F.ctypes.data, self._stream)
            self._device_force = F.copy()

    def _check_overlaps(self):
        return check_overlaps(self.beads, self.box_length, self.inp["overlap_treshold"], self.connection_matrix)

    def _upload_positions(self):
        """Sends what the caller changed since the last step: radii (rarely;
        a Bead bumps a counter when its radius is set) and positions."""
        gen = radius_generation()
        if gen != self._radius_gen or not self._own_beads:
            self._radius_gen = gen
            radii = [b.a for b in self.mobile_beads]
            if not np.array_equal(radii, self._radii):
                self._radii = np.ascontiguousarray(radii, dtype=np.float64)
                _lib.call("pbg_set_state", self._h, self._pos.ctypes.data, self._radii.ctypes.data,
                          self._conn.ctypes.data if self._conn is not None else None, self._stream)
                self._pos_synced[...] = self._pos
                return
        if not np.array_equal(self._pos, self._pos_synced):
            _lib.call("pbg_set_positions", self._h, self._pos.ctypes.data, self._stream)
            self._pos_synced[...] = self._pos

    def positions(self):
        """A copy of every bead's position (bead order, N x 3)."""
        if not self.immobile_beads:
            return self._pos.copy()
        return np.array([b.r for b in self.beads], dtype=np.float64)

    def sync_positions_from_beads(self):
        """Re-link Bead.r to the box after a caller replaced a bead's r array."""
        for i, b in enumerate(self.mobile_beads):
            if b.r is not self._pos[i] and not (b.r.base is self._pos):
                self._pos[i] = b.r
                b.r = self._pos[i]

    def _keep_beads_in_box(self):
        # Done on the device at the end of each step (box.py:614-617).
        pass

    # ------------------------------------------------------------------ views

    def _matrix(self, name):
        n = 3 * len(self.mobile_beads)
        out = np.empty((n, n), dtype=np.float64)
        _lib.call("pbg_get_matrix", self._h, _lib.MAT[name], out.ctypes.data, self._stream)
        return out

    @property
    def E(self):
        """Interaction energy at the start of the last step (box.py:406-412)."""
        e = self._E_host
        if self._h is not None and self._device_interactions.active:
            v = ctypes.c_double(0.0)
            _lib.call("pbg_get_energy", self._h, ctypes.byref(v), self._stream)
            e += v.value
        return e

    @E.setter
    def E(self, value):
        self._E_host = value

    @property
    def F(self):
        """Force vector of the last step in joules (box.py:404-428)."""
        if self._h is not None and self._device_interactions.active:
            out = np.empty(3 * len(self.mobile_beads), dtype=np.float64)
            _lib.call("pbg_get_force", self._h, out.ctypes.data, self._stream)
            return out
        return self._F

    @F.setter
    def F(self, value):
        self._F = value

    @property
    def D(self):
        return self._matrix("D")

    @property
    def B(self):
        return self._matrix("B")

    @property
    def Mff(self):
        return self._matrix("Mff")

    @property
    def Rff(self):
        return self._matrix("Rff")

    @property
    def R(self):
        return self._matrix("R")

    @property
    def rij(self):
        return compute_pointer_pbc_matrix(self.mobile_beads, self.box_length)

    # ------------------------------------------------------------------ pickling

    def __getstate__(self):
        """Restart files (output.py:72-84) carry the device state as host arrays."""
        state = {k: v for k, v in self.__dict__.items()
                 if k not in ("_h", "_stream", "_pos", "_pos_synced", "_device_force", "_device_interactions",
                              "custom_interactions", "interactions", "_force_key")}
        mats = {"D": self.D, "B": self.B}
        if self.hydrodynamics in ("rpy_lub", "rpy_smith_lub"):
            mats.update(Mff=self.Mff, Rff=self.Rff, R=self.R)
        state["_device_matrices"] = mats
        return state

    def __setstate__(self, state):
        mats = state.pop("_device_matrices", None)
        self.__dict__.update(state)
        self.custom_interactions = set_custom_interactions(self.inp)
        self.interactions = list(self.custom_interactions)
        self._device_interactions = DeviceInteractions(self.inp, self.mobile_beads, self.immobile_beads)
        self._create_device_state(matrices=mats)

    def __str__(self):
        return "simulation box"
