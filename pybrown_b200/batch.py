"""Batched replicas: many independent BD systems advanced together on one GPU.

The reference advances one ``Box`` per process (src/bdsim/pyBrown/box.py);
``ReplicaBatch`` holds many such systems -- each with its own beads, box,
temperature and noise stream -- and advances all of them with one sequence of
GPU launches per step (tier 3 of include/pybrown_b200.h).  Each replica
follows ``Box.propagate`` (box.py:150-250) for the ``rpy`` / ``rpy_smith``
hydrodynamics and the Ermak-McCammon scheme: D from the (Smith-Ewald) RPY
tensor, B = chol(D), the deterministic step, then stochastic attempts that
are undone on a bead overlap and redrawn, up to ``max_move_attempts``.

Noise per replica comes either from ``numpy.random.RandomState(seed)`` in the
reference's order (3N normals per attempt, box.py:393-399; for parity with the
reference) or from a counter-based device stream (Philox) keyed by the seed.
Either way a replica's trajectory does not depend on the other replicas in
the batch, so it is the same alone and in a mix.

    batch = ReplicaBatch(precision="mixed")
    s = batch.add(positions, radii, box_length=750.0, seed=0)
    for _ in range(steps):
        batch.propagate(dt=1.0)
    r = batch.positions(s)
"""
import ctypes
import math

import numpy as np

from . import _lib

BOLTZMANN = 1.380649e-23  # scipy.constants.Boltzmann (box.py:636)


class FactorisationError(_lib.PbgError):
    """A step's factorisation failed for some replicas (the step has run for
    all of them, so the failed replicas' moves are not to be trusted).
    slots: {slot: status of the batched factorisation}; recheck: {slot: status
    of a single-matrix factorisation of a copy of the same D} -- a recheck of
    0 means the matrix was positive definite after all."""

    def __init__(self, fn, code, message, slots, recheck):
        super().__init__(fn, code, message)
        self.slots = slots
        self.recheck = recheck


class ReplicaBatch:
    def __init__(self, precision="mixed", hydrodynamics="rpy_smith", ewald_alpha=None, ewald_real=2,
                 ewald_imag=4, stream=None):
        if hydrodynamics not in ("rpy", "rpy_smith"):
            raise ValueError("batched replicas support the rpy and rpy_smith hydrodynamics")
        p = _lib.PbgParams()
        p.precision = _lib.PREC[precision]
        p.hydrodynamics = _lib.HI[hydrodynamics]
        p.propagation_scheme = _lib.SCHEME["ermak"]
        p.ewald_alpha = math.sqrt(math.pi) if ewald_alpha is None else float(ewald_alpha)
        p.ewald_real = int(ewald_real)
        p.ewald_imag = int(ewald_imag)
        self.precision = precision
        self.hydrodynamics = hydrodynamics
        self.ewald_imag = int(ewald_imag)
        self._h = ctypes.c_void_p()
        _lib.call("pbg_batch_create", ctypes.byref(p), ctypes.byref(self._h))
        self._stream = stream
        self._rep = {}

    # ---------------------------------------------------------------- members
    def footprint(self, n_beads):
        """Device bytes one replica of n_beads takes in this batch."""
        return int(_lib.lib.pbg_batch_footprint(_lib.PREC[self.precision], _lib.HI[self.hydrodynamics],
                                                self.ewald_imag, int(n_beads)))

    def add(self, positions, radii, box_length, T=293.15, viscosity=0.01005, seed=0, noise="numpy",
            check_overlaps=True, overlap_treshold=0.0, max_move_attempts=1000000, force=None):
        """Adds a replica; returns its slot id."""
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
        rad = np.ascontiguousarray(np.asarray(radii, dtype=np.float64).reshape(-1))
        if pos.size != 3 * rad.size or rad.size == 0:
            raise ValueError("positions must be N x 3 for N radii")
        if noise not in ("numpy", "device"):
            raise ValueError("noise must be 'numpy' or 'device'")
        p = _lib.PbgParams()
        p.n_beads = int(rad.size)
        p.box_length = float(box_length)
        p.kBT = BOLTZMANN * float(T)
        p.viscosity = float(viscosity)
        p.check_overlaps = int(bool(check_overlaps))
        p.overlap_treshold = float(overlap_treshold)
        p.max_move_attempts = max(1, int(max_move_attempts))
        slot = ctypes.c_int(-1)
        _lib.call("pbg_batch_add", self._h, ctypes.byref(p), pos.ctypes.data, rad.ctypes.data, ctypes.byref(slot))
        s = slot.value
        rec = {"N": int(rad.size), "noise": noise, "max_move_attempts": int(max_move_attempts),
               "last_move_attempts": 0}
        if noise == "numpy":
            rec["rng"] = np.random.RandomState(seed)
        else:
            _lib.call("pbg_batch_set_seed", self._h, s, int(seed) & (2 ** 64 - 1), 0)
        self._rep[s] = rec
        if force is not None:
            self.set_force(s, force)
        return s

    def remove(self, slot):
        _lib.call("pbg_batch_remove", self._h, int(slot))
        del self._rep[slot]

    def slots(self):
        return sorted(self._rep)

    def set_force(self, slot, force):
        if force is None:
            _lib.call("pbg_batch_set_force", self._h, int(slot), None)
            return
        F = np.ascontiguousarray(np.asarray(force, dtype=np.float64).reshape(-1))
        if F.size != 3 * self._rep[slot]["N"]:
            raise ValueError("force must have 3N entries")
        _lib.call("pbg_batch_set_force", self._h, int(slot), F.ctypes.data)

    def set_positions(self, slot, positions):
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
        _lib.call("pbg_batch_set_positions", self._h, int(slot), pos.ctypes.data)

    def positions(self, slot):
        out = np.empty(3 * self._rep[slot]["N"])
        _lib.call("pbg_batch_get_positions", self._h, int(slot), out.ctypes.data)
        return out.reshape(-1, 3)

    def matrix(self, slot, which="D"):
        n = 3 * self._rep[slot]["N"]
        out = np.empty((n, n))
        _lib.call("pbg_batch_get_matrix", self._h, int(slot), _lib.MAT[which], out.ctypes.data)
        return out

    def draws(self, slot):
        """Draws consumed so far by the replica's device noise stream."""
        v = ctypes.c_ulonglong(0)
        _lib.call("pbg_batch_get_draws", self._h, int(slot), ctypes.byref(v))
        return v.value

    def last_move_attempts(self, slot):
        return self._rep[slot]["last_move_attempts"]

    def last_status(self, slot):
        """Factorisation status of the replica in the last step: 0, the first
        non-positive pivot (1-based), or -1 (a wait of the factorisation gave up)."""
        return self._rep[slot].get("last_status", 0)

    # ---------------------------------------------------------------- schedule
    MERGE_ORDERS = ("larger_first", "added", "smaller_first", "replica_major",
                    "chunk_32M", "chunk_64M", "chunk_128M")

    def set_schedule(self, merge_order="larger_first", ctas_per_sm=0):
        """Schedule of the batched factorisation: the interleaving of the
        replicas' task segments and the resident CTAs per SM (0 = as many as
        fit).  No choice changes a result."""
        _lib.call("pbg_batch_set_schedule", self._h, self.MERGE_ORDERS.index(merge_order), int(ctas_per_sm))

    def autotune(self, reps=3):
        """Times the factorisation of the current matrices under every
        schedule (after a step, between steps), keeps the fastest and returns
        {"merge_order", "ctas_per_sm", "ms": {(merge_order, ctas): mean ms}}."""
        n = 2 * len(self.MERGE_ORDERS)
        best = (ctypes.c_int * 2)()
        ms = (ctypes.c_float * n)()
        _lib.call("pbg_batch_autotune", self._h, int(reps), best, ms, self._stream)
        table = {(self.MERGE_ORDERS[k // 2], k % 2 + 1): float(ms[k]) for k in range(n) if ms[k] >= 0}
        return {"merge_order": self.MERGE_ORDERS[best[0]], "ctas_per_sm": int(best[1]), "ms": table}

    def graph_state(self):
        """1 while the start of a step (Ewald build, factorisation,
        deterministic move) replays one CUDA graph, 0 while its kernels are
        launched one by one (the first step after a membership or flag
        change), -1 if the driver refused the capture."""
        return int(_lib.lib.pbg_batch_graph_state(self._h))

    # ---------------------------------------------------------------- step
    def propagate(self, dt, build_D=True, cholesky=True, device_loop=None):
        """One step of every replica (box.py:150-250, Ermak scheme).  When
        every replica draws device noise the whole step -- attempts included
        -- runs on the device (pbg_batch_step: one CUDA graph launch once the
        step repeats); otherwise the attempts are driven from the host, which
        draws the RandomState noise in the reference's order.  device_loop=False
        drives the attempts from the host for device noise too (same results)."""
        if not self._rep:
            return
        h, st = self._h, self._stream
        all_device = all(rec["noise"] == "device" for rec in self._rep.values())
        if device_loop and not all_device:
            raise ValueError("the device loop needs device noise for every replica")
        if all_device and device_loop is not False:
            ns = _lib.lib.pbg_batch_slots(h)
            status = np.zeros(ns, dtype=np.int32)
            attempts = np.zeros(ns, dtype=np.int32)
            rc = _lib.lib.pbg_batch_step(h, float(dt), int(bool(build_D)), int(bool(cholesky)),
                                         status.ctypes.data, attempts.ctypes.data, st)
            for s, rec in self._rep.items():
                rec["last_move_attempts"] = int(attempts[s])
                rec["last_status"] = int(status[s])
            if rc == _lib.PBG_ERR_ATTEMPTS:
                exceeded = [s for s, rec in self._rep.items() if attempts[s] >= rec["max_move_attempts"]]
                raise AssertionError("maximal number of move attepts exceeded (slots {})".format(exceeded))
            self._raise_factorisation("pbg_batch_step", rc)
            return
        _lib.call("pbg_batch_step_begin", h, float(dt), int(bool(build_D)), int(bool(cholesky)), st)
        ns = _lib.lib.pbg_batch_slots(h)
        mask = np.zeros(ns, dtype=np.uint8)
        accepted = np.zeros(ns, dtype=np.uint8)
        pending = sorted(self._rep)
        counts = {s: 0 for s in pending}
        exceeded = []
        while pending:
            mask[:] = 0
            device = []
            for s in pending:
                rec = self._rep[s]
                counts[s] += 1
                mask[s] = 1
                if rec["noise"] == "numpy":
                    xi = rec["rng"].normal(0.0, 1.0, 3 * rec["N"])
                    _lib.call("pbg_batch_set_noise", h, s, xi.ctypes.data)
                else:
                    device.append(s)
            if device:
                dmask = np.zeros(ns, dtype=np.uint8)
                dmask[device] = 1
                _lib.call("pbg_batch_fill_noise", h, dmask.ctypes.data, st)
            _lib.call("pbg_batch_step_attempt", h, mask.ctypes.data, accepted.ctypes.data, st)
            still = []
            for s in pending:
                if accepted[s]:
                    continue
                if counts[s] >= self._rep[s]["max_move_attempts"]:
                    exceeded.append(s)
                else:
                    still.append(s)
            pending = still
        for s, c in counts.items():
            self._rep[s]["last_move_attempts"] = c
        status = np.zeros(ns, dtype=np.int32)
        rc = _lib.lib.pbg_batch_step_end(h, status.ctypes.data, st)
        for s, rec in self._rep.items():
            rec["last_status"] = int(status[s])
        if exceeded:
            raise AssertionError("maximal number of move attepts exceeded (slots {})".format(exceeded))
        self._raise_factorisation("pbg_batch_step_end", rc)

    def _raise_factorisation(self, fn, rc):
        if rc in (_lib.PBG_ERR_NOT_SPD, _lib.PBG_ERR_BARRIER):
            msg = _lib.last_error()
            bad = {s: rec["last_status"] for s, rec in self._rep.items() if rec.get("last_status", 0) != 0}
            recheck = {}
            for s in bad:
                info = ctypes.c_int(0)
                if _lib.lib.pbg_batch_check_factor(self._h, int(s), ctypes.byref(info), self._stream) == _lib.PBG_OK:
                    recheck[s] = info.value
            raise FactorisationError(fn, rc, msg, bad, recheck)
        _lib.check(fn, rc)

    def close(self):
        if self._h:
            _lib.lib.pbg_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
