"""CPU oracle: ctypes front end of a library with pyBrown's C ABI, plus a
NumPy restatement of Box.propagate for the hydrodynamic hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.

Libraries it can drive (both export the reference's symbols, diff_tensor.c /
bead.c):
  * oracle/_build/libpybrown_oracle.so -- the in-house C restatement
  * oracle/_build/libpybrown_oracle_omp.so -- the same on all host cores
  * oracle/_ref/libpyBrown.so          -- the reference's own C compiled here
  * oracle/_ref/libpyBrown_omp.so      -- the same with OpenMP
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libpybrown_oracle.so")
ORACLE_OMP_LIB = os.path.join(HERE, "_build", "libpybrown_oracle_omp.so")
REF_LIB = os.path.join(HERE, "_ref", "libpyBrown.so")
REF_OMP_LIB = os.path.join(HERE, "_ref", "libpyBrown_omp.so")

BOLTZMANN = 1.380649e-23  # scipy.constants.Boltzmann (exact SI value)

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class CLib:
    """Functions of diffusion.py / bead.py (src/bdsim/pyBrown) over a pyBrown-ABI library."""

    def __init__(self, path=ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle)")
        self.path = path
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.RPY_M_matrix.argtypes = [_dp, _dp, ctypes.c_int, _dp]
        L.RPY_Smith_M_matrix.argtypes = [_dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, _dp]
        L.JO_2B_R_matrix.argtypes = [ctypes.c_double] * 5 + [_dp]
        L.JO_R_lubrication_correction_matrix.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_double,
                                                         ctypes.c_int, _dp]
        L.pointer_pbc_matrix.argtypes = [_dp, ctypes.c_int, ctypes.c_double, _dp]
        L.check_overlaps.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, _ip]
        L.check_overlaps.restype = ctypes.c_int
        L.pointer_immobile_pbc_matrix.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp]
        L.pointer_immobile_pbc_matrix.restype = None
        for f in ("RPY_M_matrix", "RPY_Smith_M_matrix", "JO_2B_R_matrix",
                  "JO_R_lubrication_correction_matrix", "pointer_pbc_matrix"):
            getattr(L, f).restype = None

    @staticmethod
    def _d(a):
        return a.ctypes.data_as(_dp)

    def pointers(self, pos, L):
        """bead.c:27-95 -> (N, N, 3)."""
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        N = pos.size // 3
        out = np.zeros(3 * N * N)
        self.lib.pointer_pbc_matrix(self._d(pos), N, float(L), self._d(out))
        return out.reshape(N, N, 3)

    @staticmethod
    def packed(pointers):
        N = pointers.shape[0]
        return np.ascontiguousarray(-pointers[np.triu_indices(n=N, k=1)]).reshape(-1)

    def rpy(self, radii, pointers):
        radii = np.ascontiguousarray(radii, dtype=np.float64)
        N = radii.size
        p = self.packed(pointers)
        M = np.zeros(9 * N * N)
        self.lib.RPY_M_matrix(self._d(radii), self._d(p), N, self._d(M))
        return M.reshape(3 * N, 3 * N)

    def smith(self, radii, pointers, L, alpha, m, n):
        radii = np.ascontiguousarray(radii, dtype=np.float64)
        N = radii.size
        p = self.packed(pointers)
        M = np.zeros(9 * N * N)
        self.lib.RPY_Smith_M_matrix(self._d(radii), self._d(p), float(L), float(alpha), int(m), int(n), N,
                                    self._d(M))
        return M.reshape(3 * N, 3 * N)

    def jo2b(self, ai, aj, r):
        out = np.zeros(18)
        self.lib.JO_2B_R_matrix(float(ai), float(aj), float(r[0]), float(r[1]), float(r[2]), self._d(out))
        return out

    def lubrication(self, radii, pointers, cutoff, cichocki):
        radii = np.ascontiguousarray(radii, dtype=np.float64)
        N = radii.size
        p = self.packed(pointers)
        C = np.zeros(9 * N * N)
        self.lib.JO_R_lubrication_correction_matrix(self._d(radii), self._d(p), N, float(cutoff),
                                                    1 if cichocki else 0, self._d(C))
        return C.reshape(3 * N, 3 * N)

    def overlaps(self, pos, radii, L, thr, conn=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        radii = np.ascontiguousarray(radii, dtype=np.float64)
        N = radii.size
        if conn is None:
            conn = np.zeros((N, N), dtype=np.int32)
        conn = np.ascontiguousarray(conn, dtype=np.int32).ravel()
        return self.lib.check_overlaps(self._d(pos), self._d(radii), N, float(L), float(thr),
                                       conn.ctypes.data_as(_ip)) == 1

    def pointers_immobile(self, pos_mobile, pos_immobile, L):
        """bead.c:99-158 -> (N_mobile, N_immobile, 3)."""
        pm = np.ascontiguousarray(pos_mobile, dtype=np.float64).reshape(-1)
        pi = np.ascontiguousarray(pos_immobile, dtype=np.float64).reshape(-1)
        n, m = pm.size // 3, pi.size // 3
        out = np.zeros(3 * n * m)
        self.lib.pointer_immobile_pbc_matrix(self._d(pm), self._d(pi), n, m, float(L), self._d(out))
        return out.reshape(n, m, 3)


class OracleBox:
    """NumPy restatement of Box.propagate for the hot path (box.py:150-617):
    nohi / rpy / rpy_smith / rpy_lub / rpy_smith_lub, Ermak and midpoint,
    overlap rejection, RandomState noise in the reference's order."""

    def __init__(self, positions, radii, inp, clib=None):
        self.c = clib or CLib()
        self.pos = np.array(positions, dtype=np.float64).reshape(-1, 3).copy()
        self.radii = np.asarray(radii, dtype=np.float64)
        self.inp = dict(inp)
        self.L = float(inp["box_length"])
        self.hydro = inp["hydrodynamics"]
        self.scheme = inp.get("propagation_scheme", "ermak")
        self.kBT = BOLTZMANN * inp["T"]
        self.eta = inp["viscosity"]
        self.alpha = inp.get("ewald_alpha", math.sqrt(math.pi))
        self.m_max = inp.get("ewald_real", 0)
        self.n_max = inp.get("ewald_imag", 0)
        self.cutoff = inp.get("lubrication_cutoff", 1)
        self.cich = inp.get("cichocki_correction", True)
        self.m = inp.get("m_midpoint", 100)
        self.overlaps = inp.get("check_overlaps", True)
        self.thr = inp.get("overlap_treshold", 0.0)
        self.max_attempts = inp.get("max_move_attempts", 1000000)
        seed = inp.get("seed", 0)
        self.rng = np.random.RandomState(seed)
        self.draw_count = 0
        Fex = np.array(inp.get("external_force", [0.0, 0.0, 0.0]), dtype=float)
        self.F = np.array(list(Fex) * len(self.radii))
        self.attempt_log = []
        if self.hydro == "nohi":
            self._dff()
            self.B = np.sqrt(self.D)

    # box.py:486-528
    def _dff(self):
        if self.hydro == "nohi":
            self.D = self.kBT * 10 ** 19 / 6 / np.pi / np.repeat(self.radii, 3) / self.eta
            return
        rij = self.c.pointers(self.pos, self.L)
        if self.hydro in ("rpy", "rpy_lub"):
            M = self.c.rpy(self.radii, rij)
        else:
            M = self.c.smith(self.radii, rij, self.L, self.alpha, self.m_max, self.n_max)
        if self.hydro in ("rpy", "rpy_smith"):
            self.D = M * (self.kBT * 10 ** 19 / self.eta)
        else:
            self.Mff = M * 10 ** 19 / self.eta
            self.Rff = np.linalg.inv(self.Mff)

    # box.py:533-541
    def _dtot(self):
        rij = self.c.pointers(self.pos, self.L)
        self.R = self.c.lubrication(self.radii, rij, self.cutoff, self.cich) * self.eta / 10 ** 19 + self.Rff
        self.D = self.kBT * np.linalg.inv(self.R)

    def _forces(self):
        """box.py:186: forces of the step; the external force alone here."""

    def _chol(self):
        self.B = np.sqrt(self.D) if self.hydro == "nohi" else np.linalg.cholesky(self.D)

    def _build(self, b_ff, b_nf, chol):
        if self.hydro == "nohi":
            return
        if b_ff:
            self._dff()
        if self.hydro in ("rpy_lub", "rpy_smith_lub") and b_nf:
            self._dtot()
        if chol:
            self._chol()

    def _translate(self, v):
        self.pos += np.asarray(v).reshape(-1, 3)

    def _det(self, dt, mult=1.0):
        if self.hydro != "nohi":
            FX = dt / self.kBT * self.D @ self.F * mult
        else:
            FX = dt / self.kBT * self.D * self.F * mult
        self._translate(FX)

    def _stoch(self, dt, mult=1.0):
        if self.hydro == "nohi":
            BX = self.B * self.N * math.sqrt(2 * dt) * mult
        else:
            BX = self.B @ self.N * math.sqrt(2 * dt) * mult
        self._translate(BX)

    def _noise(self):
        self.N = self.rng.normal(0.0, 1.0, 3 * len(self.radii))
        self.draw_count += 3 * len(self.radii)

    def _overlap(self):
        return self.c.overlaps(self.pos, self.radii, self.L, self.thr)

    def propagate(self, dt, build_Dff=True, build_Dnf=True, cholesky=True):
        self._b_ff, self._b_nf = build_Dff, build_Dnf
        self._build(build_Dff, build_Dnf, cholesky)
        self._forces()
        if self.scheme == "ermak":
            self._ermak(dt)
        else:
            self._midpoint(dt, build_Dff, build_Dnf, cholesky)
        # keep_in_box (bead.py:170-183)
        for i in range(self.pos.shape[0]):
            for k in range(3):
                while self.pos[i, k] < -self.L / 2:
                    self.pos[i, k] += self.L
                while self.pos[i, k] >= self.L / 2:
                    self.pos[i, k] -= self.L

    # box.py:560-610: forward-difference divergence of D, eps = 1e-7.  Each
    # coordinate is moved by +eps and back by -eps (not restored from a copy),
    # as the reference's bead.translate does; the matrices are restored.
    def _divergence(self, b_ff, b_nf):
        eps = 0.0000001
        saved = (self.D.copy(), self.Mff.copy(), self.Rff.copy(), self.R.copy())
        div = -np.sum(self.D, axis=1)
        for i in range(self.pos.shape[0]):
            for j in range(3):
                self.pos[i, j] += eps
                if b_ff:
                    self._dff()
                if b_nf:
                    self._dtot()
                div += self.D[3 * i + j]
                self.pos[i, j] += -eps
        self.D, self.Mff, self.Rff, self.R = saved
        return div / eps

    # box.py:202-250
    def _ermak(self, dt):
        self._det(dt)
        if self.inp.get("divergence_term") and self.hydro in ("rpy_lub", "rpy_smith_lub"):
            self._translate(self._divergence(self._b_ff, self._b_nf) * dt)
        count = 0
        while True:
            count += 1
            self._noise()
            self._stoch(dt)
            if self.overlaps:
                if self._overlap():
                    self._stoch(dt, mult=-1)
                else:
                    break
            else:
                break
            assert count < self.max_attempts, "maximal number of move attepts exceeded"
        self.attempt_log.append(count)

    # box.py:254-349
    def _midpoint(self, dt, b_ff, b_nf, chol):
        lub = self.hydro in ("rpy_lub", "rpy_smith_lub")
        D0, B0 = self.D.copy(), self.B.copy()
        if lub:
            Mff0, Rff0, R0 = self.Mff.copy(), self.Rff.copy(), self.R.copy()
        m = self.m
        self._det(dt, mult=1.0 / m)
        count = 0
        while True:
            count += 1
            self._noise()
            self._stoch(dt, mult=1.0 / m)
            if self.overlaps and self._overlap():
                self._stoch(dt, mult=-1.0 / m)
                continue
            self._build(b_ff, b_nf, chol)
            det_drift = m * dt / (2 * self.kBT) * (self.D - D0) @ self.F
            stoch_drift = m / 2 * math.sqrt(2 * dt) * (self.D @ np.linalg.inv(np.transpose(B0)) - B0) @ self.N
            drift = stoch_drift + det_drift
            self.D, self.B = D0, B0
            if lub:
                self.Mff, self.Rff, self.R = Mff0, Rff0, R0
            self._det(dt, mult=1.0 - 1.0 / m)
            self._stoch(dt, mult=1.0 - 1.0 / m)
            self._translate(drift)
            if self.overlaps:
                if self._overlap():
                    self._det(dt, mult=-(1.0 - 1.0 / m))
                    self._stoch(dt, mult=-1)
                    self._translate(-drift)
                else:
                    break
            else:
                break
            assert count < self.max_attempts, "maximal number of move attepts exceeded"
        self.attempt_log.append(count)


# ---------------------------------------------------------------------------
# Inter-bead forces and immobile beads (box.py:404-428, 649-668;
# interactions.py:109-414, 641-821), restated as plain loops for small N.

def _lj(kind, alpha, b1, b2, p):
    """LJ_6_attractive / LJ_12_repulsive / LJ_6_12 force on b1 and energy
    (interactions.py:711-821)."""
    sigma = b1.hard_core_radius + b2.hard_core_radius
    epsilon = math.sqrt(b1.epsilon_LJ * b2.epsilon_LJ)
    dist2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2]
    dist = math.sqrt(dist2)
    s2 = sigma * sigma / dist2
    s6 = s2 * s2 * s2
    versor = p / dist
    if kind == 6:
        return 6.0 * alpha * epsilon * s6 / dist * versor, -alpha * epsilon * s6
    if kind == 12:
        s12 = s2 * s2 * s2 * s2 * s2 * s2
        return -12.0 * alpha * epsilon * s12 / dist * versor, alpha * epsilon * s12
    s12 = s6 * s6
    return alpha * epsilon / dist * (6 * s6 - 12 * s12) * versor, alpha * epsilon * (s12 - s6)


def _bond(b1, b2, p):
    """harmonic_bond_force / _energy (interactions.py:641-665)."""
    dist_eq, k = b1.bonded_how[b2.bead_id]
    dist = math.sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2])
    return p / dist * k * (dist - dist_eq), 0.5 * k * (dist - dist_eq) ** 2


def _angle(b1, b2, b3, p12, p23):
    """harmonic_angle_force / _energy (interactions.py:667-709) with
    angle_pbc (bead.py:272-278)."""
    angle_eq, k = b1.angled_how[(b2.bead_id, b3.bead_id)]
    angle = np.rad2deg(np.arccos(-(p12[0] * p23[0] + p12[1] * p23[1] + p12[2] * p23[2])
                                 / math.sqrt(p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2])
                                 / math.sqrt(p23[0] * p23[0] + p23[1] * p23[1] + p23[2] * p23[2])))
    angle_eq *= np.pi / 180.0
    angle *= np.pi / 180.0
    d2_12 = p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2]
    d2_23 = p23[0] * p23[0] + p23[1] * p23[1] + p23[2] * p23[2]
    d12, d23 = math.sqrt(d2_12), math.sqrt(d2_23)
    sc = np.zeros(9)
    sc[:3] = (p23 / d23 + np.cos(angle) * p12 / d12) / d12
    sc[3:6] = (p12 - p23) / d12 / d23 - np.cos(angle) * (p12 / d2_12 - p23 / d2_23)
    sc[6:] = -p12 / d12 / d23 - np.cos(angle) * p23 / d2_23
    return k * (angle - angle_eq) / np.sin(angle) * sc, 0.5 * k * (angle - angle_eq) ** 2


def _find(beads, bead_id):
    """get_bead_with_id (bead.py:447-453)."""
    for i, b in enumerate(beads):
        if b.bead_id == bead_id:
            return i
    return None


class OracleForceBox(OracleBox):
    """OracleBox with immobile beads and inter-bead forces.  `beads` are
    objects with r, a, label, bead_id, hard_core_radius, epsilon_LJ,
    bonded_with/bonded_how, angled_with/angled_how (the reference's Bead
    fields); they are not modified.  `custom` is a list of
    (force, energy, aux, bonded, how_many_body) tuples evaluated with the
    same loops as the built-in terms."""

    def __init__(self, beads, inp, clib=None, custom=()):
        labels = inp.get("immobile_labels", [])
        self.beads = [_BeadView(b, b.label not in labels) for b in beads]
        self.mob = [b for b in self.beads if b.mobile]
        self.imm = [b for b in self.beads if not b.mobile]
        self.mob_idx = [i for i, b in enumerate(self.beads) if b.mobile]
        super().__init__(np.array([b.r for b in self.mob]), np.array([b.a for b in self.mob]), inp, clib)
        self.pos_imm = np.array([b.r for b in self.imm], dtype=np.float64).reshape(-1, 3)
        n = len(self.beads)
        # build_connection_matrix (bead.py:401-413)
        self.conn = np.zeros((n, n), dtype=np.int32)
        for i in range(n):
            for j in range(n):
                bi, bj = self.beads[i], self.beads[j]
                if bj.bead_id in bi.bonded_with or bi.bead_id in bj.bonded_with:
                    self.conn[i][j] = self.conn[j][i] = 1
                if not (bi.mobile or bj.mobile):
                    self.conn[i][j] = self.conn[j][i] = 1
        self.radii_all = np.array([b.a for b in self.beads])
        lj6, lj12 = bool(inp.get("lennard_jones_6")), bool(inp.get("lennard_jones_12"))
        self.lj = 612 if (lj6 and lj12) else 6 if lj6 else 12 if lj12 else 0
        self.lj_alpha = inp.get("lennard_jones_alpha", 4.0)
        self.custom = list(custom)
        self.unit = inp.get("energy_unit", "joule")
        self.E = 0.0

    def _positions_all(self):
        out = np.empty((len(self.beads), 3))
        out[self.mob_idx] = self.pos
        imm_idx = [i for i, b in enumerate(self.beads) if not b.mobile]
        out[imm_idx] = self.pos_imm
        return out

    def _overlap(self):
        """check_overlaps over every bead (box.py:464-466)."""
        return self.c.overlaps(self._positions_all(), self.radii_all, self.L, self.thr, self.conn)

    def _forces(self):
        """box.py:404-428 with the interactions of interactions.py:483-515 in order."""
        for b, r in zip(self.mob, self.pos):
            b.r = r.copy()
        mob, imm = self.mob, self.imm
        rij = self.c.pointers(self.pos, self.L)
        rik = self.c.pointers_immobile(self.pos, self.pos_imm, self.L) if imm else None
        F = np.array(list(np.array(self.inp.get("external_force", [0.0, 0.0, 0.0]), dtype=float)) * len(mob))
        E = 0.0
        terms = []
        if self.lj:
            terms.append((lambda b1, b2, p: _lj(self.lj, self.lj_alpha, b1, b2, p), False, 2))
        if any(b.bonded_with for b in self.beads):
            terms.append((_bond, True, 2))
        if any(b.angled_with for b in self.beads):
            terms.append((_angle, True, 3))
        for force, energy, aux, bonded, body in self.custom:
            terms.append(((lambda *a, f=force, e=energy, x=aux: (np.asarray(f(*a, **x), dtype=float), e(*a, **x))),
                          bonded, body))
        for fe, bonded, body in terms:
            E += self._loops(fe, bonded, body, mob, imm, rij, rik, F)
        if self.unit == "kcal/mol":
            F = 10 ** (-21) * 6.9477 * F
        elif self.unit == "eV":
            F = 10 ** (-19) * 1.602176634 * F
        self.F = F
        self.E = E

    @staticmethod
    def _loops(fe, bonded, body, mob, imm, rij, rik, F):
        """Interactions.compute_forces_and_energy (interactions.py:109-414)."""
        E = 0.0
        if body == 1:
            for i in range(len(mob)):
                f, e = fe(mob[i])
                F[3 * i:3 * (i + 1)] += f
                E += e
        elif body == 2 and not bonded:
            for i in range(1, len(mob)):
                for j in range(i):
                    f, e = fe(mob[i], mob[j], rij[i][j])
                    F[3 * i:3 * (i + 1)] += f
                    F[3 * j:3 * (j + 1)] -= f
                    E += e
            for i in range(len(mob)):
                for j in range(len(imm)):
                    f, e = fe(mob[i], imm[j], rik[i][j])
                    F[3 * i:3 * (i + 1)] += f
                    E += e
        elif body == 2:
            for i in range(len(mob)):
                for idx in mob[i].bonded_with:
                    j = _find(mob, idx)
                    if j is not None:
                        f, e = fe(mob[i], mob[j], rij[i][j])
                        F[3 * i:3 * (i + 1)] += f
                        F[3 * j:3 * (j + 1)] -= f
                    else:
                        j = _find(imm, idx)
                        f, e = fe(mob[i], imm[j], rik[i][j])
                        F[3 * i:3 * (i + 1)] += f
                    E += e
            for i in range(len(imm)):
                for idx in imm[i].bonded_with:
                    j = _find(mob, idx)
                    if j is not None:
                        f, e = fe(imm[i], mob[j], -rik[j][i])
                        F[3 * j:3 * (j + 1)] -= f
                        E += e
        elif body == 3 and bonded:
            for i in range(len(mob)):
                for idx1, idx2 in mob[i].angled_with:
                    j, k = _find(mob, idx1), _find(mob, idx2)
                    if j is not None:
                        bj, p12 = mob[j], rij[i][j]
                    else:
                        j = _find(imm, idx1)
                        bj, p12 = imm[j], rik[i][j]
                    if k is not None:
                        bk = mob[k]
                        p23 = rij[j][k] if bj.mobile else -rik[k][j]
                    else:
                        k = _find(imm, idx2)
                        bk = imm[k]
                        p23 = rik[j][k] if bj.mobile else rik[i][k] - p12
                    f, e = fe(mob[i], bj, bk, p12, p23)
                    F[3 * i:3 * (i + 1)] += f[:3]
                    if bj.mobile:
                        F[3 * j:3 * (j + 1)] += f[3:6]
                    if bk.mobile:
                        F[3 * k:3 * (k + 1)] += f[6:]
                    E += e
            for i in range(len(imm)):
                for idx1, idx2 in imm[i].angled_with:
                    j, k = _find(mob, idx1), _find(mob, idx2)
                    if j is None and k is None:
                        continue
                    if j is not None and k is not None:
                        bj, bk, p12, p23 = mob[j], mob[k], -rik[j][i], rij[j][k]
                    elif j is not None:
                        k = _find(imm, idx2)
                        bj, bk, p12, p23 = mob[j], imm[k], -rik[j][i], rik[j][k]
                    else:
                        j = _find(imm, idx1)
                        bj, bk = imm[j], mob[k]
                        p23 = -rik[k][j]
                        p12 = -rik[k][i] - p23
                    f, e = fe(imm[i], bj, bk, p12, p23)
                    if bj.mobile:
                        F[3 * j:3 * (j + 1)] += f[3:6]
                    if bk.mobile:
                        F[3 * k:3 * (k + 1)] += f[6:]
                    E += e
        else:
            raise NotImplementedError((body, bonded))
        return E

    def positions_all(self):
        return self._positions_all()


class _BeadView:
    """The fields of a bead the force loops read, with its own position."""

    def __init__(self, b, mobile):
        self.r = np.array(b.r, dtype=np.float64)
        self.a = float(b.a)
        self.label = b.label
        self.bead_id = b.bead_id
        self.hard_core_radius = b.hard_core_radius
        self.epsilon_LJ = b.epsilon_LJ
        self.bonded_with = list(b.bonded_with)
        self.bonded_how = dict(b.bonded_how)
        self.angled_with = [list(x) for x in b.angled_with]
        self.angled_how = dict(b.angled_how)
        self.mobile = mobile
