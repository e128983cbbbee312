"""CPU oracle: ctypes front end of a library with pyBrown's C ABI, plus a
NumPy restatement of Box.propagate for the hydrodynamic hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.

Libraries it can drive (both export the reference's symbols, diff_tensor.c /
bead.c):
  * oracle/_build/libpybrown_oracle.so -- the in-house C restatement
  * oracle/_ref/libpyBrown.so          -- the reference's own C compiled here
  * oracle/_ref/libpyBrown_omp.so      -- the same with OpenMP
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libpybrown_oracle.so")
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
