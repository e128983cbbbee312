"""Hydrodynamic tensors (drop-in for pyBrown.diffusion, src/bdsim/pyBrown/diffusion.py).

Same functions, arguments and return shapes as the reference; the work runs
on the GPU through the reference ABI exported by libpybrown_b200.  Pair
vectors are packed exactly as the reference packs them: the upper triangle of
-pointers in row-major order (diffusion.py:40,70,155).
"""
import numpy as np

from ._lib import dptr, lib


def _radii(beads):
    return np.ascontiguousarray([b.a for b in beads], dtype=np.float64)


def _packed_pairs(pointers, N):
    iu = np.triu_indices(n=N, k=1)
    return np.ascontiguousarray(-np.asarray(pointers)[iu], dtype=np.float64).reshape(-1)


def RPY_M_matrix(beads, pointers):
    """diffusion.py:30-56: free-space RPY mobility, (3N, 3N)."""
    N = len(beads)
    a = _radii(beads)
    p = _packed_pairs(pointers, N)
    M = np.zeros(9 * N * N, dtype=np.float64)
    lib.RPY_M_matrix(dptr(a), dptr(p), N, dptr(M))
    return M.reshape(3 * N, 3 * N)


def RPY_Smith_M_matrix(beads, pointers, box_length, alpha, m, n):
    """diffusion.py:60-94: RPY mobility under Smith's Ewald summation, (3N, 3N)."""
    N = len(beads)
    a = _radii(beads)
    p = _packed_pairs(pointers, N)
    M = np.zeros(9 * N * N, dtype=np.float64)
    lib.RPY_Smith_M_matrix(dptr(a), dptr(p), float(box_length), float(alpha), int(m), int(n), N, dptr(M))
    return M.reshape(3 * N, 3 * N)


def JO_2B_R_matrix(beadi, beadj):
    """diffusion.py:98-141: Jeffrey-Onishi two-body resistance, (6, 6)."""
    out = np.zeros(18, dtype=np.float64)
    r = beadj.r - beadi.r
    lib.JO_2B_R_matrix(float(beadi.a), float(beadj.a), float(r[0]), float(r[1]), float(r[2]), dptr(out))
    R = np.zeros((6, 6))
    R[0][0], R[1][1], R[2][2] = out[0], out[1], out[2]
    R[0][1] = R[1][0] = out[3]
    R[0][2] = R[2][0] = out[4]
    R[1][2] = R[2][1] = out[5]
    R[3][3], R[4][4], R[5][5] = out[6], out[7], out[8]
    R[3][4] = R[4][3] = out[9]
    R[3][5] = R[5][3] = out[10]
    R[4][5] = R[5][4] = out[11]
    R[3][0] = R[0][3] = out[12]
    R[4][1] = R[1][4] = out[13]
    R[5][2] = R[2][5] = out[14]
    R[4][0] = R[0][4] = R[3][1] = R[1][3] = out[15]
    R[5][0] = R[0][5] = R[3][2] = R[2][3] = out[16]
    R[5][1] = R[1][5] = R[4][2] = R[2][4] = out[17]
    return R


def JO_R_lubrication_correction_matrix(beads, pointers, lubrication_cutoff, cichocki_correction):
    """diffusion.py:145-175: lubrication correction of the resistance, (3N, 3N)."""
    N = len(beads)
    a = _radii(beads)
    p = _packed_pairs(pointers, N)
    C = np.zeros(9 * N * N, dtype=np.float64)
    lib.JO_R_lubrication_correction_matrix(dptr(a), dptr(p), N, float(lubrication_cutoff),
                                           1 if cichocki_correction else 0, dptr(C))
    return C.reshape(3 * N, 3 * N)
