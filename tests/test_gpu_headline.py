"""Parity at the full sizes of the benchmarked configurations, against the
FP64 oracle (the C restatement built with OpenMP: identical results to the
serial build, all host cores) on the same positions and the same
RandomState noise:

  * BD with HI, N = 1024 (polydisperse radii U[10, 40] A, box 1500 A,
    Smith-Ewald m = 2, n = 4, Ermak, dt = 0.5 ps): the FP64 GPU path matches
    D, B and the positions after 5 steps to 1e-10 with identical draw counts;
  * the same workload on the mixed-precision path: D, B, B xi and the
    displacement after 5 steps within 1e-5 of the FP64 oracle;
  * Stokesian dynamics, N = 512 at volume fraction 0.30 (gap >= 0.05 a,
    rpy_smith_lub, cutoff 0.5, Cichocki, midpoint m = 100, dt = 0.1 ps), FP64:
    R, Rff, D, B and the positions after 2 steps to 1e-10;
  * a 512-bead replica inside a batch with smaller ones, FP64 and mixed,
    against the oracle run alone.

Errors are max |a - b| / max |b| (rel_err), the bar used throughout."""
import math

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _config(seed, N, L, a_lo, a_hi, gap=0.0):
    """Sequential rejection sampling (the bench's placement)."""
    rng = np.random.default_rng(seed)
    pos = np.zeros((N, 3))
    radii = np.zeros(N)
    k = 0
    while k < N:
        a = rng.uniform(a_lo, a_hi)
        p = rng.uniform(-L / 2, L / 2, size=3)
        if k:
            d = pos[:k] - p
            d -= L * np.round(d / L)
            if np.any(np.sqrt((d * d).sum(1)) <= radii[:k] + a + gap):
                continue
        pos[k], radii[k] = p, a
        k += 1
    return pos, radii


def _inp(**kw):
    d = {"box_length": 1500.0, "T": 293.15, "viscosity": 0.01005, "seed": 0, "hydrodynamics": "rpy_smith",
         "ewald_alpha": math.sqrt(math.pi), "ewald_real": 2, "ewald_imag": 4, "propagation_scheme": "ermak",
         "immobile_labels": [], "check_overlaps": True, "overlap_treshold": 0.0, "max_move_attempts": 1000000,
         "external_force": [0.0, 0.0, 0.0], "energy_unit": "joule", "verbose": False, "debug": False,
         "lubrication_cutoff": 0.5, "cichocki_correction": True, "m_midpoint": 100,
         "lennard_jones_6": False, "lennard_jones_12": False, "custom_interactions": False}
    d.update(kw)
    return d


def _box(pos, radii, inp):
    from pybrown_b200.bead import Bead
    from pybrown_b200.box import Box
    return Box([Bead(p.copy(), float(a)) for p, a in zip(pos, radii)], dict(inp))


def _positions(box):
    return np.array([b.r for b in box.beads])


def _disp_err(got, ref, init, L):
    dg, dr = got - init, ref - init
    dg -= L * np.round((dg - dr) / L)  # a bead wrapped in one path only
    return rel_err(dg, dr)


@pytest.fixture(scope="module")
def bd1024():
    return _config(0, 1024, 1500.0, 10.0, 40.0)


def test_bd_hi_n1024_fp64_vs_oracle(bd1024, oracle_omp_lib):
    from oracle.oracle import OracleBox
    pos, radii = bd1024
    inp = _inp()
    box = _box(pos, radii, inp)
    ref = OracleBox(pos, radii, inp, clib=oracle_omp_lib)
    for step in range(5):
        box.propagate(0.5)
        ref.propagate(0.5)
        assert box.draw_count == ref.draw_count, step
        if step in (0, 4):
            assert rel_err(box.D, ref.D) <= 1e-10, step
            assert rel_err(np.tril(box.B), ref.B) <= 1e-10, step
    assert _disp_err(_positions(box), ref.pos, pos, 1500.0) <= 1e-10


def test_bd_hi_n1024_mixed_vs_fp64_oracle(bd1024, oracle_omp_lib):
    """The mixed path's D, B and B xi at the start positions and its
    displacement after 5 steps, each within 1e-5 of the FP64 oracle."""
    from oracle.oracle import OracleBox
    pos, radii = bd1024
    inp = _inp(precision="mixed")
    box = _box(pos, radii, inp)
    ref_inp = dict(inp)
    ref_inp.pop("precision")
    ref = OracleBox(pos, radii, ref_inp, clib=oracle_omp_lib)
    box.propagate(0.5)
    ref.propagate(0.5)
    xi = np.random.RandomState(0).normal(0.0, 1.0, 3 * len(radii))  # the first step's noise
    B = np.tril(box.B)
    errs = {"D": rel_err(box.D, ref.D), "B": rel_err(B, ref.B), "Bxi": rel_err(B @ xi, ref.B @ xi)}
    for _ in range(4):
        box.propagate(0.5)
        ref.propagate(0.5)
    assert box.draw_count == ref.draw_count
    errs["disp"] = _disp_err(_positions(box), ref.pos, pos, 1500.0)
    print("mixed vs FP64 oracle, N=1024:", errs)
    assert all(v <= 1e-5 for v in errs.values()), errs


def test_sd_n512_fp64_midpoint_vs_oracle(oracle_omp_lib):
    from oracle.oracle import OracleBox
    N, a, phi = 512, 20.0, 0.30
    L = (N * 4.0 * math.pi * a ** 3 / 3.0 / phi) ** (1.0 / 3.0)
    pos, radii = _config(0, N, L, a, a, gap=0.05 * a)
    inp = _inp(box_length=L, hydrodynamics="rpy_smith_lub", propagation_scheme="midpoint")
    box = _box(pos, radii, inp)
    ref = OracleBox(pos, radii, inp, clib=oracle_omp_lib)
    for step in range(2):
        box.propagate(0.1)
        ref.propagate(0.1)
        assert box.draw_count == ref.draw_count, step
    # the matrices of the last step start (the midpoint ones are not kept by either)
    assert rel_err(box.Rff, ref.Rff) <= 1e-10
    assert rel_err(box.R, ref.R) <= 1e-10
    assert rel_err(box.D, ref.D) <= 1e-10
    assert rel_err(np.tril(box.B), ref.B) <= 1e-10
    assert _disp_err(_positions(box), ref.pos, pos, L) <= 1e-10


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_batch_replica_n512_vs_oracle(oracle_omp_lib, precision, tol):
    """A replica of 512 beads (the largest N of the batched configuration:
    radii U[10, 30], volume fraction 0.05) advanced in a batch next to smaller
    replicas, against the oracle run alone."""
    from oracle.oracle import OracleBox
    from pybrown_b200.batch import ReplicaBatch
    batch = ReplicaBatch(precision=precision)
    reps = []
    for k, N in enumerate((512, 40, 200)):
        rng = np.random.default_rng(900 + k)
        radii = rng.uniform(10.0, 30.0, size=N)
        L = float((np.sum(4.0 / 3.0 * np.pi * radii ** 3) / 0.05) ** (1.0 / 3.0))
        pos, radii = _config(900 + k, N, L, 10.0, 30.0)
        inp = _inp(box_length=L, seed=50 + k)
        slot = batch.add(pos, radii, L, T=inp["T"], viscosity=inp["viscosity"], seed=inp["seed"], noise="numpy")
        reps.append((slot, OracleBox(pos, radii, inp, clib=oracle_omp_lib), pos, L))
    draws = {s: 0 for s, _, _, _ in reps}
    for step in range(3):
        batch.propagate(0.5)
        for s, box, init, L in reps:
            box.propagate(0.5)
            draws[s] += 3 * len(init) * batch.last_move_attempts(s)
            assert draws[s] == box.draw_count, (s, step)
    s, box, init, L = reps[0]
    assert _disp_err(batch.positions(s), box.pos, init, L) <= tol
    assert rel_err(batch.matrix(s, "D"), box.D) <= tol
    assert rel_err(np.tril(batch.matrix(s, "B")), box.B) <= tol
    for s, box, init, L in reps[1:]:
        assert _disp_err(batch.positions(s), box.pos, init, L) <= tol, s
    batch.close()


def test_batch_replica_n2048_mixed_vs_oracle(oracle_omp_lib):
    """The largest request of the serving stream (2048 beads, radii
    U[10, 40], volume fraction 0.05: 96 tile columns for the left-looking
    batched factorisation) in a batch with a small replica, one step against
    the oracle run alone."""
    from oracle.oracle import OracleBox
    from pybrown_b200.batch import ReplicaBatch
    batch = ReplicaBatch(precision="mixed")
    reps = []
    for k, N in enumerate((2048, 64)):
        rng = np.random.default_rng(950 + k)
        radii = rng.uniform(10.0, 40.0, size=N)
        L = float((np.sum(4.0 / 3.0 * np.pi * radii ** 3) / 0.05) ** (1.0 / 3.0))
        pos, radii = _config(950 + k, N, L, 10.0, 40.0)
        inp = _inp(box_length=L, seed=70 + k)
        slot = batch.add(pos, radii, L, T=inp["T"], viscosity=inp["viscosity"], seed=inp["seed"], noise="numpy")
        reps.append((slot, OracleBox(pos, radii, inp, clib=oracle_omp_lib), pos, L))
    batch.propagate(1.0)
    for s, box, init, L in reps:
        box.propagate(1.0)
        assert 3 * len(init) * batch.last_move_attempts(s) == box.draw_count, s
    s, box, init, L = reps[0]
    assert rel_err(batch.matrix(s, "D"), box.D) <= 1e-5
    assert rel_err(np.tril(batch.matrix(s, "B")), box.B) <= 1e-5
    for s, box, init, L in reps:
        assert _disp_err(batch.positions(s), box.pos, init, L) <= 1e-5, s
    batch.close()
