"""The synthetic workloads of bench.py and its CPU reference arm for the
lubricated configuration (CPU only).

The bench's inputs are seeded synthetic bead configurations; these tests pin
their defining properties: the lubricated box edge follows from the volume
fraction, placements respect the minimum gap under the minimum image, the
same seed gives the same configuration, and the reference arm runs the
reference's own C library on that workload.
"""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _min_gap(pos, radii, L):
    d = pos[:, None, :] - pos[None, :, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d * d).sum(-1))
    gap = r - (radii[:, None] + radii[None, :])
    np.fill_diagonal(gap, np.inf)
    return gap.min()


def test_lubricated_workload_volume_fraction_and_gap():
    import bench
    w = bench.lub_workload()
    N, a, L = w["n_beads"], w["radius"], w["box_length"]
    assert N * 4.0 / 3.0 * math.pi * a ** 3 / L ** 3 == pytest.approx(0.30, rel=1e-12)
    pos, radii = bench.bead_config(w["seed"], N, L, a, a, gap=w["min_gap"])
    assert pos.shape == (N, 3) and np.all(radii == a)
    assert np.all(np.abs(pos) <= L / 2)
    assert _min_gap(pos, radii, L) > w["min_gap"]
    pos2, _ = bench.bead_config(w["seed"], N, L, a, a, gap=w["min_gap"])
    assert np.array_equal(pos, pos2)


def test_headline_workload_placement():
    import bench
    pos, radii = bench.bead_config(0, 1024, bench.WORKLOAD["box_length"], 10.0, 40.0)
    assert np.all((radii >= 10.0) & (radii <= 40.0))
    assert _min_gap(pos, radii, bench.WORKLOAD["box_length"]) > 0.0


def test_lubricated_input_keywords():
    import bench
    inp = bench.lub_input("mixed")
    assert inp["hydrodynamics"] == "rpy_smith_lub" and inp["propagation_scheme"] == "midpoint"
    assert inp["lubrication_cutoff"] == 0.5 and inp["cichocki_correction"] is True
    assert inp["m_midpoint"] == 100.0 and inp["precision"] == "mixed"


def test_lubricated_reference_arm_runs_the_reference():
    import bench
    from oracle.oracle import REF_OMP_LIB
    if not os.path.exists(REF_OMP_LIB):
        pytest.skip("oracle/_ref not built (the reference's C sources were absent at build time)")
    sps, cores, kind, sample = bench.cpu_reference_lub_steps(steps=1)
    assert sps > 0 and cores >= 1 and kind == "reference" and "libpyBrown_omp.so" in sample
