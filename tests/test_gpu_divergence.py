"""Divergence term of the lubricated diffusion matrix (box.py:211-215,
560-610) on the GPU against the oracle.

The term is a forward difference with eps = 1e-7: each of its 3N entries is
(sum of D rows at moved positions - row sums of D) / eps, so a relative
rounding difference r between two correct builds of D shows up as about
3e2 * r in div (measured on the oracle: r = 1e-13 gives 3.7e-5, r = 1e-14
gives 3.5e-6).  The GPU and the oracle build D with different summation orders
and inversions, so div is held to 1e-3, while the displacement of the step, of
which div * dt is a small part, keeps a 1e-8 bar."""
import math

import numpy as np
import pytest

from conftest import rel_err
from test_gpu_box import _box, _config, _inp

pytestmark = pytest.mark.gpu


def _dense(N, seed, phi=0.30):
    a = 20.0
    L = (N * 4 * math.pi * a ** 3 / 3 / phi) ** (1 / 3)
    pos, radii = _config(seed, N, L, a, a, 0.05 * a)
    return pos, radii, L


# Free-space RPY under the minimum image is not positive definite at phi = 0.3
# (the oracle's Cholesky fails there too), so rpy_lub runs at phi = 0.1.
@pytest.mark.parametrize("hydro,phi", [("rpy_lub", 0.1), ("rpy_smith_lub", 0.3)])
def test_divergence_term_vs_oracle(oracle_lib, hydro, phi):
    from oracle.oracle import OracleBox
    pos, radii, L = _dense(16, 5, phi)
    dt = 0.1
    inp = _inp(box_length=L, hydrodynamics=hydro, lubrication_cutoff=0.5, divergence_term=True)
    with_div = _box(pos, radii, inp)
    without = _box(pos, radii, dict(inp, divergence_term=False))
    ref = OracleBox(pos, radii, inp, clib=oracle_lib)
    ref._build(True, True, True)
    ref._det(dt)
    div_ref = ref._divergence(True, True) * dt

    with_div.propagate(dt)
    without.propagate(dt)
    assert with_div.draw_count == without.draw_count
    got = np.array([b.r for b in with_div.beads]) - np.array([b.r for b in without.beads])
    assert np.linalg.norm(div_ref) > 0
    assert rel_err(got.ravel(), div_ref) <= 1e-3


def test_divergence_trajectory_vs_oracle(oracle_lib):
    """Three Ermak steps of rpy_smith_lub with the divergence term."""
    from oracle.oracle import OracleBox
    pos, radii, L = _dense(12, 7)
    inp = _inp(box_length=L, hydrodynamics="rpy_smith_lub", lubrication_cutoff=0.5, divergence_term=True)
    box = _box(pos, radii, inp)
    ref = OracleBox(pos, radii, inp, clib=oracle_lib)
    for _ in range(3):
        box.propagate(0.1)
        ref.propagate(0.1)
        assert box.draw_count == ref.draw_count
    got = np.array([b.r for b in box.beads])
    assert rel_err(got - pos, ref.pos - pos) <= 1e-8
    assert rel_err(box.D, ref.D) <= 1e-10


def test_divergence_ignored_outside_lubricated_ermak(oracle_lib):
    """The keyword changes nothing for rpy_smith or for the midpoint scheme
    (box.py:211-213 applies it only to the lubrication modes under Ermak)."""
    pos, radii, L = _dense(12, 9)
    for kw in ({"hydrodynamics": "rpy_smith"},
               {"hydrodynamics": "rpy_smith_lub", "propagation_scheme": "midpoint"}):
        inp = _inp(box_length=L, lubrication_cutoff=0.5, **kw)
        a = _box(pos, radii, dict(inp, divergence_term=True))
        b = _box(pos, radii, dict(inp, divergence_term=False))
        a.propagate(0.1)
        b.propagate(0.1)
        assert np.array_equal(np.array([x.r for x in a.beads]), np.array([x.r for x in b.beads]))
