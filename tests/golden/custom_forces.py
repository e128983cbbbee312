"""A custom-interactions file in the reference's format (interactions.py:591-637):
functions named <name>_<k>b_force / <name>_<k>b_energy, "bonded" in the name
for bonded terms, every auxiliary keyword passed to every function.  Used by
the force fixtures (make_golden_forces.py) and their tests."""
import math

import numpy as np


def tether_1b_force(bead1, tether_k, soft_eps):
    """Harmonic tether of each bead to the origin."""
    return -tether_k * np.array(bead1.r, dtype=float)


def tether_1b_energy(bead1, tether_k, soft_eps):
    r = np.array(bead1.r, dtype=float)
    return 0.5 * tether_k * float(r @ r)


def soft_2b_force(bead1, bead2, pointer, tether_k, soft_eps):
    """Gaussian-core repulsion between every pair."""
    d2 = float(pointer @ pointer)
    return -0.5 * soft_eps * math.exp(-d2 / 4.0) * pointer


def soft_2b_energy(bead1, bead2, pointer, tether_k, soft_eps):
    return soft_eps * math.exp(-float(pointer @ pointer) / 4.0)
