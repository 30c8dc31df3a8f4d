"""SI conversion at the API edge and the CODATA constants the path uses.

Arguments may be plain SI numbers or any quantity object exposing `.si(unit)` (accusim's
`Quantity`, accusim/units.py:123-129); `si()` mirrors accusim/units.py:219-223.
"""
from __future__ import annotations

import math

import numpy as np

k_B = 1.380649e-23              # J/K
N_A = 6.02214076e23             # 1/mol
e_charge = 1.602176634e-19      # C
epsilon_0 = 8.8541878128e-12    # C^2/J/m
k_e = 1 / (4 * math.pi * epsilon_0)
amu = 1.66053906660e-27         # kg
c_light = 299792458.0           # m/s


def si(x, unit=None):
    """SI number from a quantity (checked by its own `.si`) or a plain number passed through."""
    if hasattr(x, "si") and callable(getattr(x, "si")):
        return x.si(unit)
    if hasattr(x, "value") and hasattr(x, "dim"):
        return x.value
    return np.asarray(x, dtype=float) if not np.isscalar(x) else float(x)
