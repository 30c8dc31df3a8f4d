"""SI values of accusim's physical constants (accusim/units.py:226-233) as plain floats for the host code and the
engine's unit conversion, and accusim's own `si()` for arguments given as quantities."""
from __future__ import annotations

from ._accusim import units as _u

si = _u.si
k_B = float(_u.k_B.value)                         # J/K
N_A = float(_u.N_A.value)                         # 1/mol
e_charge = float(_u.e_charge.value)               # C
k_e = float(_u.k_e.value)                         # J m / C^2
amu = float(_u.parse_unit("u").value)             # kg
c_light = float(_u.c.value)                       # m/s
