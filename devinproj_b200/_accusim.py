"""The host framework these plug-ins plug into: the `accusim` package (erezbz/DevinProj).

The GPU classes of this package subclass accusim's own `Force` and `Integrator` classes, so that accusim's
`Simulation.run`, `AccuracyReport`, `calibrate_dt` and `timescales` accept them and their `isinstance` checks
(accusim/accuracy.py:149, accusim/advisor.py:36) see the reference classes. accusim is pure Python; it is
imported from the environment, or else from the repository's own offline install under `baseline/_ref`
(made by `baseline/install_reference.sh`).
"""
from __future__ import annotations

import os
import sys

_REPO_INSTALL = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref")

try:
    import accusim  # noqa: F401
except ImportError:
    if os.path.isdir(os.path.join(_REPO_INSTALL, "accusim")):
        sys.path.append(_REPO_INSTALL)
        import accusim  # noqa: F401
    else:
        raise ImportError("devinproj_b200 plugs into the accusim package, which is not importable: install it "
                          "(pip install <accusim checkout>, or baseline/install_reference.sh)") from None

import accusim.accuracy as accuracy  # noqa: E402
import accusim.forces as forces  # noqa: E402
import accusim.integrators as integrators  # noqa: E402
import accusim.simulation as simulation  # noqa: E402
import accusim.system as system  # noqa: E402
import accusim.units as units  # noqa: E402

__all__ = ["accusim", "accuracy", "forces", "integrators", "simulation", "system", "units"]
