"""Trajectory files and the msd observable against files and values written by the reference itself
(tests/golden/make_golden.py: io_traj108.npz is accusim/io.py:save's own output). CPU only."""
import os

import numpy as np

from devinproj_b200 import io as bio
from devinproj_b200.analysis import msd
from devinproj_b200.system import System

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _system_from_meta(meta, box):
    s = System(3, box=box, periodic=True)
    for m in meta:
        s.add_species(m["name"], m["mass"], charge=m["charge"])
    return s


def test_reference_file_loads_and_saves_back_identically(tmp_path, golden):
    g = golden("analysis_msd108")
    tr, meta = bio.load(os.path.join(GOLDEN, "io_traj108.npz"))
    assert [m["name"] for m in meta] == ["Ar"]
    assert np.array_equal(np.array(tr.t), g["t_frames"])
    assert np.array_equal(np.array(tr.positions), g["frames"])
    out = tmp_path / "again.npz"
    bio.save(tr, _system_from_meta(meta, g["box"]), out)
    a, b = np.load(os.path.join(GOLDEN, "io_traj108.npz")), np.load(out)
    assert sorted(a.files) == sorted(b.files)
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k


def test_msd_matches_reference(golden):
    g = golden("analysis_msd108")
    tr, _ = bio.load(os.path.join(GOLDEN, "io_traj108.npz"))
    t, m = msd(tr, box=g["box"])
    assert np.array_equal(t, g["t"]) and np.array_equal(m, g["msd"])


def test_error_behaviour_matches_reference():
    """The reference's exceptions for the same misuse, raised before any device work (accusim/forces.py:360-367,
    accusim/simulation.py:96-97)."""
    import numpy as np
    import pytest
    from devinproj_b200 import Simulation, System
    from devinproj_b200.ewald import Ewald
    s = System(3)                                   # open boundaries
    s.add_species("Na", 1.0, charge=1.0)
    s.add_species("Cl", 1.0, charge=-1.0)
    s.add("Na", [[0.0, 0.0, 0.0]])
    s.add("Cl", [[1.0, 0.0, 0.0]])
    with pytest.raises(ValueError, match="3D periodic"):
        Ewald(k=1.0).compute(s)
    p = System(3, box=4.0, periodic=True)
    p.add_species("Na", 1.0, charge=1.0)
    p.add("Na", [[0.0, 0.0, 0.0], [2.0, 0.0, 0.0]])
    with pytest.raises(ValueError, match="charge-neutral"):
        Ewald(k=1.0).compute(p)
    sim = Simulation(p, [])
    with pytest.raises(ValueError, match="set dt"):
        sim.run(steps=1)
    assert np.all(sim.force == 0)
