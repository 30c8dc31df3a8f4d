"""Host-side behaviour of the plug-ins that needs no GPU: the reference's exceptions for the same misuse, raised
before any device work (accusim/forces.py:360-367, accusim/simulation.py:96-97), and the plug-ins' identity as
accusim classes (the isinstance checks of accusim/accuracy.py:149 and accusim/advisor.py:36)."""
import numpy as np
import pytest


def test_error_behaviour_matches_reference():
    import accusim

    from devinproj_b200 import Ewald
    s = accusim.System(3)                                   # open boundaries
    s.add_species("Na", 1.0, charge=1.0)
    s.add_species("Cl", 1.0, charge=-1.0)
    s.add("Na", [[0.0, 0.0, 0.0]])
    s.add("Cl", [[1.0, 0.0, 0.0]])
    with pytest.raises(ValueError, match="3D periodic"):
        Ewald(k=1.0).compute(s)
    p = accusim.System(3, box=4.0, periodic=True)
    p.add_species("Na", 1.0, charge=1.0)
    p.add("Na", [[0.0, 0.0, 0.0], [2.0, 0.0, 0.0]])
    with pytest.raises(ValueError, match="charge-neutral"):
        Ewald(k=1.0).compute(p)
    sim = accusim.Simulation(p, [])
    with pytest.raises(ValueError, match="set dt"):
        sim.run(steps=1)
    assert np.all(sim.force == 0)


def test_plugins_are_accusim_classes():
    """accusim's own report and advisor recognise the GPU classes through their isinstance checks, and the
    inherited attributes are the reference's."""
    import accusim

    import devinproj_b200 as b200
    lj = b200.LennardJones({"Ar": (1.0, 2.0)}, cutoff=2.5)
    dsf = b200.DampedShiftedCoulomb(rcut=10e-10)
    assert isinstance(lj, accusim.LennardJones) and isinstance(dsf, accusim.DampedShiftedCoulomb)
    assert isinstance(b200.VelocityVerlet(), accusim.VelocityVerlet)
    assert isinstance(b200.Langevin(300.0, 1e12), accusim.Langevin)
    assert isinstance(b200.NoseHoover(300.0, 1e-13), accusim.NoseHoover)
    assert isinstance(b200.Ewald(), accusim.Ewald)
    ref = accusim.DampedShiftedCoulomb(rcut=10e-10)
    assert (dsf.alpha, dsf.skin, dsf.k, dsf.pairlist_threshold) == (ref.alpha, ref.skin, ref.k, ref.pairlist_threshold)
    assert lj.rebuilds == 0 and dsf._vl.rebuilds == 0
    assert b200.VelocityVerlet.order == 2 and b200.VelocityVerlet.symplectic
    assert b200.Langevin.stochastic and b200.NoseHoover.thermostat


def test_gpu_system_host_semantics():
    """GpuSystem behaves as accusim's System on the host (no device work): building, copying, reading."""
    from devinproj_b200 import GpuSystem
    s = GpuSystem(3, box=10.0, periodic=True)
    s.add_species("Ar", 2.0)
    ids = s.add("Ar", np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]]), vel=np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]))
    assert list(ids) == [0, 1] and s.n == 2
    assert s.kinetic_energy() == pytest.approx(2.0)
    c = s.copy()
    assert isinstance(c, GpuSystem) and c.n == 2 and c.pos is not s.pos
    c.pos += 1.0
    assert s.pos[0, 0] == 1.0 and c.pos[0, 0] == 2.0
    s.apply_boundaries()
    assert np.array_equal(s.pos, [[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]])
    s.remove(np.array([True, False]))
    assert s.n == 1 and list(s.ids) == [1]
