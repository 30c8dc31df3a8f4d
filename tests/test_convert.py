"""`gpu_twin` / `to_gpu` host logic (no GPU): an accusim force or integrator becomes this package's plug-in of the
same parameters and state, which accusim's `isinstance` checks still see as the accusim class; classes without a
GPU plug-in, user subclasses and plug-ins that are already GPU ones come back unchanged."""
import accusim

import devinproj_b200 as b200
from devinproj_b200.forces import VerletList


def test_forces_take_their_parameters_over():
    lj = accusim.forces.LennardJones({"Ar": (1.6e-21, 3.4e-10), "Kr": (2.3e-21, 3.6e-10)}, cutoff=2.2,
                                     pairlist_threshold=100, skin=0.4)
    t = b200.gpu_twin(lj)
    assert type(t) is b200.LennardJones and isinstance(t, accusim.forces.LennardJones)
    assert t.params == lj.params and t.cutoff == 2.2 and t.pairlist_threshold == 100 and t.skin == 0.4
    assert isinstance(t._vl, VerletList) and t._vl is not lj._vl and t.rebuilds == 0
    dsf = accusim.forces.DampedShiftedCoulomb(rcut=9e-10, alpha=0.25e10, k=1.0, exclude=[(0, 3), (5, 2)], skin=1e-10)
    t = b200.gpu_twin(dsf)
    assert type(t) is b200.DampedShiftedCoulomb and isinstance(t, accusim.forces.DampedShiftedCoulomb)
    assert (t.rcut, t.alpha, t.k, t.skin, t.exclude, t.pairlist_threshold) == \
        (dsf.rcut, dsf.alpha, dsf.k, dsf.skin, dsf.exclude, dsf.pairlist_threshold)
    assert isinstance(t._vl, VerletList)
    ew = accusim.forces.Ewald(alpha=3e9, rcut=1.2e-9, kmax=9)
    t = b200.gpu_twin(ew)
    assert type(t) is b200.Ewald and (t.alpha, t.rcut, t.kmax, t.k) == (ew.alpha, ew.rcut, ew.kmax, ew.k)


def test_integrators_take_their_state_over():
    nh = accusim.integrators.NoseHoover(300.0, 1e-13)
    nh.xi, nh.eta, nh.Q = 1.5e11, -0.25, 3.0e-44
    t = b200.gpu_twin(nh)
    assert type(t) is b200.NoseHoover and isinstance(t, accusim.integrators.NoseHoover)
    assert (t.T, t.tau, t.xi, t.eta, t.Q) == (300.0, 1e-13, 1.5e11, -0.25, 3.0e-44)
    lv = accusim.integrators.Langevin(1200.0, 5e12)
    t = b200.gpu_twin(lv)
    assert type(t) is b200.Langevin and (t.T, t.gamma) == (1200.0, 5e12)
    assert type(b200.gpu_twin(accusim.integrators.VelocityVerlet())) is b200.VelocityVerlet


def test_others_come_back_unchanged():
    keep = [accusim.forces.HarmonicBond([(0, 1)], 100.0, 1e-10), accusim.integrators.Yoshida4(),
            b200.LennardJones({"Ar": (1.6e-21, 3.4e-10)})]

    class MyLJ(accusim.forces.LennardJones):
        pass

    keep.append(MyLJ({"Ar": (1.6e-21, 3.4e-10)}))
    for obj in keep:
        assert b200.gpu_twin(obj) is obj


def test_to_gpu_decides_where_the_state_lives(monkeypatch):
    """to_gpu swaps forces and integrator always, and the system for a GpuSystem only when asked, for 3-D systems
    and simulations without reactions (accusim's reaction engine keeps the system it was built with); it then
    recomputes the forces once (a stand-in here: no GPU)."""
    from devinproj_b200 import configs, convert
    from devinproj_b200 import state as st

    made = []
    monkeypatch.setattr(st.GpuSystem, "from_system", classmethod(lambda cls, s: made.append(s) or ("gpu", s)))

    class FakeSim:
        def __init__(self, system, reactions=None):
            self.system, self.reactions = system, reactions
            self.forces = [accusim.forces.LennardJones({"Ar": (1.6e-21, 3.4e-10)}),
                           accusim.forces.UniformField(E=[1.0, 0.0, 0.0])]
            self.integrator = accusim.integrators.VelocityVerlet()
            self.updates = 0

        def update_forces(self):
            self.updates += 1

    s, _ = configs.lj_fluid(2, seed=0)
    sim = convert.to_gpu(FakeSim(s))
    assert sim.system == ("gpu", s) and made == [s] and sim.updates == 1
    assert type(sim.forces[0]) is b200.LennardJones and type(sim.forces[1]) is accusim.forces.UniformField
    assert type(sim.integrator) is b200.VelocityVerlet
    for kw, sim in (({"resident": False}, FakeSim(s)), ({}, FakeSim(s, reactions=object()))):
        convert.to_gpu(sim, **kw)
        assert sim.system is s and type(sim.forces[0]) is b200.LennardJones and sim.updates == 1
    flat = accusim.System(2, box=[1e-9, 1e-9], periodic=True)
    sim = convert.to_gpu(FakeSim(flat))
    assert sim.system is flat and made == [s]
