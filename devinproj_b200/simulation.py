"""Simulation driver with the interface of accusim's `Simulation` and `Trajectory`
(accusim/simulation.py:14-131): the step loop that calls the integrator plug-in and records the
conserved quantities. Reactions are outside this package's scope and are rejected."""
from __future__ import annotations

import copy
from dataclasses import dataclass, field

import numpy as np

from .integrators import VelocityVerlet
from .units import c_light, si


@dataclass
class Trajectory:
    t: list = field(default_factory=list)
    kinetic: list = field(default_factory=list)
    potential: list = field(default_factory=list)
    internal: list = field(default_factory=list)
    released: list = field(default_factory=list)
    momentum: list = field(default_factory=list)
    angular_momentum: list = field(default_factory=list)
    mass: list = field(default_factory=list)
    charge: list = field(default_factory=list)
    counts: list = field(default_factory=list)
    positions: list = field(default_factory=list)
    velocities: list = field(default_factory=list)
    bath: list = field(default_factory=list)
    species: list = field(default_factory=list)

    @property
    def total_energy(self) -> np.ndarray:
        return (np.array(self.kinetic) + np.array(self.potential) + np.array(self.internal)
                - np.array(self.released))

    def count(self, name) -> np.ndarray:
        return np.array([c.get(name, 0) for c in self.counts])


class Simulation:
    def __init__(self, system, forces=(), reactions=(), integrator=None, dt=None, seed=None):
        if reactions:
            raise NotImplementedError("reactions are not part of the accusim_b200 force-and-step path")
        self.system = system
        self.forces = list(forces)
        self.integrator = integrator or VelocityVerlet()
        self.dt = None if dt is None else si(dt, "s")
        self.rng = np.random.default_rng(seed)
        self.seed = seed
        self.reactions = None
        self.time = 0.0
        self.steps = 0
        self.trajectory = Trajectory()
        self.update_forces()
        self._m0 = self._mass_energy()
        self._initial = None

    def potential(self):
        s = self.system
        f = np.zeros_like(s.pos)
        u = 0.0
        for force in self.forces:
            fi, ui = force.compute(s)
            f += fi
            u += ui
        return f, u

    def update_forces(self):
        self.force, self.pe = self.potential()
        m = self.system.masses
        self.acc = self.force / m[:, None] if len(m) else self.force

    def _mass_energy(self):
        return float(np.sum(self.system.masses))

    def record(self, positions=True):
        s, tr = self.system, self.trajectory
        tr.t.append(self.time)
        tr.kinetic.append(s.kinetic_energy())
        tr.potential.append(self.pe)
        tr.internal.append(float(np.sum(s.eint)))
        tr.released.append(0.0)
        tr.momentum.append(s.momentum())
        tr.angular_momentum.append(s.angular_momentum() if s.dim in (2, 3) else np.zeros(1))
        tr.mass.append(self._mass_energy())
        tr.charge.append(float(np.sum(s.charges)))
        tr.counts.append(s.counts())
        bath = getattr(self.integrator, "bath_energy", None)
        tr.bath.append(bath(s) if bath else 0.0)
        if positions:
            tr.positions.append(s.pos.copy())
            tr.velocities.append(s.vel.copy())
            tr.species.append(s.sp.copy())

    def run(self, duration=None, steps=None, record_every=1, positions=True):
        if self.dt is None:
            raise ValueError("set dt (or use accusim.advisor.suggest_dt)")
        if steps is None:
            steps = int(round(si(duration, "s") / self.dt))
        if not self.trajectory.t:
            if self._initial is None:
                self._initial = self.clone()
            self.record(positions)
        for k in range(1, steps + 1):
            self.integrator.step(self, self.dt)
            self.time += self.dt
            self.steps += 1
            if k % record_every == 0 or k == steps:
                self.record(positions)
        return self.trajectory

    def clone(self, dt=None):
        """Fresh simulation from the current state; Force objects are shared, as in the reference."""
        sim = Simulation.__new__(Simulation)
        sim.__dict__.update(self.__dict__)
        sim.system = self.system.copy()
        sim.forces = list(self.forces)
        sim.integrator = copy.deepcopy(self.integrator)
        sim.rng = np.random.default_rng(self.seed)
        sim.trajectory = Trajectory()
        sim.dt = self.dt if dt is None else dt
        sim.update_forces()
        return sim

    def accuracy_report(self, convergence_duration=None):
        from .accuracy import AccuracyReport
        return AccuracyReport.build(self, convergence_duration)


__all__ = ["Simulation", "Trajectory", "c_light"]
