"""Particle state with the interface of accusim's `System` (accusim/system.py:11-160).

Flat float64 NumPy arrays in SI units: `pos`, `vel` (n, dim); `sp` species index; `ids` stable particle
ids. The GPU plug-ins in this package read only these attributes, so they accept this class or the
reference's own `System` interchangeably.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .units import k_B, si


@dataclass(frozen=True)
class Species:
    name: str
    mass: float
    charge: float = 0.0
    radius: float = 0.0
    diffusion: float = 0.0


class System:
    """Particles in `dim` dimensions; `periodic=True` wraps with minimum-image distances, a
    non-periodic box reflects off its walls (accusim/system.py:20-40)."""

    def __init__(self, dim: int = 3, box=None, periodic: bool = False):
        self.dim = dim
        self.box = None if box is None else np.broadcast_to(si(box, "m"), (dim,)).astype(float).copy()
        self.periodic = bool(periodic) and self.box is not None
        self.species: list[Species] = []
        self._index: dict[str, int] = {}
        self.pos = np.zeros((0, dim))
        self.vel = np.zeros((0, dim))
        self.sp = np.zeros(0, dtype=int)
        self.ids = np.zeros(0, dtype=int)
        self.eint = np.zeros(0)
        self.wall_impulse = 0.0
        self.constrained_dof = 0
        self._next_id = 0

    def add_species(self, name, mass, charge=0.0, radius=0.0, diffusion=0.0) -> Species:
        if name in self._index:
            raise ValueError(f"species '{name}' already defined")
        spc = Species(name, si(mass, "kg"), si(charge, "C"), si(radius, "m"), si(diffusion, "m^2/s"))
        if spc.mass <= 0:
            raise ValueError("mass must be positive")
        self._index[name] = len(self.species)
        self.species.append(spc)
        return spc

    def species_index(self, name: str) -> int:
        if name not in self._index:
            raise KeyError(f"unknown species '{name}'")
        return self._index[name]

    def add(self, species: str, pos, vel=None, eint=0.0) -> np.ndarray:
        p = np.atleast_2d(si(pos, "m")).astype(float)
        if p.shape[1] != self.dim:
            raise ValueError(f"positions must have {self.dim} components")
        v = np.zeros_like(p) if vel is None else np.broadcast_to(np.atleast_2d(si(vel, "m/s")), p.shape).astype(float)
        k = len(p)
        new_ids = np.arange(self._next_id, self._next_id + k)
        self._next_id += k
        self.pos = np.vstack([self.pos, p])
        self.vel = np.vstack([self.vel, v])
        self.sp = np.concatenate([self.sp, np.full(k, self.species_index(species))])
        self.ids = np.concatenate([self.ids, new_ids])
        self.eint = np.concatenate([self.eint, np.broadcast_to(np.asarray(eint, float), (k,))])
        return new_ids

    def remove(self, mask):
        keep = ~np.asarray(mask)
        self.pos, self.vel, self.sp, self.ids, self.eint = (self.pos[keep], self.vel[keep], self.sp[keep],
                                                            self.ids[keep], self.eint[keep])

    @property
    def n(self) -> int:
        return len(self.pos)

    def species_table(self, attr: str) -> np.ndarray:
        return np.array([getattr(x, attr) for x in self.species], dtype=float)

    @property
    def masses(self) -> np.ndarray:
        return self.species_table("mass")[self.sp] if self.n else np.zeros(0)

    @property
    def charges(self) -> np.ndarray:
        return self.species_table("charge")[self.sp] if self.n else np.zeros(0)

    def count(self, name: str) -> int:
        return int(np.sum(self.sp == self.species_index(name)))

    def counts(self) -> dict:
        return {x.name: int(np.sum(self.sp == k)) for k, x in enumerate(self.species)}

    def displacements(self, idx_a=None, idx_b=None) -> np.ndarray:
        a = self.pos if idx_a is None else self.pos[idx_a]
        b = self.pos if idx_b is None else self.pos[idx_b]
        d = b[None, :, :] - a[:, None, :]
        if self.periodic:
            d -= self.box * np.round(d / self.box)
        return d

    def kinetic_energy(self) -> float:
        return 0.5 * float(np.sum(self.masses[:, None] * self.vel ** 2))

    def momentum(self) -> np.ndarray:
        return np.sum(self.masses[:, None] * self.vel, axis=0)

    def angular_momentum(self) -> np.ndarray:
        return np.atleast_1d(np.sum(np.cross(self.pos, self.masses[:, None] * self.vel), axis=0))

    def center_of_mass_velocity(self) -> np.ndarray:
        return self.momentum() / np.sum(self.masses)

    def temperature(self) -> float:
        dof = max(self.dim * self.n - self.dim - self.constrained_dof, 1)
        return 2 * self.kinetic_energy() / (dof * k_B)

    def apply_boundaries(self):
        """Periodic wrap or elastic walls (accusim/system.py:124-140)."""
        if self.box is None:
            return
        if self.periodic:
            self.pos %= self.box
            return
        for _ in range(4):
            low, high = self.pos < 0, self.pos > self.box
            if not (low.any() or high.any()):
                break
            self.pos = np.where(low, -self.pos, self.pos)
            self.pos = np.where(high, 2 * self.box - self.pos, self.pos)
            hit = low | high
            m = self.masses
            self.wall_impulse += float(np.sum(2 * m[:, None] * np.abs(self.vel) * hit))
            self.vel = np.where(hit, -self.vel, self.vel)

    def copy(self) -> "System":
        other = System.__new__(System)
        other.__dict__.update(self.__dict__)
        for k in ("pos", "vel", "sp", "ids", "eint"):
            setattr(other, k, getattr(self, k).copy())
        other.species = list(self.species)
        other._index = dict(self._index)
        other.box = None if self.box is None else self.box.copy()
        return other

    def maxwell_boltzmann(self, temperature, rng=None, zero_momentum=True):
        """Gaussian velocities at `temperature` with the net momentum removed (accusim/system.py:152-160)."""
        rng = rng or np.random.default_rng()
        T = si(temperature, "K")
        sigma = np.sqrt(k_B * T / self.masses)[:, None]
        self.vel = rng.normal(size=self.pos.shape) * sigma
        if zero_momentum and self.n > 1:
            self.vel -= self.center_of_mass_velocity()


def species_arrays(s):
    """(names, masses, charges) of any accusim-shaped system (this class or the reference's)."""
    names = [x.name for x in s.species]
    return names, np.array([x.mass for x in s.species], float), np.array([x.charge for x in s.species], float)
