"""Seeded synthetic inputs for the benchmark configurations of this path.

Lattices follow the reference's own example setups: fcc with basis [[0,0,0],[.5,.5,0],[.5,0,.5],[0,.5,.5]]
+ 0.25 (examples/rahman_argon.py:23-27) and rock-salt by grid parity with a +0.5 offset
(examples/molten_salt.py:26-33). Systems are accusim `System` objects (a `GpuSystem` with gpu=True), with
velocities from accusim's `System.maxwell_boltzmann` and `np.random.default_rng(seed)`
(accusim/system.py:152-160). Reduced LJ units map to SI through argon (sigma = 3.4 A, eps/kB = 120 K,
m = 39.948 u).
"""
from __future__ import annotations

import math

import numpy as np

from ._accusim import system as _asys
from .forces import DampedShiftedCoulomb, LennardJones
from .state import GpuSystem
from .units import N_A, amu, e_charge, k_B


def _new_system(L, gpu):
    return (GpuSystem if gpu else _asys.System)(3, box=L, periodic=True)

AR_SIGMA = 3.4e-10
AR_EPS = 120 * k_B
AR_MASS = 39.948 * amu
AR_TAU = AR_SIGMA * math.sqrt(AR_MASS / AR_EPS)   # 2.151 ps

NA_MASS, CL_MASS = 22.98977 * amu, 35.453 * amu
NACL_LJ = {"Na": (0.544e3 / N_A, 2.35e-10), "Cl": (0.418e3 / N_A, 4.40e-10)}


def fcc_positions(n_cells: int, L: float) -> np.ndarray:
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) + 0.25
    g = np.stack(np.meshgrid(*[np.arange(n_cells)] * 3, indexing="ij"), -1).reshape(-1, 1, 3)
    return ((g + base[None]).reshape(-1, 3)) * L / n_cells


def lj_fluid(n_cells: int, rho_star: float = 0.8442, T_star: float = 0.72, seed: int = 0, L_sigma=None,
             gpu: bool = False):
    """Argon fcc lattice of n_cells^3 unit cells (4 n_cells^3 atoms) at reduced density rho*, MB velocities
    at T*; returns (system, LennardJones)."""
    n = 4 * n_cells ** 3
    L = (L_sigma if L_sigma is not None else (n / rho_star) ** (1 / 3)) * AR_SIGMA
    s = _new_system(L, gpu)
    s.add_species("Ar", AR_MASS)
    s.add("Ar", fcc_positions(n_cells, L))
    s.maxwell_boltzmann(T_star * 120.0, np.random.default_rng(seed))
    return s, LennardJones({"Ar": (AR_EPS, AR_SIGMA)}, cutoff=2.5, skin=0.3)


def argon864(seed: int = 0, gpu: bool = False):
    """864 Ar, fcc 6^3, box 10.229 sigma, 94.4 K, dt 10 fs (the FP64 CPU-runnable case)."""
    s, lj = lj_fluid(6, seed=seed, L_sigma=10.229, gpu=gpu)
    s.maxwell_boltzmann(94.4, np.random.default_rng(seed))
    return s, [lj], 10 * 1e-15


def nacl_melt(n_sites: int = 16, density_g_cm3: float = 1.55, T: float = 1200.0, rcut=12e-10, alpha=0.2e10,
              seed: int = 0, gpu: bool = False):
    """Rock-salt lattice of n_sites^3 ions (n_sites/2 conventional cells per edge) at the given density,
    +-1 e charges, LJ with Lorentz-Berthelot mixing plus DSF; returns (system, [lj, dsf])."""
    mass_g = n_sites ** 3 / 2 * (22.98977 + 35.453) / N_A
    L = (mass_g / density_g_cm3) ** (1 / 3) * 1e-2
    s = _new_system(L, gpu)
    s.add_species("Na", NA_MASS, charge=e_charge)
    s.add_species("Cl", CL_MASS, charge=-e_charge)
    g = np.stack(np.meshgrid(*[np.arange(n_sites)] * 3, indexing="ij"), -1).reshape(-1, 3)
    odd = g.sum(1) % 2 == 1
    s.add("Na", (g[~odd] + 0.5) * L / n_sites)
    s.add("Cl", (g[odd] + 0.5) * L / n_sites)
    s.maxwell_boltzmann(T, rng=np.random.default_rng(seed))
    lj = LennardJones(NACL_LJ, cutoff=2.5)
    dsf = DampedShiftedCoulomb(rcut=rcut, alpha=alpha)
    return s, [lj, dsf]


def nacl4096(seed: int = 0, gpu: bool = False):
    """4096-ion molten-salt case: 16^3 sites, 1.55 g/cm^3, 1200 K, DSF alpha 0.2/A rc 12 A, dt 1 fs."""
    s, forces = nacl_melt(16, seed=seed, gpu=gpu)
    return s, forces, 1e-15


def nacl8000(seed: int = 0):
    """8000-ion melt for the learned DSF->Ewald correction: 20^3 sites, 1300 K, DSF rc 10 A."""
    s, forces = nacl_melt(20, T=1300.0, rcut=10e-10, seed=seed)
    return s, forces, 1e-15


def replica_sizes(n_replicas: int = 256, seed: int = 0):
    """Atom counts log-uniform in [256, 32000], rounded to fcc sizes 4 nc^3 with nc in [4, 20]."""
    rng = np.random.default_rng(seed)
    u = np.exp(rng.uniform(np.log(256), np.log(32000), n_replicas))
    nc = np.clip(np.rint((u / 4) ** (1 / 3)), 4, 20).astype(int)
    return nc


def lj_large(n_cells: int = 64, seed: int = 0, gpu: bool = False):
    """1,048,576-atom LJ fluid at n_cells=64: rho* 0.8442, T* 0.72, rc 2.5 sigma, skin 0.3 sigma,
    dt* 0.005."""
    s, lj = lj_fluid(n_cells, seed=seed, gpu=gpu)
    return s, [lj], 0.005 * AR_TAU
