"""GPU drop-ins for accusim's `VelocityVerlet`, `Langevin` and `NoseHoover` (accusim/integrators.py:9-116).

`step(sim, dt)` performs kick-drift-wrap-force-kick with FP64 kernels in the reference's IEEE operation
order (no FMA), so given the same accelerations it is bit-identical to the reference step. When every
force of the simulation is a GPU plug-in the forces are evaluated on the device positions directly;
otherwise `sim.update_forces()` runs the plug-in protocol unchanged.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import require_cuda, stream_handle, to_dev
from .units import k_B, si


class Integrator:
    order = 1
    symplectic = False
    stochastic = False
    thermostat = False

    def step(self, sim, dt):
        raise NotImplementedError


def _masses_table(s):
    return np.ascontiguousarray([x.mass for x in s.species], dtype=np.float64)


def device_forces(sim, pos_d, sp_d):
    """Sum of the forces of `sim` on device positions; None if some force is not a GPU plug-in."""
    from .forces import DampedShiftedCoulomb, LennardJones
    s = sim.system
    F = None
    U = None
    for f in sim.forces:
        if isinstance(f, LennardJones):
            Fi, Ui = f.compute_device(s, pos_d, sp_d)
        elif isinstance(f, DampedShiftedCoulomb):
            Fi, Ui = f.compute_device(s, pos_d)
        else:
            return None
        F = Fi.clone() if F is None else F.add_(Fi)
        U = Ui.clone() if U is None else U.add_(Ui)
    if F is None:
        F = torch.zeros((s.n, 3), dtype=torch.float64, device="cuda")
        U = torch.zeros(1, dtype=torch.float64, device="cuda")
    return F, U


def _begin(sim):
    """Upload the state for a device step: (library, stream, n, pos, vel, acc) device tensors."""
    s = sim.system
    if s.dim != 3:
        raise ValueError("accusim_b200 integrators handle 3-dimensional systems")
    require_cuda()
    return (_lib.lib(), stream_handle(), s.n, to_dev(s.pos), to_dev(s.vel),
            to_dev(np.asarray(sim.acc, dtype=np.float64)))


def _drift(L, st, s, pos_d, vel_d, n, dt, wrap):
    """pos += dt * vel, then pos %= box for periodic boxes when `wrap`."""
    boxarr, boxp = _lib.dbl3(s.box) if (wrap and s.box is not None) else (None, None)
    periodic = 1 if (wrap and s.box is not None and s.periodic) else 0
    _lib.check(L.acs_vv_drift_wrap(pos_d.data_ptr(), vel_d.data_ptr(), n, float(dt), boxp, periodic, st),
               "acs_vv_drift_wrap")


def _finish(sim, L, st, pos_d, vel_d, acc_d, h):
    """Walls, forces at the new positions (device plug-ins, else the plug-in protocol), the closing kick
    and the download: accusim/integrators.py:29-31."""
    s = sim.system
    n = s.n
    if s.box is not None and not s.periodic:
        # elastic walls: the reference's reflection and wall-impulse ledger (accusim/system.py:130-140)
        s.pos = pos_d.cpu().numpy()
        s.vel = vel_d.cpu().numpy()
        s.apply_boundaries()
        pos_d, vel_d = to_dev(s.pos), to_dev(s.vel)
    sp_d = to_dev(s.sp, torch.int32)
    res = device_forces(sim, pos_d, sp_d)
    if res is None:
        s.pos = pos_d.cpu().numpy()
        s.vel = vel_d.cpu().numpy()
        sim.update_forces()
        acc_d = to_dev(np.asarray(sim.acc, dtype=np.float64))
    else:
        F_d, U_d = res
        m = _masses_table(s)
        _lib.check(L.acs_vv_accel(acc_d.data_ptr(), F_d.data_ptr(), sp_d.data_ptr(), m.ctypes.data, len(m), n,
                                  st), "acs_vv_accel")
        s.pos = pos_d.cpu().numpy()
        sim.force = F_d.cpu().numpy()
        sim.pe = float(U_d.item())
        sim.acc = acc_d.cpu().numpy()
    _lib.check(L.acs_vv_kick(vel_d.data_ptr(), acc_d.data_ptr(), n, h, st), "acs_vv_kick")
    s.vel = vel_d.cpu().numpy()


class VelocityVerlet(Integrator):
    """Kick-drift-kick leapfrog: 2nd order, symplectic, time reversible."""

    order = 2
    symplectic = True

    def step(self, sim, dt):
        L, st, n, pos_d, vel_d, acc_d = _begin(sim)
        h = 0.5 * dt
        _lib.check(L.acs_vv_kick(vel_d.data_ptr(), acc_d.data_ptr(), n, h, st), "acs_vv_kick")
        _drift(L, st, sim.system, pos_d, vel_d, n, dt, True)
        _finish(sim, L, st, pos_d, vel_d, acc_d, h)


class Langevin(Integrator):
    """BAOAB Langevin dynamics (Leimkuhler-Matthews), accusim/integrators.py:50-71: samples temperature T.

    Same operations in the same IEEE order as the reference, with the normal draws taken from `sim.rng` as
    the reference takes them, so a step is bit-identical to the reference's given the same accelerations and
    generator state. B and A run on the device (acs_vv_kick, acs_vv_drift_wrap), O is acs_langevin_ou."""

    order = 2
    stochastic = True
    thermostat = True

    def __init__(self, temperature, friction):
        self.T = si(temperature, "K")
        self.gamma = si(friction, "1/s")

    def step(self, sim, dt):
        s = sim.system
        L, st, n, pos_d, vel_d, acc_d = _begin(sim)
        h = 0.5 * dt
        _lib.check(L.acs_vv_kick(vel_d.data_ptr(), acc_d.data_ptr(), n, h, st), "acs_vv_kick")
        _drift(L, st, s, pos_d, vel_d, n, h, False)
        c1 = np.exp(-self.gamma * dt)
        sig = np.ascontiguousarray(np.sqrt((1 - c1 ** 2) * k_B * self.T / s.masses), dtype=np.float64)
        noise = to_dev(np.ascontiguousarray(sim.rng.normal(size=s.vel.shape), dtype=np.float64))
        sig_d = to_dev(sig)
        _lib.check(L.acs_langevin_ou(vel_d.data_ptr(), noise.data_ptr(), sig_d.data_ptr(), n, float(c1), st),
                   "acs_langevin_ou")
        _drift(L, st, s, pos_d, vel_d, n, h, True)
        _finish(sim, L, st, pos_d, vel_d, acc_d, h)


class NoseHoover(Integrator):
    """Nose-Hoover thermostat with the Trotter splitting of accusim/integrators.py:74-116 (Martyna-Tuckerman-
    Klein): canonical sampling with the conserved extended energy E + Q xi^2 / 2 + N_f kT eta.

    The thermostat half-steps are O(n) scalar updates on the host arrays, with the reference's NumPy
    expressions (so the kinetic-energy sum has the reference's summation order); the VelocityVerlet step
    between them runs on the device. `period` sets the thermostat mass Q = N_f kT period^2."""

    order = 2
    thermostat = True

    def __init__(self, temperature, period):
        self.T = si(temperature, "K")
        self.tau = si(period, "s")
        self.xi = 0.0
        self.eta = 0.0
        self.Q = None
        self._vv = VelocityVerlet()

    @staticmethod
    def dof(s):
        return s.dim * max(s.n - 1, 1)

    def _half(self, s, dt):
        kT, nf = k_B * self.T, self.dof(s)
        if self.Q is None:
            self.Q = nf * kT * self.tau ** 2
        k2 = float(np.sum(s.masses[:, None] * s.vel ** 2))
        self.xi += 0.25 * dt * (k2 - nf * kT) / self.Q
        scale = np.exp(-0.5 * dt * self.xi)
        s.vel *= scale
        self.eta += 0.5 * dt * self.xi
        self.xi += 0.25 * dt * (k2 * scale ** 2 - nf * kT) / self.Q

    def step(self, sim, dt):
        s = sim.system
        self._half(s, dt)
        self._vv.step(sim, dt)
        self._half(s, dt)

    def bath_energy(self, s):
        if self.Q is None:
            return 0.0
        return 0.5 * self.Q * self.xi ** 2 + self.dof(s) * k_B * self.T * self.eta
