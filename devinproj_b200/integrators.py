"""GPU drop-ins for accusim's `VelocityVerlet`, `Langevin` and `NoseHoover` (accusim/integrators.py:19-116).

The classes subclass accusim's own (class flags, constructor arguments, the Nose-Hoover thermostat state and its
half-steps `_half`, `dof`, `bath_energy` are inherited) and replace the kick-drift-wrap-force-kick with FP64
kernels in the reference's IEEE operation order (no FMA): given the same accelerations a step is bit-identical
to the reference's. When every force of the simulation is one of this package's GPU plug-ins the forces are
evaluated on the device positions directly; otherwise `sim.update_forces()` runs accusim's plug-in protocol.

On a `GpuSystem` the state stays on the device across steps: positions, velocities and accelerations are not
copied back; `sim.force` and `sim.acc` are refreshed when the host next reads the system (accusim's
`Simulation.record` does), and only the potential energy `sim.pe` (a float in accusim's contract) is read back
every step. On any other accusim `System` each step uploads the state and downloads it again.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._accusim import integrators as _ai
from .device import require_cuda, stream_handle, to_dev
from .state import is_gpu_system
from .units import k_B


def _masses_table(s):
    return np.ascontiguousarray([x.mass for x in s.species], dtype=np.float64)


def device_forces(sim, pos_d, sp_d):
    """Sum of the forces of `sim` on device positions as (F (n, 3), U (1,)) device tensors; None if some force
    is not one of this package's GPU plug-ins."""
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


class _DeviceStep:
    """One integrator step's device state: positions, velocities, accelerations and species of `sim.system`
    on the GPU (the resident copy of a GpuSystem, else uploaded from the host arrays)."""

    def __init__(self, sim):
        s = sim.system
        if s.dim != 3:
            raise ValueError("accusim_b200 integrators handle 3-dimensional systems")
        require_cuda()
        self.sim, self.s = sim, s
        self.L, self.st, self.n = _lib.lib(), stream_handle(), s.n
        self.resident = is_gpu_system(s)
        if self.resident:
            self.pos, self.vel = s.device_state()
            acc = s.device_acc()
            self.acc = acc if acc is not None else to_dev(np.asarray(sim.acc, dtype=np.float64))
            self.sp = s.device_species()
        else:
            self.pos, self.vel = to_dev(s.pos), to_dev(s.vel)
            self.acc = to_dev(np.asarray(sim.acc, dtype=np.float64))
            self.sp = None

    def kick(self, h):
        """vel += h * acc"""
        _lib.check(self.L.acs_vv_kick(self.vel.data_ptr(), self.acc.data_ptr(), self.n, h, self.st), "acs_vv_kick")

    def drift(self, dt, wrap):
        """pos += dt * vel, then pos %= box for periodic boxes when `wrap`."""
        s = self.s
        boxarr, boxp = _lib.dbl3(s.box) if (wrap and s.box is not None) else (None, None)
        periodic = 1 if (wrap and s.box is not None and s.periodic) else 0
        _lib.check(self.L.acs_vv_drift_wrap(self.pos.data_ptr(), self.vel.data_ptr(), self.n, float(dt), boxp,
                                            periodic, self.st), "acs_vv_drift_wrap")

    def forces_and_kick(self, h):
        """Walls, forces at the new positions (device plug-ins, else the plug-in protocol on host arrays), the
        closing kick, and the hand-back of the state: accusim/integrators.py:29-31."""
        sim, s = self.sim, self.s
        walls = s.box is not None and not s.periodic
        sp = self.sp if self.sp is not None else to_dev(np.asarray(s.sp), torch.int32)
        res = None if walls else device_forces(sim, self.pos, sp)
        if res is None:
            # elastic walls (accusim/system.py:130-140) or a force without a device path: host protocol
            s.pos = self.pos.cpu().numpy()
            s.vel = self.vel.cpu().numpy()
            if walls:
                s.apply_boundaries()
            sim.update_forces()
            self.vel = to_dev(s.vel)
            self.acc = to_dev(np.asarray(sim.acc, dtype=np.float64))
            self.kick(h)
            s.vel = self.vel.cpu().numpy()
            return
        F, U = res
        m = _masses_table(s)
        _lib.check(self.L.acs_vv_accel(self.acc.data_ptr(), F.data_ptr(), sp.data_ptr(), m.ctypes.data, len(m),
                                       self.n, self.st), "acs_vv_accel")
        self.kick(h)
        sim.pe = float(U.item())
        if self.resident:
            mirrors = []
            for name, dev in (("force", F), ("acc", self.acc)):
                host = getattr(sim, name, None)
                if not (isinstance(host, np.ndarray) and host.shape == (self.n, 3) and host.dtype == np.float64):
                    host = np.empty((self.n, 3))
                    setattr(sim, name, host)
                mirrors.append((host, dev))
            s.stepped_on_device(self.acc, F, mirrors)
        else:
            s.pos = self.pos.cpu().numpy()
            sim.force = F.cpu().numpy()
            sim.acc = self.acc.cpu().numpy()
            s.vel = self.vel.cpu().numpy()


class VelocityVerlet(_ai.VelocityVerlet):
    """accusim's kick-drift-kick leapfrog (2nd order, symplectic) with the step on the GPU."""

    def step(self, sim, dt):
        d = _DeviceStep(sim)
        h = 0.5 * dt
        d.kick(h)
        d.drift(dt, True)
        d.forces_and_kick(h)


class Langevin(_ai.Langevin):
    """accusim's BAOAB Langevin dynamics (Leimkuhler-Matthews) with B and A on the GPU.

    The normal draws come from `sim.rng` exactly as the reference takes them, and the O-step runs as
    acs_langevin_ou in the reference's operation order, so a step is bit-identical to the reference's given the
    same accelerations and generator state."""

    def step(self, sim, dt):
        s = sim.system
        d = _DeviceStep(sim)
        h = 0.5 * dt
        d.kick(h)
        d.drift(h, False)
        c1 = np.exp(-self.gamma * dt)
        masses = _masses_table(s)[np.asarray(s.host_species() if d.resident else s.sp)]
        sig = np.ascontiguousarray(np.sqrt((1 - c1 ** 2) * k_B * self.T / masses), dtype=np.float64)
        noise = to_dev(np.ascontiguousarray(sim.rng.normal(size=(d.n, s.dim)), dtype=np.float64))
        sig_d = to_dev(sig)
        _lib.check(d.L.acs_langevin_ou(d.vel.data_ptr(), noise.data_ptr(), sig_d.data_ptr(), d.n, float(c1), d.st),
                   "acs_langevin_ou")
        d.drift(h, True)
        d.forces_and_kick(h)


class NoseHoover(_ai.NoseHoover):
    """accusim's Nose-Hoover thermostat (Trotter splitting, Martyna-Tuckerman-Klein): the thermostat half-steps
    are accusim's own (`_half`, on the host arrays, so the kinetic-energy sum keeps the reference's summation
    order); the VelocityVerlet step between them runs on the GPU."""

    def step(self, sim, dt):
        s = sim.system
        self._half(s, dt)
        VelocityVerlet.step(self, sim, dt)
        self._half(s, dt)
