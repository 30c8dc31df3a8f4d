"""GPU drop-in for accusim's `VelocityVerlet` (accusim/integrators.py:9-31).

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


class VelocityVerlet(Integrator):
    """Kick-drift-kick leapfrog: 2nd order, symplectic, time reversible."""

    order = 2
    symplectic = True

    def step(self, sim, dt):
        s = sim.system
        if s.dim != 3:
            raise ValueError("accusim_b200 VelocityVerlet handles 3-dimensional systems")
        require_cuda()
        L = _lib.lib()
        st = stream_handle()
        n = s.n
        pos_d = to_dev(s.pos)
        vel_d = to_dev(s.vel)
        acc_d = to_dev(np.asarray(sim.acc, dtype=np.float64))
        h = 0.5 * dt
        _lib.check(L.acs_vv_kick(vel_d.data_ptr(), acc_d.data_ptr(), n, h, st), "acs_vv_kick")
        boxarr, boxp = _lib.dbl3(s.box) if s.box is not None else (None, None)
        periodic = 1 if (s.box is not None and s.periodic) else 0
        _lib.check(L.acs_vv_drift_wrap(pos_d.data_ptr(), vel_d.data_ptr(), n, float(dt), boxp, periodic, st),
                   "acs_vv_drift_wrap")
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
