"""`GpuSystem`: accusim's `System` (accusim/system.py:20-160) with positions and velocities resident on the GPU.

The FP64 plug-ins of this package step a `GpuSystem` on the device without copying the state back every step.
The host arrays (`pos`, `vel`, and `sp`, `ids`) are accusim's attributes turned into properties that synchronise
lazily:

* reading or assigning one of them on the host makes the host copy authoritative (the caller may modify the
  returned array in place); the next device step uploads it again;
* a device step (this package's integrators) makes the device copy authoritative; the next host read
  downloads it, together with the simulation's `force` and `acc` arrays that the integrator registered.

Inside `accusim.Simulation.run` with this package's integrator and forces, the state therefore crosses PCIe only
at `record` steps (which read `pos`, `vel` and `sp` for the kinetic energy, momenta and counts); every other
step runs on device-resident arrays. Everything else of accusim's `System` is inherited unchanged.
"""
from __future__ import annotations

import numpy as np
import torch

from ._accusim import system as _asys
from .device import to_dev


class GpuSystem(_asys.System):
    """accusim `System` whose `pos`/`vel` (FP64, SI) stay on the GPU between host accesses."""

    _OWN = ("_where", "_pos", "_vel", "_sp", "_ids", "_pos_d", "_vel_d", "_sp_d", "_ids_version", "_mirrors",
            "_acc_d", "_force_d")

    def _fresh(self):
        self.__dict__.update(_where="host", _pos=None, _vel=None, _sp=None, _ids=None, _pos_d=None, _vel_d=None,
                             _sp_d=None, _ids_version=0, _mirrors=[], _acc_d=None, _force_d=None)

    def __init__(self, dim: int = 3, box=None, periodic: bool = False):
        self._fresh()
        super().__init__(dim, box, periodic)

    @classmethod
    def from_system(cls, s) -> "GpuSystem":
        """A GpuSystem holding a copy of an accusim system's state (species, arrays, box, counters)."""
        g = cls.__new__(cls)
        g._fresh()
        for k, v in s.__dict__.items():
            if k in cls._OWN or k in ("pos", "vel", "sp", "ids"):
                continue
            g.__dict__[k] = v.copy() if isinstance(v, (np.ndarray, list, dict)) else v
        g.pos = np.array(s.pos, dtype=float)
        g.vel = np.array(s.vel, dtype=float)
        g.sp = np.array(s.sp)
        g.ids = np.array(s.ids)
        return g

    # ---------------------------------------------------------------- lazily synchronised host arrays
    def _host(self):
        """Make the host arrays current (download after device steps) and authoritative."""
        if self._where == "device":
            self._pos = self._pos_d.cpu().numpy()
            self._vel = self._vel_d.cpu().numpy()
            for host, dev in self._mirrors:
                np.copyto(host, dev.cpu().numpy().reshape(host.shape))
        self._where = "host"
        self._acc_d = self._force_d = None

    @property
    def pos(self):
        self._host()
        return self._pos

    @pos.setter
    def pos(self, value):
        self._host()
        self._pos = value

    @property
    def vel(self):
        self._host()
        return self._vel

    @vel.setter
    def vel(self, value):
        self._host()
        self._vel = value

    @property
    def sp(self):
        self._sp_d = None
        return self._sp

    @sp.setter
    def sp(self, value):
        self._sp_d = None
        self._sp = value

    @property
    def ids(self):
        self._ids_version += 1
        return self._ids

    @ids.setter
    def ids(self, value):
        self._ids_version += 1
        self._ids = value

    @property
    def n(self) -> int:
        return len(self._pos_d) if self._where == "device" else len(self._pos)

    # ---------------------------------------------------------------- device side (this package's plug-ins)
    def device_state(self):
        """(pos, vel) device tensors (n, 3) FP64, uploaded if the host copy is authoritative."""
        if self._where == "host":
            self._pos_d = to_dev(np.asarray(self._pos, dtype=np.float64))
            self._vel_d = to_dev(np.asarray(self._vel, dtype=np.float64))
            self._where = "both"
        return self._pos_d, self._vel_d

    def device_species(self):
        """Species indices as a device int32 tensor (cached until `sp` is touched on the host)."""
        if self._sp_d is None:
            self._sp_d = {"sp": to_dev(np.asarray(self._sp), torch.int32)}
        return self._sp_d["sp"]

    def device_charges(self):
        """(per-atom charges as a device FP64 tensor, whether any is non-zero), cached like the species."""
        self.device_species()
        if "q" not in self._sp_d:
            q = np.array([x.charge for x in self.species], dtype=np.float64)[np.asarray(self._sp)]
            self._sp_d["q"] = (to_dev(q), bool(np.any(q)))
        return self._sp_d["q"]

    def host_species(self):
        """The host species indices, read without invalidating the device copy (the caller must not modify)."""
        return self._sp

    def ids_version(self) -> int:
        """Counter bumped by every host access to `ids`: unchanged means the ids cannot have changed."""
        return self._ids_version

    def stepped_on_device(self, acc_d, force_d, mirrors):
        """Record a device step: the device state is authoritative, `acc_d` holds the accelerations of the
        current positions, and the host arrays in `mirrors` [(host array, device tensor)] are refreshed when
        the host next reads the state."""
        self._where = "device"
        self._acc_d = acc_d
        self._force_d = force_d
        self._mirrors = mirrors

    def device_acc(self):
        """Accelerations of the current device positions from the last device step, or None."""
        return self._acc_d if self._where in ("device", "both") else None

    def copy(self) -> "GpuSystem":
        """A host-authoritative copy (accusim's `System.copy` would return the base class)."""
        return GpuSystem.from_system(self)


def is_gpu_system(s) -> bool:
    return isinstance(s, GpuSystem)
