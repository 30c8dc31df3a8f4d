"""Move an accusim `Simulation` onto the GPU path in place, for simulations built by accusim's own code (for example
`accusim.model.build` from a JSON model, accusim/model.py:102-135, or a script that uses accusim's classes).

Each force and integrator that this package has a GPU plug-in for is replaced by that plug-in, carrying the same
parameters and state (all SI already, so they are taken over as they are, attribute by attribute), and the system
becomes a `GpuSystem` when `resident` is set. Everything else (bonds, external fields, reactions, other
integrators) stays accusim's own and runs through its plug-in protocol on the host arrays, as the GPU integrators
already allow.
"""
from __future__ import annotations

from ._accusim import forces as _af
from ._accusim import integrators as _ai


def _gpu_classes():
    from .ewald import Ewald
    from .forces import DampedShiftedCoulomb, LennardJones, VerletList, _Scratch
    from .integrators import Langevin, NoseHoover, VelocityVerlet

    def fresh_lists(obj):
        obj._vl = VerletList()
        obj._scr = _Scratch()

    def nothing(obj):
        pass

    # accusim class -> (GPU class, state the GPU plug-in keeps of its own); the exact class is matched, so a
    # user's own subclass of an accusim class is left alone
    return {_af.LennardJones: (LennardJones, fresh_lists), _af.DampedShiftedCoulomb: (DampedShiftedCoulomb, fresh_lists),
            _af.Ewald: (Ewald, nothing), _ai.VelocityVerlet: (VelocityVerlet, nothing), _ai.Langevin: (Langevin, nothing),
            _ai.NoseHoover: (NoseHoover, nothing)}


def gpu_twin(obj):
    """The GPU plug-in with the parameters and state of an accusim force or integrator, or `obj` itself when this
    package has none for its class (or it is already a GPU plug-in)."""
    table = _gpu_classes()
    entry = table.get(type(obj))
    if entry is None:
        return obj
    cls, init_own = entry
    twin = cls.__new__(cls)
    twin.__dict__.update({k: v for k, v in obj.__dict__.items() if k not in ("_vl", "_scr", "_kcache")})
    if isinstance(obj, _af.Ewald):
        twin._kcache = None
    init_own(twin)
    return twin


def to_gpu(sim, resident: bool = True):
    """Swap `sim`'s forces and integrator for their GPU plug-ins (`gpu_twin`) and, with `resident`, its system for
    a `GpuSystem` holding the same state (not for a simulation with reactions, whose engine keeps the system it
    was built with, nor for 1- or 2-dimensional systems); the force, acceleration and potential energy of the
    current state are recomputed with the new plug-ins. The plug-ins start with empty neighbour lists (their
    `rebuilds` counters restart at zero). Returns `sim`."""
    from .state import GpuSystem, is_gpu_system
    sim.forces = [gpu_twin(f) for f in sim.forces]
    sim.integrator = gpu_twin(sim.integrator)
    if resident and sim.reactions is None and not is_gpu_system(sim.system) and sim.system.dim == 3:
        sim.system = GpuSystem.from_system(sim.system)
    sim.update_forces()
    return sim
