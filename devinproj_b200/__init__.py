"""devinproj_b200: B200-native (sm_100a) short-range force-and-step path for accusim.

GPU plug-ins that subclass accusim's own classes (`LennardJones`, `DampedShiftedCoulomb`, `VelocityVerlet`,
`Langevin`, `NoseHoover`, `Ewald`) and run inside accusim's `Simulation.run`; `GpuSystem`, an accusim `System`
whose state stays on the GPU; `to_gpu`, which moves a simulation built by accusim's own code onto those plug-ins;
and `GpuSimulation`, the device-resident engine (FP32-compensated pairs, FP64
state, CUDA-graph step loops, batched replicas). All compute is hand-written CUDA in libaccusim_b200.so.
"""
from . import _accusim  # noqa: F401  (accusim, the host framework)
from .analysis import rdf
from .convert import gpu_twin, to_gpu
from .engine import GpuSimulation
from .ensemble import ReplicaEnsemble, calibrate_dt_ensemble, richardson_ensemble
from .ewald import Ewald
from .forces import DampedShiftedCoulomb, LennardJones, VerletList, cell_list_pairs
from .integrators import Langevin, NoseHoover, VelocityVerlet
from .learned import LearnedCorrection
from .state import GpuSystem

__all__ = ["DampedShiftedCoulomb", "Ewald", "GpuSimulation", "GpuSystem", "Langevin", "LearnedCorrection",
           "LennardJones", "NoseHoover", "ReplicaEnsemble", "VelocityVerlet", "VerletList", "calibrate_dt_ensemble",
           "cell_list_pairs", "gpu_twin", "rdf", "richardson_ensemble", "to_gpu"]
__version__ = "0.2.0"
