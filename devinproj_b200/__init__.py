"""accusim_b200: B200-native (sm_100a) short-range force-and-step path of accusim.

Drop-in plug-ins with the reference's interfaces (`LennardJones`, `DampedShiftedCoulomb`,
`VelocityVerlet`, driven by `Simulation.run`) backed by hand-written CUDA in libaccusim_b200.so.
"""
from .accuracy import AccuracyReport, calibrate_dt, suggest_dt, timescales, timestep_convergence
from .engine import GpuSimulation
from .ewald import Ewald
from .learned import LearnedCorrection
from .forces import DampedShiftedCoulomb, Force, LennardJones, VerletList, cell_list_pairs
from .integrators import Integrator, Langevin, NoseHoover, VelocityVerlet
from .simulation import Simulation, Trajectory
from .system import Species, System
from .units import k_B, k_e

__all__ = ["AccuracyReport", "Ewald", "GpuSimulation", "LearnedCorrection", "DampedShiftedCoulomb", "Force", "Integrator", "LennardJones", "Simulation",
           "Langevin", "NoseHoover", "Species", "System", "Trajectory", "VelocityVerlet", "VerletList", "calibrate_dt", "cell_list_pairs",
           "k_B", "k_e", "suggest_dt", "timescales", "timestep_convergence"]
__version__ = "0.1.0"
