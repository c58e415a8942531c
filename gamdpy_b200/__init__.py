"""gamdpy_b200: gamdpy's molecular-dynamics hot path on NVIDIA B200.

Drop-in for the part of gamdpy's API that runs the simulation hot path --
pair-potential forces/virial/energy over N^2 or cell neighbour lists (with
exclusions, plus harmonic bonds for molecules), the NVE,
NVT (Nose-Hoover), NVT_Langevin and NPT_Atomic steps, ScalarSaver / MomentumReset /
ConfigurationSaver, and the RDF and S(q) calculators.  The compute path is the hand-written
sm_100a CUDA library libgamdb200.so (include/gamdb200.h), called through
ctypes.  There is no CPU fallback: operations raise if the library is missing.

    import gamdpy_b200 as gp      # in place of: import gamdpy as gp
"""
from . import integrators as _integrators_mod
from .calculators import CalculatorRadialDistribution, CalculatorStructureFactor
from .configuration import (Configuration, colarray, generate_random_velocities, get_default_compute_flags,
                            make_lattice, unit_cells)
from .interactions import Bonds, Interaction, NbList2, NbListLinkedLists, PairPotential
from .misc import extract_scalars, make_function_constant, make_function_ramp
from .potential_functions import (LJ_12_6, LJ_12_6_sigma_epsilon, apply_shifted_force_cutoff,
                                  apply_shifted_potential_cutoff, harmonic_bond_function)
from .runtime_actions import ConfigurationSaver, MomentumReset, RuntimeAction, ScalarSaver
from .simulation import Simulation, get_default_compute_plan, get_default_sim
from .batch import SimulationBatch
from .simulation_boxes import Orthorhombic
from .tools import Evaluator, calc_dynamics

integrators = _integrators_mod

__version__ = "0.1.0"
