"""sors_b200: B200-native implicit-Euler FEM step of SORS (Neo-Hookean tets/hexes,
fixed-pattern block-CSR assembly, block-Jacobi PCG Newton) behind the py_sors API.

The compute path is libsors_b200.so (CUDA, sm_100a) through the C ABI in
include/sors_b200.h.
"""
from .py_sors import (Energy, EnergyHex, EnergyTet, IO, Params, SimulationSettings, Solver, SolverHex,  # noqa: F401
                      SolverTet)

__all__ = ["Energy", "EnergyTet", "EnergyHex", "Solver", "SolverTet", "SolverHex", "Params", "SimulationSettings",
           "IO"]
