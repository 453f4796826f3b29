"""pyro_cmc_b200: B200-native (sm_100a) Monte Carlo hot path of pyro_cmc.

Classical Heisenberg spins on the pyrochlore lattice with J1-J3 and a field:
colour-sliced Metropolis + overrelaxation sweeps, FP64 energy reductions, the
static structure factor, batched on-device parallel tempering and
differentiable energy / S(q), all in hand-written CUDA behind the C ABI of
include/pyrocmc.h (libpyrocmc.so, built in-tree).
"""
from .engine import System, pyrochlore_system, displacements, sublattice_offsets  # noqa: F401
from ._lib import PyroCMCError, InvalidArgument, lib_path  # noqa: F401

__all__ = ["System", "pyrochlore_system", "displacements", "sublattice_offsets", "PyroCMCError",
           "InvalidArgument", "lib_path"]
