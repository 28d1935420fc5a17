"""pygfmc_b200 -- Green's-function Monte Carlo on NVIDIA B200 (sm_100a).

A drop-in for the hot path of PyGFMC: ``run(walkers, n_steps, hamiltonian,
step_size, guide, p_array, *, method, rng_key, lam, warmup_steps, ...)`` with
PyGFMC's SpinHalf / BoseHubbard Hamiltonians and Jastrow guides, executed by
hand-written CUDA kernels behind a C ABI (``include/gfmc_b200.h``).
"""
from . import diagnostics, hamiltonian, learn, protocols, random, walkers, wavefunction
from .diagnostics import statistics
from .engine import GFMCEngine, run, run_gfmc
from .estimators import evaluate_observables
from .hamiltonian import BoseHubbard, SpinHalf, chain, exact_diagonalization, kagome, square
from .protocols import DiagonalOperator, Guide, Operator
from .random import PRNGKey
from .walkers import (Walker, prepare_walkers_from_configs, prepare_walkers_occupations,
                      prepare_walkers_random, prepare_walkers_sz)
from .wavefunction import (ExactGroundState, JastrowBoseHubbard, JastrowSpinHalf, MLPBoseHubbard,
                           RBMSpinHalf)

__version__ = "0.1.0"

__all__ = ["run", "run_gfmc", "statistics", "GFMCEngine", "evaluate_observables", "SpinHalf", "BoseHubbard",
           "chain", "square", "kagome", "PRNGKey", "Walker", "prepare_walkers_random",
           "prepare_walkers_sz", "prepare_walkers_from_configs", "prepare_walkers_occupations",
           "JastrowSpinHalf", "JastrowBoseHubbard", "RBMSpinHalf", "MLPBoseHubbard", "ExactGroundState",
           "exact_diagonalization", "Operator", "DiagonalOperator", "Guide", "hamiltonian", "protocols",
           "random", "walkers",
           "wavefunction", "__version__"]
