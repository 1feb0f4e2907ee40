"""emulators_b200 -- B200-native (sm_100a) emu-sv time-evolution hot path.

Drop-in replacements for the emu-sv state-vector stepper chain of Pasqal's
``emulators`` package: ``RydbergHamiltonian`` (fused H*psi), ``krylov_exp`` (Lanczos
exponential with the Expokit error estimate, on the GPU), the time steppers with a
hand-written adjoint, the Monte Carlo quantum-jump stepper (noisy Hamiltonian, Arnoldi
exponential), and the occupation / correlation / energy observables.  All
compute runs in ``libemusv_b200.so`` (CUDA, sm_100a); there is no CPU path.
"""

from .hamiltonian import RydbergHamiltonian
from .krylov import DEFAULT_MAX_KRYLOV_DIM, HamiltonianExpOperator, krylov_exp, krylov_exp_impl
from .observables import (
    correlation_matrix_sv_impl,
    energy_second_moment_sv_impl,
    energy_sv_impl,
    energy_variance_sv_impl,
    qubit_occupation_sv_impl,
)
from .state_vector import StateVector, inner
from .algebra import apply, expect_batch
from .brents_root_finding import BrentsRootFinder, find_root_brents
from .jump_lindblad_operators import compute_noise_from_lindbladians, get_lindblad_operators
from .time_evolution import (
    BaseStepper,
    DifferentiableStateVectorEvolution,
    EvolveMonteCarlo,
    EvolveStateVector,
)

__version__ = "0.1.0"

__all__ = [
    "RydbergHamiltonian", "StateVector", "inner", "krylov_exp", "krylov_exp_impl",
    "HamiltonianExpOperator", "DEFAULT_MAX_KRYLOV_DIM", "BaseStepper", "EvolveStateVector",
    "DifferentiableStateVectorEvolution", "qubit_occupation_sv_impl",
    "correlation_matrix_sv_impl", "energy_sv_impl", "energy_variance_sv_impl",
    "energy_second_moment_sv_impl", "EvolveMonteCarlo", "expect_batch", "apply",
    "BrentsRootFinder", "find_root_brents", "compute_noise_from_lindbladians",
    "get_lindblad_operators", "__version__",
]
