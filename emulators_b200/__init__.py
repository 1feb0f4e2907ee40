"""emulators_b200 -- B200-native (sm_100a) emu-sv time-evolution hot path.

Drop-in replacements for the emu-sv state-vector stepper chain of Pasqal's
``emulators`` package: ``RydbergHamiltonian`` (fused H*psi), ``krylov_exp`` (Lanczos
exponential with the Expokit error estimate, on the GPU), the time steppers with a
hand-written adjoint, and the occupation / correlation / energy observables.  All
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
from .time_evolution import BaseStepper, DifferentiableStateVectorEvolution, EvolveStateVector

__version__ = "0.1.0"

__all__ = [
    "RydbergHamiltonian", "StateVector", "inner", "krylov_exp", "krylov_exp_impl",
    "HamiltonianExpOperator", "DEFAULT_MAX_KRYLOV_DIM", "BaseStepper", "EvolveStateVector",
    "DifferentiableStateVectorEvolution", "qubit_occupation_sv_impl",
    "correlation_matrix_sv_impl", "energy_sv_impl", "energy_variance_sv_impl",
    "energy_second_moment_sv_impl", "__version__",
]
