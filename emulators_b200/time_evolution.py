"""Time steppers, the drop-in for ``emu_sv.time_evolution`` (reference
emu_sv/time_evolution/interface.py:7-37, implementations.py:16-60, torch.py:122-378).

``DifferentiableStateVectorEvolution`` keeps the reference's autograd.Function contract:
forward = exp(-i dt H) psi through the fused GPU Krylov step; backward = the adjoint
(gradients for Omega, delta, phi, U and the input state) computed by
:mod:`emulators_b200.adjoint`.  ``EvolveMonteCarlo`` (implementations.py:123-250) evolves
under the noisy non-Hermitian Hamiltonian by the fused GPU Arnoldi step and takes quantum
jumps with the reference's random draws, Brent bracketing and jump weights.
"""

from __future__ import annotations

import random
from abc import ABC, abstractmethod
from typing import Any

import numpy as np
import torch

from . import _lib
from .algebra import apply_inplace, expect_batch
from .brents_root_finding import BrentsRootFinder
from .hamiltonian import RydbergHamiltonian
from .jump_lindblad_operators import compute_noise_from_lindbladians
from .krylov import DEFAULT_MAX_KRYLOV_DIM, HamiltonianExpOperator, krylov_exp

JUMP_TIME_TOLERANCE_FRACTION = 0.1


class DifferentiableStateVectorEvolution(torch.autograd.Function):
    """One time step as a torch.autograd.Function (torch.py:122-378)."""

    @staticmethod
    def get_hamiltonian(omegas, deltas, phis, interaction_matrix, device) -> RydbergHamiltonian:
        return RydbergHamiltonian(omegas=omegas, deltas=deltas, phis=phis,
                                  interaction_matrix=interaction_matrix, device=device, noise=None)

    @staticmethod
    def evolve(dt, omegas, deltas, phis, interaction_matrix, state, krylov_tolerance,
               max_krylov_dim):
        """torch.py:143-172."""
        ham = DifferentiableStateVectorEvolution.get_hamiltonian(
            omegas, deltas, phis, interaction_matrix, state.device)
        res = krylov_exp(HamiltonianExpOperator(ham, dt), state, norm_tolerance=krylov_tolerance,
                         exp_tolerance=krylov_tolerance, is_hermitian=True,
                         max_krylov_dim=max_krylov_dim)
        return res, ham

    @staticmethod
    def forward(ctx: Any, dt, omegas, deltas, phis, interaction_matrix, state, krylov_tolerance,
                max_krylov_dim):
        """torch.py:174-219: returns (exp(-i dt H) psi, H)."""
        res, ham = DifferentiableStateVectorEvolution.evolve(
            dt, omegas, deltas, phis, interaction_matrix, state, krylov_tolerance, max_krylov_dim)
        ctx.save_for_backward(omegas, deltas, phis, interaction_matrix, state)
        ctx.dt = dt
        ctx.tolerance = krylov_tolerance
        ctx.max_krylov_dim = max_krylov_dim
        return res, ham

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx: Any, grad_state_out: torch.Tensor, gham: None):
        """torch.py:223-378: gradients via the adjoint of the Krylov step."""
        from .adjoint import step_adjoint

        omegas, deltas, phis, interaction_matrix, state = ctx.saved_tensors
        needs = tuple(ctx.needs_input_grad[1:6])
        g = step_adjoint(ctx.dt, omegas, deltas, phis, interaction_matrix, state,
                         grad_state_out, ctx.tolerance, ctx.max_krylov_dim, needs)
        return (None, *g, None, None)


class BaseStepper(ABC):
    """interface.py:7-37."""

    def __init__(self, max_krylov_dim: int) -> None:
        self.max_krylov_dim = max_krylov_dim

    @staticmethod
    @abstractmethod
    def get_hamiltonian(omegas, deltas, phis, pulser_lindblads, interaction_matrix, device):
        pass

    @abstractmethod
    def apply(self, dt, omegas, deltas, phis, full_interaction_matrix, state, krylov_tolerance,
              pulser_lindblads):
        pass


class EvolveStateVector(BaseStepper):
    """implementations.py:16-60."""

    def __init__(self, max_krylov_dim: int = DEFAULT_MAX_KRYLOV_DIM) -> None:
        super().__init__(max_krylov_dim)

    @staticmethod
    def get_hamiltonian(omegas, deltas, phis, pulser_lindblads, interaction_matrix, device):
        return DifferentiableStateVectorEvolution.get_hamiltonian(
            omegas, deltas, phis, interaction_matrix, device)

    def apply(self, dt, omegas, deltas, phis, full_interaction_matrix, state, krylov_tolerance,
              pulser_lindblads=None):
        if pulser_lindblads:
            raise NotImplementedError("emulators_b200: Lindblad noise is not implemented")
        return DifferentiableStateVectorEvolution.apply(
            dt, omegas, deltas, phis, full_interaction_matrix, state, krylov_tolerance,
            self.max_krylov_dim)


def _norm2(state: torch.Tensor) -> float:
    """||state||^2 (FP64 sum on the GPU, read back)."""
    L = _lib.load()
    res = torch.empty(2, dtype=torch.float64, device=state.device)
    sc = _lib.scratch(state.device, L.emusv_scratch_bytes(1, 0))
    _lib.check(L.emusv_vec_dot(state.numel(), _lib.dtype_code(state.dtype), state.data_ptr(),
                               state.data_ptr(), res.data_ptr(), sc.data_ptr(), sc.numel(),
                               _lib.stream_of(state)), "norm")
    return float(res[0])


class EvolveMonteCarlo(BaseStepper):
    """Monte Carlo quantum-jump stepper (implementations.py:123-250).  The random draws
    come from Python's ``random`` module in the reference's order (threshold at
    construction and after every jump, one ``random.choices`` per jump)."""

    def __init__(self, max_krylov_dim: int = DEFAULT_MAX_KRYLOV_DIM) -> None:
        super().__init__(max_krylov_dim)
        self.jump_threshold = random.uniform(0.0, 1.0)

    @staticmethod
    def get_hamiltonian(omegas, deltas, phis, pulser_lindblads, interaction_matrix, device):
        return RydbergHamiltonian(omegas=omegas, deltas=deltas, phis=phis,
                                  interaction_matrix=interaction_matrix, device=device,
                                  noise=compute_noise_from_lindbladians(pulser_lindblads))

    def evolve(self, dt, hamiltonian, state, krylov_tolerance):
        """exp(-i dt H) state by Arnoldi (implementations.py:148-166)."""
        return krylov_exp(HamiltonianExpOperator(hamiltonian, dt), state,
                          norm_tolerance=krylov_tolerance, exp_tolerance=krylov_tolerance,
                          is_hermitian=False, max_krylov_dim=self.max_krylov_dim)

    def do_quantum_jump(self, state, lindblad_ops, aggregated_lindblad_ops, n_qubits):
        """implementations.py:168-190: pick (qubit, L) with weight <L^dag L>, apply, renormalise."""
        weights = expect_batch(state, aggregated_lindblad_ops, n_qubits).real
        qubit, op = random.choices([(q, op) for q in range(n_qubits) for op in lindblad_ops],
                                   weights=weights.reshape(-1).tolist())[0]
        state = state.clone()
        apply_inplace(state, qubit, op)
        inv = 1.0 / np.sqrt(_norm2(state))
        apply_inplace(state, 0, torch.eye(2, dtype=torch.complex128) * inv)
        self.jump_threshold = random.uniform(0.0, _norm2(state))
        return state

    def apply(self, dt, omegas, deltas, phis, full_interaction_matrix, state, krylov_tolerance,
              pulser_lindblads):
        """implementations.py:192-250."""
        ham = self.get_hamiltonian(omegas, deltas, phis, pulser_lindblads, full_interaction_matrix,
                                   state.device)
        current_time = 0.0
        tol = dt * JUMP_TIME_TOLERANCE_FRACTION
        new_gap = _norm2(state) - self.jump_threshold
        stacked = torch.stack([torch.as_tensor(L).to(torch.complex128) for L in pulser_lindblads])
        aggregated = stacked.conj().transpose(1, 2) @ stacked
        while abs(dt - current_time) > 1e-5:
            old_gap = new_gap
            state = self.evolve(dt - current_time, ham, state, krylov_tolerance)
            new_gap = _norm2(state) - self.jump_threshold
            if new_gap > 0.0:
                break
            rf = BrentsRootFinder(start=current_time, end=dt, f_start=old_gap, f_end=new_gap,
                                  epsilon=tol)
            current_time = dt
            while not rf.is_converged(tolerance=tol):
                target = rf.get_next_abscissa()
                state = self.evolve(target - current_time, ham, state, krylov_tolerance)
                current_time = target
                new_gap = _norm2(state) - self.jump_threshold
                rf.provide_ordinate(current_time, new_gap)
            state = self.do_quantum_jump(state, pulser_lindblads, aggregated, len(omegas))
            new_gap = _norm2(state) - self.jump_threshold
        return state, ham


class EvolveDensityMatrix(BaseStepper):
    """Evolution of a density matrix under the Lindbladian (implementations.py:63-120):
    exp(-i dt L) rho by the fused Arnoldi step over the 4^N vector."""

    def __init__(self, max_krylov_dim: int = DEFAULT_MAX_KRYLOV_DIM) -> None:
        super().__init__(max_krylov_dim)

    @staticmethod
    def get_hamiltonian(omegas, deltas, phis, pulser_lindblads, interaction_matrix, device):
        from .density_matrix import RydbergLindbladian

        return RydbergLindbladian(omegas=omegas, deltas=deltas, phis=phis,
                                  pulser_lindblads=pulser_lindblads,
                                  interaction_matrix=interaction_matrix, device=device)

    def apply(self, dt, omegas, deltas, phis, full_interaction_matrix, state, krylov_tolerance,
              pulser_lindblads):
        from .krylov import fused_lindblad_step

        ham = self.get_hamiltonian(omegas, deltas, phis, pulser_lindblads, full_interaction_matrix,
                                   state.device)
        out, info, st = fused_lindblad_step(ham, dt, state, krylov_tolerance, krylov_tolerance,
                                            self.max_krylov_dim)
        if st != _lib.OK:
            raise RecursionError("exponentiation algorithm did not converge to precision in "
                                 "allotted number of steps.")
        return out, ham
