"""Time steppers, the drop-in for ``emu_sv.time_evolution`` (reference
emu_sv/time_evolution/interface.py:7-37, implementations.py:16-60, torch.py:122-378).

``DifferentiableStateVectorEvolution`` keeps the reference's autograd.Function contract:
forward = exp(-i dt H) psi through the fused GPU Krylov step; backward = the adjoint
(gradients for Omega, delta, phi, U and the input state) computed by
:mod:`emulators_b200.adjoint`.
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from typing import Any

import torch

from .hamiltonian import RydbergHamiltonian
from .krylov import DEFAULT_MAX_KRYLOV_DIM, HamiltonianExpOperator, krylov_exp


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
