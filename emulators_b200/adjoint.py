"""Adjoint of one Krylov time step (reference emu_sv/time_evolution/torch.py:223-378)."""

from __future__ import annotations


def step_adjoint(dt, omegas, deltas, phis, interaction_matrix, state, grad_state_out, tolerance,
                 max_krylov_dim, needs):
    raise NotImplementedError("emulators_b200: the adjoint step is not built yet")
