"""Adjoint of one Krylov time step (reference emu_sv/time_evolution/torch.py:223-378).

``step_adjoint`` is the body of ``DifferentiableStateVectorEvolution.backward``: the
parameter gradients come from one ``emusv_adjoint_step`` call (the double-Krylov
Frechet derivative of exp(-i dt H) along |state><grad| and its contraction with the
derivative operators dH/dOmega, dH/ddelta, dH/dphi, dH/dU, all on the GPU), and the state
gradient exp(+i dt H) grad is a fused Krylov step with -dt (torch.py:355-366).
"""

from __future__ import annotations

import dataclasses

import numpy as np
import torch

from . import _lib
from .hamiltonian import RydbergHamiltonian
from .krylov import HamiltonianExpOperator, fused_step

MAX_ADJOINT_QUBITS = 20  # register accumulators of the contraction kernel


@dataclasses.dataclass
class _AdjCache:
    buf: torch.Tensor | None = None
    capacity: int = 0


_caches: dict = {}


def release_workspaces() -> None:
    _caches.clear()


def _grads_to(like: torch.Tensor, g: np.ndarray) -> torch.Tensor:
    """zeros_like(param) filled with g (torch.py:325,333,340,347)."""
    return torch.from_numpy(g).to(dtype=like.dtype, device=like.device).reshape(like.shape)


def parameter_gradients(ham: RydbergHamiltonian, dt: float, state: torch.Tensor,
                        grad_state_out: torch.Tensor, tolerance: float, max_krylov_dim: int,
                        needs=(True, True, True, True)):
    """(dL/dOmega, dL/ddelta, dL/dphi, dL/dU) as float64 numpy arrays (None where not
    needed) for psi_out = exp(-i dt H) state and dL/dpsi_out = grad_state_out."""
    state = _lib.require_cuda_vector(state, "state")
    grad = _lib.require_cuda_vector(grad_state_out, "grad_state_out")
    n = _lib.nqubits_of(state)
    if n > MAX_ADJOINT_QUBITS:
        raise ValueError(f"the adjoint step supports up to {MAX_ADJOINT_QUBITS} qubits, got {n}")
    if grad.dtype != state.dtype or grad.shape != state.shape:
        raise ValueError("grad_state_out must match the state's shape and dtype")
    code = _lib.dtype_code(state.dtype)
    L = _lib.load()
    outs = [np.zeros(n) if needs[0] else None, np.zeros(n) if needs[1] else None,
            np.zeros(n) if needs[2] else None, np.zeros((n, n)) if needs[3] else None]
    ptrs = [o.ctypes.data if o is not None else None for o in outs]
    key = (state.device.index, n, code)
    c = _caches.setdefault(key, _AdjCache())
    if c.buf is None:
        c.capacity = min(max_krylov_dim + 1, 32)
    while True:
        need = L.emusv_adjoint_workspace_bytes(n, code, c.capacity)
        if need == 0:
            raise ValueError("adjoint step: unsupported register or precision")
        if c.buf is None or c.buf.numel() < need:
            c.buf = None
            c.buf = torch.empty(need, dtype=torch.uint8, device=state.device)
        st = L.emusv_adjoint_step(n, code, float(dt), *ham._params(), state.data_ptr(),
                                  grad.data_ptr(), float(tolerance), int(max_krylov_dim),
                                  *ptrs, c.buf.data_ptr(), c.buf.numel(),
                                  _lib.stream_of(state))
        if st == _lib.WORKSPACE_TOO_SMALL and c.capacity < max_krylov_dim + 1:
            c.capacity = min(2 * c.capacity, max_krylov_dim + 1)
            continue
        break
    if st == _lib.NOT_CONVERGED:  # double_krylov.py:107-110
        raise RecursionError(
            "Lanczos iteration did not converge to precision in allotted number of steps.")
    _lib.check(st, "adjoint step")
    return outs


def state_gradient(ham: RydbergHamiltonian, dt: float, grad_state_out: torch.Tensor,
                   tolerance: float, max_krylov_dim: int) -> torch.Tensor:
    """exp(+i dt H) grad_state_out (torch.py:355-366)."""
    out, _info, st = fused_step(HamiltonianExpOperator(ham, -float(dt)),
                                grad_state_out.detach(), tolerance, tolerance, max_krylov_dim)
    if st == _lib.NOT_CONVERGED:  # krylov_exp.py:126-129
        raise RecursionError("exponentiation algorithm did not converge to precision in "
                             "allotted number of steps.")
    return out


def step_adjoint(dt, omegas, deltas, phis, interaction_matrix, state, grad_state_out, tolerance,
                 max_krylov_dim, needs):
    """Gradients (omegas, deltas, phis, interaction_matrix, state) of one step, None where
    ``needs`` (ctx.needs_input_grad[1:6]) is false -- torch.py:300-378."""
    ham = RydbergHamiltonian(omegas=omegas, deltas=deltas, phis=phis,
                             interaction_matrix=interaction_matrix, device=state.device)
    g_om = g_de = g_ph = g_U = g_state = None
    if any(needs[:4]):
        om, de, ph, U = parameter_gradients(ham, dt, state, grad_state_out, tolerance,
                                            max_krylov_dim, needs[:4])
        g_om = _grads_to(omegas, om) if om is not None else None
        g_de = _grads_to(deltas, de) if de is not None else None
        g_ph = _grads_to(phis, ph) if ph is not None else None
        g_U = _grads_to(interaction_matrix, U) if U is not None else None
    if needs[4]:
        g_state = state_gradient(ham, dt, grad_state_out, tolerance, max_krylov_dim)
    return g_om, g_de, g_ph, g_U, g_state
