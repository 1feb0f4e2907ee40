"""State-vector observables, the drop-ins for emu_sv/custom_callback_implementations.py.

Each is one pass over the state on the GPU with FP64 accumulation; results come back
as float64 CPU tensors like the reference's (``.cpu()`` at the end of each function).
"""

from __future__ import annotations

import torch

from . import _lib
from .hamiltonian import RydbergHamiltonian
from .state_vector import StateVector


def occupation(psi: torch.Tensor) -> torch.Tensor:
    """<n_i> for every qubit, float64 on the device (one pass, no host sync)."""
    psi = _lib.require_cuda_vector(psi, "state")
    n = _lib.nqubits_of(psi)
    out = torch.empty(n, dtype=torch.float64, device=psi.device)
    L = _lib.load()
    sc = _lib.scratch(psi.device, L.emusv_scratch_bytes(n, _lib.dtype_code(psi.dtype)))
    _lib.check(L.emusv_occupation(n, _lib.dtype_code(psi.dtype), psi.data_ptr(), out.data_ptr(),
                                  sc.data_ptr(), sc.numel(), _lib.stream_of(psi)), "occupation")
    return out


def correlation(psi: torch.Tensor) -> torch.Tensor:
    """<n_i n_j>, float64 [N, N] on the device."""
    psi = _lib.require_cuda_vector(psi, "state")
    n = _lib.nqubits_of(psi)
    out = torch.empty(n, n, dtype=torch.float64, device=psi.device)
    L = _lib.load()
    sc = _lib.scratch(psi.device, L.emusv_scratch_bytes(n, _lib.dtype_code(psi.dtype)))
    _lib.check(L.emusv_correlation(n, _lib.dtype_code(psi.dtype), psi.data_ptr(), out.data_ptr(),
                                   sc.data_ptr(), sc.numel(), _lib.stream_of(psi)), "correlation")
    return out


def qubit_occupation_sv_impl(self=None, *, config=None, state: StateVector,
                             hamiltonian=None) -> torch.Tensor:
    """custom_callback_implementations.py:30-47."""
    return occupation(state.data).cpu()


def correlation_matrix_sv_impl(self=None, *, config=None, state: StateVector,
                               hamiltonian=None) -> torch.Tensor:
    """custom_callback_implementations.py:77-102."""
    return correlation(state.data).cpu()


def energy_sv_impl(self=None, *, config=None, state: StateVector,
                   hamiltonian: RydbergHamiltonian) -> torch.Tensor:
    """pulser Energy -> RydbergHamiltonian.expect (hamiltonian.py:164-172)."""
    return hamiltonian.expect(state).cpu()


def energy_variance_sv_impl(self=None, *, config=None, state: StateVector,
                            hamiltonian: RydbergHamiltonian) -> torch.Tensor:
    """custom_callback_implementations.py:131-147 (one fused pass)."""
    return hamiltonian.variance(state).cpu()


def energy_second_moment_sv_impl(self=None, *, config=None, state: StateVector,
                                 hamiltonian: RydbergHamiltonian) -> torch.Tensor:
    """custom_callback_implementations.py:170-185 (one fused pass)."""
    return hamiltonian.second_moment(state).cpu()
