"""Single-qubit algebra on state vectors, the drop-in for ``emu_sv.algebra``
(reference emu_sv/algebra.py:1-37), on the GPU.

``expect_batch`` reduces the state once to its single-qubit density matrices
(``emusv_qubit_densities``) and takes the traces with the operators on the host (n x K
2x2 traces); ``apply`` runs ``emusv_apply_1q`` in place on a copy.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib


def qubit_densities(state_vector: torch.Tensor) -> torch.Tensor:
    """[n, 2, 2] complex128 single-qubit reduced density matrices (unnormalised state)."""
    v = _lib.require_cuda_vector(state_vector, "state")
    n = _lib.nqubits_of(v)
    L = _lib.load()
    rho = torch.empty(n * 8, dtype=torch.float64, device=v.device)
    sc = _lib.scratch(v.device, L.emusv_qubit_densities_scratch_bytes(n))
    _lib.check(L.emusv_qubit_densities(n, _lib.dtype_code(v.dtype), v.data_ptr(), rho.data_ptr(),
                                       sc.data_ptr(), sc.numel(), _lib.stream_of(v)),
               "qubit densities")
    return torch.view_as_complex(rho.view(n, 2, 2, 2))


def expect_batch(state_vector: torch.Tensor, single_qubit_operators: torch.Tensor,
                 n_qubits: int) -> torch.Tensor:
    """T[q, i] = <psi| op_i on qubit q |psi> (algebra.py:4-25): Tr(op_i rho_q)."""
    rho = qubit_densities(state_vector)
    if rho.shape[0] != n_qubits:
        raise ValueError(f"state has {rho.shape[0]} qubits, expected {n_qubits}")
    ops = torch.as_tensor(single_qubit_operators).to(rho.device, torch.complex128)
    # Tr(O rho) = sum_ab O[a][b] rho[b][a]
    return torch.einsum("iab,qba->qi", ops, rho)


def _op8(op) -> np.ndarray:
    o = torch.as_tensor(op).detach().to("cpu", torch.complex128)
    if tuple(o.shape) != (2, 2):
        raise ValueError("single-qubit operator must be 2x2")
    return np.ascontiguousarray(torch.view_as_real(o).numpy().reshape(-1))


def apply_inplace(state_vector: torch.Tensor, qubit_index: int, single_qubit_operator) -> None:
    v = _lib.require_cuda_vector(state_vector, "state")
    n = _lib.nqubits_of(v)
    op = _op8(single_qubit_operator)
    _lib.check(_lib.load().emusv_apply_1q(n, _lib.dtype_code(v.dtype), v.data_ptr(), int(qubit_index),
                                          _lib.ptr(op), _lib.stream_of(v)), "apply")


def apply(state_vector: torch.Tensor, qubit_index: int, single_qubit_operator) -> torch.Tensor:
    """single_qubit_operator applied to qubit ``qubit_index`` (algebra.py:28-37)."""
    out = _lib.require_cuda_vector(state_vector, "state").clone()
    apply_inplace(out, qubit_index, single_qubit_operator)
    return out
