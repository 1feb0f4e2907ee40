"""Density matrices and the Lindbladian, the drop-ins for ``emu_sv.density_matrix_state.
DensityMatrix`` (reference emu_sv/density_matrix_state.py:14-120) and
``emu_sv.lindblad_operator.RydbergLindbladian`` (emu_sv/lindblad_operator.py:11-218), with
the density-matrix observables of emu_sv/custom_callback_implementations.py:50-200.

A density matrix is a 2^N x 2^N complex tensor on the GPU (row-major, as the reference
stores it).  ``RydbergLindbladian @ rho`` runs ``emusv_lindblad_apply``: the Lindbladian as
one 2N-bit operator (the H*psi kernels on the row and column indices plus the jump kernel).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .state_vector import StateVector

dtype = torch.complex128


class DensityMatrix:
    """density_matrix_state.py:14-120 (GPU only)."""

    def __init__(self, data: torch.Tensor, gpu: bool = True, eigenstates=("r", "g")):
        if gpu is False:
            raise ValueError("emulators_b200 runs on the GPU only (gpu=False is not supported)")
        data = torch.as_tensor(data)
        if data.ndim != 2 or data.shape[0] != data.shape[1] or data.shape[0] & (data.shape[0] - 1):
            raise ValueError("a density matrix is a square 2^N x 2^N tensor")
        if not data.is_cuda:
            data = data.to("cuda")
        self.data = data
        self.eigenstates = eigenstates

    @property
    def n_qudits(self) -> int:
        return int(self.data.shape[0]).bit_length() - 1

    @classmethod
    def make(cls, n_atoms: int, gpu: bool = True) -> "DensityMatrix":
        """|0...0><0...0| (density_matrix_state.py:33-38)."""
        r = torch.zeros(2 ** n_atoms, 2 ** n_atoms, dtype=dtype, device="cuda")
        r[0, 0] = 1.0
        return cls(r, gpu=gpu)

    @classmethod
    def from_state_vector(cls, state: StateVector) -> "DensityMatrix":
        """|psi><psi| (density_matrix_state.py:62-89)."""
        v = state.data.reshape(-1)
        return cls(torch.outer(v, v.conj()))

    def __add__(self, other):
        raise NotImplementedError("Not implemented")

    def __rmul__(self, scalar: complex) -> "DensityMatrix":
        return DensityMatrix(self.data * scalar)

    def norm(self) -> torch.Tensor:
        """Tr(rho) (density_matrix_state.py:52-60), float64 on the host."""
        return diagonal_probabilities(self.data).sum().cpu()

    def _normalize(self) -> None:
        tr = self.norm()
        if not torch.allclose(tr, torch.tensor(1.0, dtype=torch.float64)):
            self.data = self.data / tr.item()


def _ops8(ops) -> np.ndarray:
    out = [torch.view_as_real(torch.as_tensor(L).detach().to("cpu", torch.complex128)).numpy().reshape(-1)
           for L in ops]
    for L in ops:
        if tuple(torch.as_tensor(L).shape) != (2, 2):
            raise ValueError("the Lindbladian takes single-qubit (2 x 2) jump operators")
    return np.ascontiguousarray(np.concatenate(out) if out else np.zeros(8))


def diagonal_amplitudes(rho: torch.Tensor) -> torch.Tensor:
    """sqrt(max(Re rho_rr, 0)) as a state-vector-shaped tensor (device)."""
    n = int(rho.shape[0]).bit_length() - 1
    a = torch.empty(rho.shape[0], dtype=rho.dtype, device=rho.device)
    _lib.check(_lib.load().emusv_dm_diagonal_amplitudes(n, _lib.dtype_code(rho.dtype), rho.data_ptr(),
                                                        a.data_ptr(), _lib.stream_of(rho)), "diagonal")
    return a


def diagonal_probabilities(rho: torch.Tensor) -> torch.Tensor:
    a = diagonal_amplitudes(rho)
    return a.real.to(torch.float64) ** 2


class RydbergLindbladian:
    """lindblad_operator.py:11-218: ``L @ rho`` = Heff rho - (Heff rho)^dag
    + i sum_kq L_kq rho L_kq^dag for Hermitian rho; ``expect`` = Tr(H rho)."""

    def __init__(self, omegas, deltas, phis, pulser_lindblads, interaction_matrix, device):
        self.nqubits = len(omegas)
        if not 1 <= self.nqubits <= _lib.MAX_QUBITS // 2:
            raise ValueError(f"1..{_lib.MAX_QUBITS // 2} qubits supported, got {self.nqubits}")
        self.omegas = omegas / 2.0
        self.deltas = deltas
        self.phis = phis
        self.interaction_matrix = interaction_matrix
        self.pulser_lindblads = list(pulser_lindblads)
        self.device = torch.device(device)
        n = self.nqubits
        self._om = _lib.host_f64(omegas, n, "omegas")
        self._de = _lib.host_f64(deltas, n, "deltas")
        self._ph = _lib.host_f64(phis, n, "phis")
        self._U = _lib.host_f64(interaction_matrix, n * n, "interaction_matrix").reshape(n, n).copy()
        self._ops = _ops8(self.pulser_lindblads)
        self.complex = bool((self._ph != 0.0).any())

    def _params(self):
        return (_lib.ptr(self._om), _lib.ptr(self._de), _lib.ptr(self._ph), _lib.ptr(self._U))

    def _check(self, rho: torch.Tensor) -> torch.Tensor:
        if not rho.is_cuda:
            raise RuntimeError("density matrix must be a CUDA tensor")
        if tuple(rho.shape) != (1 << self.nqubits, 1 << self.nqubits):
            raise ValueError("density matrix shape does not match the register")
        return rho.contiguous()

    def __matmul__(self, density_matrix: torch.Tensor) -> torch.Tensor:
        rho = self._check(density_matrix)
        out = torch.empty_like(rho)
        _lib.check(_lib.load().emusv_lindblad_apply(
            self.nqubits, _lib.dtype_code(rho.dtype), *self._params(), len(self.pulser_lindblads),
            _lib.ptr(self._ops), rho.data_ptr(), out.data_ptr(), _lib.stream_of(rho)), "lindbladian")
        return out

    def _moments(self, rho: torch.Tensor) -> torch.Tensor:
        rho = self._check(rho)
        L = _lib.load()
        res = torch.empty(4, dtype=torch.float64, device=rho.device)
        code = _lib.dtype_code(rho.dtype)
        sc = _lib.scratch(rho.device, L.emusv_dm_scratch_bytes(self.nqubits, code))
        _lib.check(L.emusv_dm_energy(self.nqubits, code, *self._params(), rho.data_ptr(),
                                     res.data_ptr(), sc.data_ptr(), sc.numel(), _lib.stream_of(rho)),
                   "density-matrix energy")
        return res

    def expect(self, state: DensityMatrix) -> torch.Tensor:
        """Tr(H rho) (lindblad_operator.py:213-218)."""
        m = self._moments(state.data)
        assert abs(float(m[1])) <= 1e-8 * max(1.0, abs(float(m[0]))), "imaginary energy"
        return m[0]

    def second_moment(self, state: DensityMatrix) -> torch.Tensor:
        """Tr(H^2 rho) (custom_callback_implementations.py:188-200)."""
        return self._moments(state.data)[2]

    def variance(self, state: DensityMatrix) -> torch.Tensor:
        """Tr(H^2 rho) - Tr(H rho)^2 (custom_callback_implementations.py:150-167)."""
        m = self._moments(state.data)
        return m[2] - m[0] ** 2


# ---------------------------------------------------------------- observables
def qubit_occupation_sv_den_mat_impl(self=None, *, config=None, state: DensityMatrix,
                                     hamiltonian=None) -> torch.Tensor:
    """custom_callback_implementations.py:50-74: Tr(rho n_i)."""
    from .observables import occupation

    return occupation(diagonal_amplitudes(state.data)).cpu()


def correlation_matrix_sv_den_mat_impl(self=None, *, config=None, state: DensityMatrix,
                                       hamiltonian=None) -> torch.Tensor:
    """custom_callback_implementations.py:105-128: Tr(rho n_i n_j)."""
    from .observables import correlation

    return correlation(diagonal_amplitudes(state.data)).cpu()


def energy_variance_sv_den_mat_impl(self=None, *, config=None, state: DensityMatrix,
                                    hamiltonian: RydbergLindbladian) -> torch.Tensor:
    return hamiltonian.variance(state).cpu()


def energy_second_moment_den_mat_impl(self=None, *, config=None, state: DensityMatrix,
                                      hamiltonian: RydbergLindbladian) -> torch.Tensor:
    return hamiltonian.second_moment(state).cpu()
