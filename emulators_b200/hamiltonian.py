"""Matrix-free Rydberg Hamiltonian, the drop-in for ``emu_sv.hamiltonian.RydbergHamiltonian``
(reference emu_sv/hamiltonian.py:5-172).

    H = sum_j Omega_j/2 [cos(phi_j) X_j + sin(phi_j) Y_j] - sum_j delta_j n_j
        + sum_{i<j} U_ij n_i n_j

Same constructor, attributes and methods as the reference, including the noise term
-0.5i sum_j L_j^dag L_j (``noise``, the Monte Carlo stepper's non-Hermitian part).
``H * psi`` runs the fused sm_100a kernel (diagonal rebuilt on chip, all flip terms in one
pass) on the tensor's CUDA stream; ``diag`` is built on demand (the kernels never read it).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .state_vector import StateVector


class RydbergHamiltonian:
    """Attributes mirror the reference: ``nqubits``, ``omegas`` (already halved,
    hamiltonian.py:52), ``deltas``, ``phis``, ``interaction_matrix``, ``device``,
    ``noise``, ``complex`` (hamiltonian.py:61) and ``diag``."""

    def __init__(self, omegas: torch.Tensor, deltas: torch.Tensor, phis: torch.Tensor,
                 interaction_matrix: torch.Tensor, device: torch.device | str,
                 noise: torch.Tensor | None = None):
        self.nqubits: int = len(omegas)
        if not 1 <= self.nqubits <= _lib.MAX_QUBITS:
            raise ValueError(f"1..{_lib.MAX_QUBITS} qubits supported, got {self.nqubits}")
        self.omegas = omegas / 2.0
        self.deltas = deltas
        self.phis = phis
        self.interaction_matrix = interaction_matrix
        self.device = torch.device(device)
        self.noise = noise
        n = self.nqubits
        # host float64 copies passed by pointer to every kernel launch
        self._om = _lib.host_f64(omegas, n, "omegas")
        self._de = _lib.host_f64(deltas, n, "deltas")
        self._ph = _lib.host_f64(phis, n, "phis")
        U = _lib.host_f64(interaction_matrix, n * n, "interaction_matrix")
        self._U = U.reshape(n, n).copy()
        self._nz = None
        if noise is not None:  # -0.5i sum L^dag L, 2x2 (hamiltonian.py:61-67)
            nz = torch.as_tensor(noise).detach().to("cpu", torch.complex128)
            if tuple(nz.shape) != (2, 2):
                raise ValueError("noise must be a 2x2 matrix")
            self._nz = np.ascontiguousarray(torch.view_as_real(nz).numpy().reshape(-1))
        self.complex = bool((self._ph != 0.0).any()) or noise is not None
        self._diag: torch.Tensor | None = None

    # -- kernel argument tuple --------------------------------------------------------
    def _params(self):
        return (_lib.ptr(self._om), _lib.ptr(self._de), _lib.ptr(self._ph), _lib.ptr(self._U))

    def _noise_ptr(self):
        return None if self._nz is None else _lib.ptr(self._nz)

    @property
    def diag(self) -> torch.Tensor:
        """-sum_j delta_j n_j + sum_{i<j} U_ij n_i n_j (+ the noise diagonal) as
        complex128 [2^N] (hamiltonian.py:139-162), computed on the GPU."""
        if self._diag is None:
            d = torch.empty(1 << self.nqubits, dtype=torch.float64, device=self.device)
            _lib.check(_lib.load().emusv_hamiltonian_diag(
                self.nqubits, _lib.ptr(self._de), _lib.ptr(self._U), d.data_ptr(),
                _lib.stream_of(d)), "hamiltonian diag")
            d = d.to(torch.complex128)
            if self._nz is not None:  # noise diagonal per qubit (hamiltonian.py:147-151)
                n00 = complex(self._nz[0], self._nz[1])
                n11 = complex(self._nz[6], self._nz[7])
                x = torch.arange(1 << self.nqubits, device=self.device)
                pop = torch.zeros_like(x)
                for p in range(self.nqubits):
                    pop += (x >> p) & 1
                d += self.nqubits * n00 + pop.to(torch.complex128) * (n11 - n00)
            self._diag = d
        return self._diag

    def __mul__(self, vec: torch.Tensor) -> torch.Tensor:
        """H * |psi> (hamiltonian.py:69-91), one fused kernel."""
        vec = _lib.require_cuda_vector(vec, "state")
        if _lib.nqubits_of(vec) != self.nqubits:
            raise ValueError(f"state has {_lib.nqubits_of(vec)} qubits, Hamiltonian {self.nqubits}")
        out = torch.empty_like(vec)
        if self._nz is not None:
            _lib.check(_lib.load().emusv_hpsi_noisy(
                self.nqubits, _lib.dtype_code(vec.dtype), *self._params(), self._noise_ptr(),
                vec.data_ptr(), out.data_ptr(), _lib.stream_of(vec)), "H*psi")
            return out
        _lib.check(_lib.load().emusv_hpsi(
            self.nqubits, _lib.dtype_code(vec.dtype), *self._params(), vec.data_ptr(),
            out.data_ptr(), _lib.stream_of(vec)), "H*psi")
        return out

    def _moments(self, vec: torch.Tensor) -> torch.Tensor:
        """[Re<v|H|v>, Im<v|H|v>, <Hv|Hv>] as a float64 device tensor (one pass)."""
        vec = _lib.require_cuda_vector(vec, "state")
        res = torch.empty(3, dtype=torch.float64, device=vec.device)
        L = _lib.load()
        nb = L.emusv_scratch_bytes(self.nqubits, _lib.dtype_code(vec.dtype))
        sc = _lib.scratch(vec.device, nb)
        _lib.check(L.emusv_expect(self.nqubits, _lib.dtype_code(vec.dtype), *self._params(),
                                  vec.data_ptr(), res.data_ptr(), sc.data_ptr(), sc.numel(),
                                  _lib.stream_of(vec)), "energy")
        return res

    def expect(self, state: StateVector) -> torch.Tensor:
        """Re <psi|H|psi> (hamiltonian.py:164-172)."""
        assert isinstance(state, StateVector), \
            "Currently, only expectation values of StateVectors are supported"
        if self._nz is not None:  # Re <psi|H psi> with the noise term, no Hermiticity check
            v = _lib.require_cuda_vector(state.data, "state")
            hv = self * v
            res = torch.empty(2, dtype=torch.float64, device=v.device)
            L = _lib.load()
            sc = _lib.scratch(v.device, L.emusv_scratch_bytes(1, 0))
            _lib.check(L.emusv_vec_dot(v.numel(), _lib.dtype_code(v.dtype), v.data_ptr(),
                                       hv.data_ptr(), res.data_ptr(), sc.data_ptr(), sc.numel(),
                                       _lib.stream_of(v)), "energy")
            return res[0]
        m = self._moments(state.data)
        # H is Hermitian: the imaginary part is rounding only.  complex128 keeps the
        # reference's absolute bound (hamiltonian.py:170-171); complex64 storage rounds
        # H psi at ~6e-8 relative, so its bound scales with ||H psi||.
        atol = 1e-8 if state.data.dtype == torch.complex128 else 1e-8 + 1e-6 * float(m[2].sqrt())
        assert abs(float(m[1])) <= atol, f"imaginary energy {float(m[1])}"
        return m[0]

    def second_moment(self, state: StateVector) -> torch.Tensor:
        """<psi|H^2|psi> = <H psi|H psi> (custom_callback_implementations.py:170-185); the
        noise term is left out, as the reference's _strip_noise does (19-27)."""
        return self._moments(state.data)[2]

    def variance(self, state: StateVector) -> torch.Tensor:
        """<H^2> - <H>^2 without the noise term (custom_callback_implementations.py:131-147)."""
        m = self._moments(state.data)
        return m[2] - m[0] ** 2
