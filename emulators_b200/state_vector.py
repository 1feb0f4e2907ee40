"""State vector container, the drop-in for ``emu_sv.state_vector.StateVector``
(reference emu_sv/state_vector.py:17-210, emu_sv/dense_state.py:17-140).

A 1-D complex tensor of length 2^N on the GPU; qubit 0 is the most significant bit of
the index and bit value 1 is the Rydberg state |r> (eigenstates ("r", "g")).  Unlike
the reference, ``complex64`` storage is allowed (the precision form), and CPU storage
is refused: this package has no CPU path.
"""

from __future__ import annotations

import math
from collections import Counter
from typing import Sequence

import torch

from . import _lib

dtype = torch.complex128


def _device(gpu: bool) -> torch.device:
    if not gpu:
        raise RuntimeError("emulators_b200 keeps states on the GPU (gpu=False is not supported)")
    if not torch.cuda.is_available():
        raise RuntimeError("emulators_b200 needs a CUDA device")
    return torch.device("cuda", torch.cuda.current_device())


class StateVector:
    def __init__(self, data: torch.Tensor, *, gpu: bool = True,
                 eigenstates: Sequence[str] = ("r", "g")):
        assert data.dim() == 1
        self.eigenstates = tuple(eigenstates)
        tgt = data.dtype if data.dtype in (torch.complex128, torch.complex64) else dtype
        self.data = data.to(dtype=tgt, device=_device(gpu))

    @property
    def n_qudits(self) -> int:
        return int(math.log2(self.data.shape[0]))

    @classmethod
    def zero(cls, num_sites: int, gpu: bool = True, eigenstates=("r", "g"),
             dtype: torch.dtype = dtype) -> "StateVector":
        return cls(torch.zeros(2**num_sites, dtype=dtype, device=_device(gpu)), gpu=gpu,
                   eigenstates=eigenstates)

    @classmethod
    def make(cls, num_sites: int, gpu: bool = True, dtype: torch.dtype = dtype) -> "StateVector":
        """|00..0> (state_vector.py:81-105)."""
        r = cls.zero(num_sites, gpu=gpu, dtype=dtype)
        r.data[0] = 1.0
        return r

    def norm(self) -> torch.Tensor:
        """||psi|| on the CPU (state_vector.py:157-164)."""
        return torch.linalg.vector_norm(self.data.to(torch.complex128)).cpu()

    def inner(self, other: "StateVector") -> torch.Tensor:
        assert isinstance(other, StateVector), "Other state must be a StateVector"
        assert self.data.shape == other.data.shape, "States do not have the same shape"
        return torch.vdot(self.data.to(torch.complex128),
                          other.data.to(self.data.device, torch.complex128)).cpu()

    def _normalize(self) -> None:
        norm = torch.linalg.vector_norm(self.data)
        if abs(self.norm() ** 4 - 1.0) > 1e-12:
            self.data = self.data / norm

    def __add__(self, other: "StateVector") -> "StateVector":
        assert isinstance(other, StateVector), "`Other` state can only be a StateVector"
        return StateVector(self.data + other.data, eigenstates=self.eigenstates)

    def __rmul__(self, scalar: complex) -> "StateVector":
        return StateVector(scalar * self.data, eigenstates=self.eigenstates)

    def sample(self, num_shots: int = 1000) -> Counter:
        """Bitstring counts drawn from |psi|^2 (dense_state.py:40-95) by inverting the
        cumulative distribution on the GPU (emusv_sample; the reference's path for
        registers above 2^24 amplitudes, emu_sv/utils.py:17-49, used here at every size)."""
        psi = _lib.require_cuda_vector(self.data, "state")
        n = _lib.nqubits_of(psi)
        u = torch.rand(num_shots, dtype=torch.float64, device=psi.device)
        idx = sample_indices(psi, u)
        return Counter(format(i, f"0{n}b") for i in idx.tolist())

    def __repr__(self) -> str:
        return repr(self.data)


def inner(left: StateVector, right: StateVector) -> torch.Tensor:
    return left.inner(right)


def sample_indices(psi: torch.Tensor, uniforms: torch.Tensor) -> torch.Tensor:
    """Indices drawn from |psi|^2 for the given uniforms in [0, 1): the first index whose
    cumulative probability exceeds u * total (emu_sv/utils.py:40-49), on the GPU."""
    psi = _lib.require_cuda_vector(psi, "state")
    n = _lib.nqubits_of(psi)
    u = uniforms.to(device=psi.device, dtype=torch.float64).contiguous()
    out = torch.empty(u.numel(), dtype=torch.int64, device=psi.device)
    L = _lib.load()
    sc = _lib.scratch(psi.device, L.emusv_sample_scratch_bytes(n))
    st = L.emusv_sample(n, _lib.dtype_code(psi.dtype), psi.data_ptr(), u.numel(), u.data_ptr(),
                        out.data_ptr(), sc.data_ptr(), sc.numel(), _lib.stream_of(psi))
    if st == _lib.NONFINITE:  # torch.multinomial's exception and message
        raise RuntimeError("invalid multinomial distribution (sum of probabilities <= 0)")
    _lib.check(st, "sample")
    return out
