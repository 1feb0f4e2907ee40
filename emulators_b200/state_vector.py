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
        """Bitstring counts drawn from |psi|^2 (dense_state.py:40-95)."""
        p = (self.data.real.double() ** 2 + self.data.imag.double() ** 2)
        if p.numel() <= 2**24:
            idx = torch.multinomial(p, num_shots, replacement=True)
        else:
            cdf = torch.cumsum(p, 0)
            cdf /= cdf[-1].clone()
            idx = torch.searchsorted(cdf, torch.rand(num_shots, dtype=torch.float64,
                                                     device=cdf.device), right=True)
            idx.clamp_(max=p.numel() - 1)
        n = self.n_qudits
        return Counter(format(i, f"0{n}b") for i in idx.tolist())

    def __repr__(self) -> str:
        return repr(self.data)


def inner(left: StateVector, right: StateVector) -> torch.Tensor:
    return left.inner(right)
