"""Lindblad operators of the noise model and the noise term of the Hamiltonian, the
drop-in for ``emu_base.jump_lindblad_operators`` (reference
emu_base/jump_lindblad_operators.py:1-93).  Host-side 2x2 algebra.

``get_lindblad_operators`` reads the same attributes of a pulser ``NoiseModel``
(``noise_types``, ``relaxation_rate``, ``dephasing_rate``, ``hyperfine_dephasing_rate``,
``depolarizing_rate``, ``eff_noise_rates``, ``eff_noise_opers``) from any object that has
them.
"""

from __future__ import annotations

import math

import torch

dtype = torch.complex128


def get_lindblad_operators(*, noise_type: str, noise_model, interact_type: str = "ising",
                           dim: int = 2) -> list[torch.Tensor]:
    """jump_lindblad_operators.py:8-76 (qubit order of emu-sv: |g> = 0, |r> = 1)."""
    assert noise_type in noise_model.noise_types
    if noise_type == "relaxation":  # sqrt(rate) |g><r|
        op = torch.zeros(dim, dim, dtype=dtype)
        op[0, 1] = math.sqrt(noise_model.relaxation_rate)
        return [op]
    if noise_type == "dephasing":
        if noise_model.hyperfine_dephasing_rate != 0.0:
            raise NotImplementedError(
                "hyperfine dephasing acts on the digital basis, which this emulator does not "
                "simulate (only the ground-Rydberg basis)")
        c = math.sqrt(noise_model.dephasing_rate / 2)
        return [torch.diag(torch.tensor([c, -c], dtype=dtype))]
    if noise_type == "depolarizing":  # sqrt(rate/4) X, Y, Z
        c = math.sqrt(noise_model.depolarizing_rate / 4)
        x = torch.tensor([[0, c], [c, 0]], dtype=dtype)
        y = torch.tensor([[0, -1j * c], [1j * c, 0]], dtype=dtype)
        z = torch.tensor([[c, 0], [0, -c]], dtype=dtype)
        return [x, y, z]
    if noise_type == "eff_noise":
        ops = [torch.tensor(op, dtype=dtype) for op in noise_model.eff_noise_opers]
        if not all(op.shape == (dim, dim) for op in ops):
            raise ValueError(f"effective noise operators must be {dim} x {dim} matrices")
        out = [math.sqrt(rate) * op for rate, op in zip(noise_model.eff_noise_rates, ops)]
        if interact_type == "ising":  # pulser's ising basis order to emu-sv's
            for t in out:
                t[:2, :2] = torch.flip(t[:2, :2], (0, 1))
        return out
    if noise_type == "leakage":
        return []
    raise ValueError(f"no Lindblad operators for the noise type {noise_type!r}")


def compute_noise_from_lindbladians(lindbladians: list[torch.Tensor], dim: int = 2) -> torch.Tensor:
    """-0.5i sum_j L_j^dag L_j (jump_lindblad_operators.py:79-93)."""
    assert all(L.shape == (dim, dim) for L in lindbladians), \
        f"the noise term takes single-qubit ({dim} x {dim}) Lindblad operators"
    acc = torch.zeros(dim, dim, dtype=dtype)
    for L in lindbladians:
        L = torch.as_tensor(L).to(dtype)
        acc = acc + L.mH @ L
    return -0.5j * acc
