"""Drive preparation on the GPU: PCHIP interpolation and midpoint drive samples, the
drop-in for ``emu_base.math.pchip_torch.PCHIP1D`` (reference emu_base/math/pchip_torch.py:
218-269) and the sampling core of ``_extract_omega_delta_phi``
(emu_base/pulser_adapter.py:155-231).

``PCHIP1D(x, y)`` validates like the reference and evaluates with ``emusv_pchip_eval``;
``y`` may also be 2-D ``[signals, knots]`` (many signals on the same knots, one launch).
``midpoint_samples`` turns per-qubit amplitude / detuning / phase samples on pulser's
1 ns grid into the stepper's midpoint samples for a list of target times, all signals of a
sequence in one launch.
"""

from __future__ import annotations

import torch

from . import _lib


class PCHIP1D:
    """Shape-preserving C1 piecewise-cubic Hermite interpolant (pchip_torch.py:218-269)."""

    def __init__(self, x: torch.Tensor, y: torch.Tensor):
        self.x, self.y = self._validate_xy(x, y)
        dev = self.x.device if self.x.is_cuda else torch.device("cuda", torch.cuda.current_device())
        self._dev = dev
        self._xd = self.x.to(dev, torch.float64).contiguous()
        y2 = self.y.reshape(-1, self.y.shape[-1]) if self.y.ndim == 2 else self.y.reshape(1, -1)
        self._yd = y2.to(dev, torch.float64).contiguous()

    @staticmethod
    def _validate_xy(x, y):
        """pchip_torch.py:235-256 (plus 2-D y: signals x knots)."""
        x = torch.as_tensor(x)
        if not x.is_floating_point():
            raise TypeError("x must be a floating point tensor")
        y = torch.as_tensor(y, dtype=x.dtype, device=x.device)
        if not y.is_floating_point():
            raise TypeError("y must be a floating point tensor")
        if x.ndim != 1 or y.ndim not in (1, 2):
            raise ValueError("x and y must be 1D tensors")
        if x.numel() != y.shape[-1]:
            raise ValueError("x and y must have the same length")
        if x.numel() < 2:
            raise ValueError("Need at least 2 points")
        if not torch.all(x[1:] > x[:-1]):
            raise ValueError("x must be strictly increasing")
        return x, y

    def __call__(self, xq: torch.Tensor) -> torch.Tensor:
        xq = torch.as_tensor(xq, dtype=self.x.dtype, device=self.x.device)
        q = xq.reshape(-1).to(self._dev, torch.float64).contiguous()
        S, n = self._yd.shape
        out = torch.empty(S, q.numel(), dtype=torch.float64, device=self._dev)
        _lib.check(_lib.load().emusv_pchip_eval(
            n, self._xd.data_ptr(), S, self._yd.data_ptr(), n, q.numel(), q.data_ptr(),
            out.data_ptr(), q.numel(), torch.cuda.current_stream(self._dev).cuda_stream), "pchip")
        shape = tuple(xq.shape) if self.y.ndim == 1 else (S, *xq.shape)
        return out.reshape(shape).to(self.x.device, self.x.dtype)


def midpoint_samples(amp: torch.Tensor, det: torch.Tensor, phase: torch.Tensor, target_times,
                     device=None):
    """(omega, delta, phi) [steps, qubits] complex128 at the midpoints of ``target_times``
    (ns) from per-qubit samples ``[qubits, T]`` on pulser's grid t = 0, 1, ..., T-1
    (pulser_adapter.py:188-231): PCHIP of every signal, the last amplitude sample clamped
    at zero from below.  Qubits without samples are rows of zeros, as in the reference."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    tt = torch.as_tensor(target_times, dtype=torch.float64)
    t_mid = (0.5 * (tt[:-1] + tt[1:])).to(dev)
    T = int(torch.as_tensor(amp).shape[-1])
    t_grid = torch.arange(T, dtype=torch.float64, device=dev)
    sig = torch.cat([torch.as_tensor(a, dtype=torch.float64).reshape(-1, T)
                     for a in (amp, det, phase)]).to(dev)
    Q = sig.shape[0] // 3
    vals = PCHIP1D(t_grid, sig)(t_mid)  # [3Q, steps]
    om, de, ph = (vals[k * Q:(k + 1) * Q].T.contiguous() for k in range(3))
    om[-1] = torch.where(om[-1] > 0, om[-1], torch.zeros_like(om[-1]))
    return tuple(a.to(torch.complex128) for a in (om, de, ph))
