"""Batched pulse gradients: many parameter sets of one register, forward and adjoint in
persistent launches, with checkpointed states.

The reference differentiates a loss of the final state through one
``DifferentiableStateVectorEvolution`` per time step (emu_sv/time_evolution/torch.py:
122-378), one parameter set at a time, and keeps every step's input state
(torch.py:215).  :class:`PulseGradientBatch` takes a batch of parameter sets of the same
register and

* evolves all of them through every step in one persistent launch
  (``emusv_batch_launch_steps``), keeping the states after every ``checkpoint_every``-th
  step (the checkpoints);
* walks back over the checkpoint segments: recomputes the segment's states from its
  checkpoint (one launch, every state kept), then takes the segment's adjoint steps from
  the last to the first, each one launch for the whole batch (``emusv_batch_adjoint_launch``:
  both Lanczos bases, the Frechet-derivative block, the flip and bit sums the derivative
  operators reduce to, and exp(+i dt H) g from the gradient's own basis);
* sums the per-step, per-qubit gradients into the per-segment pulse parameters.

Loss: mean squared error between the final Rydberg occupations and a target pattern.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib

BMAXQ = 20  # row length of the per-step gradient records (emusv_batch_adjoint_launch)


class PulseGradientBatch:
    """``nsets`` piecewise-constant global pulses (``omega_seg``, ``delta_seg`` [nsets, nseg],
    rad/us; phi = 0), each segment ``steps_per_segment`` steps of ``dt`` (us), on the
    register with interaction matrix ``U``; loss MSE(<n_i>, target)."""

    def __init__(self, U, dt, omega_seg, delta_seg, steps_per_segment, target,
                 precision: str = "c128", checkpoint_every: int = 16, tolerance: float = 1e-10,
                 max_krylov_dim: int = 100, capacity: int | None = None,
                 tile_bits: int | None = None,
                 blocks_per_sm: int = 1, device="cuda", engine: int = 1):
        self.U = np.ascontiguousarray(U, dtype=np.float64)
        self.n = self.U.shape[0]
        self.dt = float(dt)
        self.omega_seg = np.asarray(omega_seg, dtype=np.float64)
        self.delta_seg = np.asarray(delta_seg, dtype=np.float64)
        self.nsets, self.nseg = self.omega_seg.shape
        self.sps = int(steps_per_segment)
        self.nsteps = self.nseg * self.sps
        self.target = torch.as_tensor(np.asarray(target, dtype=np.float64))
        self.dtype = torch.complex64 if precision == "c64" else torch.complex128
        self.code = _lib.dtype_code(self.dtype)
        self.ck = int(checkpoint_every)
        self.tol = float(tolerance)
        self.maxdim = int(max_krylov_dim)
        self.capacity = int(min(capacity or max_krylov_dim, max_krylov_dim))
        self.T = tile_bits or (9 if self.n >= 9 else 8)
        self.bps = int(blocks_per_sm)
        # forward scheduling (emusv_batch_set_engine): the parameter sets are registers of
        # one size with similar iteration counts, where each register's own phase sequence
        # beats lock-step rounds
        self.engine = int(engine)
        self.device = torch.device(device)
        if self.n > BMAXQ or self.n < self.T:
            raise ValueError(f"register of {self.n} qubits outside the batched range")
        self._prepare()

    # ------------------------------------------------------------------ set-up
    def _drives(self):
        seg = np.arange(self.nsteps) // self.sps
        om = np.repeat(self.omega_seg[:, seg][:, :, None], self.n, axis=2)  # [S, steps, n]
        de = np.repeat(self.delta_seg[:, seg][:, :, None], self.n, axis=2)
        return (np.ascontiguousarray(om.reshape(-1)), np.ascontiguousarray(de.reshape(-1)),
                np.zeros(om.size))

    def _prepare(self):
        L = _lib.load()
        S, D = self.nsets, 1 << self.n
        self.nq = np.full(S, self.n, dtype=np.int32)
        self.ns = np.full(S, self.nsteps, dtype=np.int32)
        self.dts = np.full(S, self.dt)
        self.om, self.de, self.ph = self._drives()
        self.Us = np.ascontiguousarray(np.tile(self.U.reshape(-1), S))
        dev = self.device
        self.states = torch.zeros(S * D, dtype=self.dtype, device=dev)
        self.states.view(S, D)[:, 0] = 1.0
        self.initial = self.states.clone()
        stream = torch.cuda.current_stream(dev).cuda_stream
        nf = L.emusv_batch_workspace_bytes(S, self.nq.ctypes.data, self.ns.ctypes.data, self.code,
                                           self.T, self.capacity)
        na = L.emusv_batch_adjoint_workspace_bytes(S, self.nq.ctypes.data, self.ns.ctypes.data,
                                                   self.code, self.T, self.capacity)
        if not nf or not na:
            raise ValueError("unsupported batch shape")
        self.ws_f = torch.empty(nf, dtype=torch.uint8, device=dev)
        self.ws_a = torch.empty(na, dtype=torch.uint8, device=dev)
        args = (S, self.nq.ctypes.data, self.ns.ctypes.data, self.dts.ctypes.data, self.code,
                self.om.ctypes.data, self.de.ctypes.data, self.ph.ctypes.data, self.Us.ctypes.data)
        _lib.check(L.emusv_batch_prepare(*args, self.states.data_ptr(), self.tol, self.tol,
                                         self.maxdim, self.T, self.capacity, self.ws_f.data_ptr(),
                                         nf, stream), "batch prepare")
        _lib.check(L.emusv_batch_set_engine(self.ws_f.data_ptr(), self.engine), "batch engine")
        _lib.check(L.emusv_batch_adjoint_prepare(*args, self.tol, self.maxdim, self.T, self.capacity,
                                                 self.ws_a.data_ptr(), na, stream),
                   "batch adjoint prepare")
        nck = self.nsteps // self.ck
        self.hist = torch.empty(max(nck, 1) * S * D, dtype=self.dtype, device=dev)
        self.rec = torch.empty(self.ck * S * D, dtype=self.dtype, device=dev)
        self.work = torch.empty(S * D, dtype=self.dtype, device=dev)
        self.g = torch.empty(S * D, dtype=self.dtype, device=dev)
        self.g2 = torch.empty_like(self.g)
        self.grads = torch.zeros(self.nsteps, S, 3, BMAXQ, dtype=torch.float64, device=dev)
        self.status = torch.zeros(self.nsteps, S, dtype=torch.int32, device=dev)

    # ------------------------------------------------------------------ passes
    def _launch_f(self, first, steps, states, hist, every):
        _lib.check(_lib.load().emusv_batch_launch_steps(
            self.code, self.T, self.bps, first, steps, states.data_ptr(),
            hist.data_ptr() if hist is not None else None, every, self.ws_f.data_ptr(),
            torch.cuda.current_stream(self.device).cuda_stream), "batch forward")

    def _launch_a(self, step, psi, gin, gout):
        _lib.check(_lib.load().emusv_batch_adjoint_launch(
            self.code, self.T, self.bps, step, psi.data_ptr(), gin.data_ptr(), gout.data_ptr(),
            self.grads[step].data_ptr(), self.status[step].data_ptr(), self.ws_a.data_ptr(),
            torch.cuda.current_stream(self.device).cuda_stream), "batch adjoint")

    def forward(self, check: bool = True) -> None:
        """All steps of every set; checkpoints after every ``checkpoint_every`` steps."""
        self.states.copy_(self.initial)
        self._launch_f(0, self.nsteps, self.states, self.hist, self.ck)
        if check:
            st = np.zeros(self.nsets, dtype=np.int32)
            it = np.zeros((self.nsets, self.nsteps), dtype=np.int32)
            _lib.check(_lib.load().emusv_batch_results(
                self.nsets, self.nsteps, self.ws_f.data_ptr(), st.ctypes.data, it.ctypes.data,
                torch.cuda.current_stream(self.device).cuda_stream), "batch forward")
            self.forward_iterations = it

    def occupations(self) -> torch.Tensor:
        """[nsets, n] Rydberg occupations of the current states
        (custom_callback_implementations.py:30-47)."""
        S, n = self.nsets, self.n
        p = (self.states.view(S, 1 << n).abs() ** 2).to(torch.float64)
        return torch.stack([p.view(S, 2 ** i, 2, -1)[:, :, 1].sum(dim=(1, 2)) for i in range(n)], 1)

    def _seed(self, occ: torch.Tensor) -> torch.Tensor:
        """dL/dpsi of the MSE loss in torch's convention: 2 (dL/d<n_i>) n_i psi summed."""
        S, n = self.nsets, self.n
        w = 2.0 * (occ - self.target.to(occ.device)) / n  # dL/d<n_i>
        x = torch.arange(1 << n, device=occ.device)
        bits = torch.stack([((x >> (n - 1 - i)) & 1).to(torch.float64) for i in range(n)])  # [n, D]
        fac = w @ bits  # [S, D]
        return (2.0 * fac).to(self.dtype) * self.states.view(S, 1 << n)

    def backward(self, occ: torch.Tensor) -> None:
        """Adjoint over the checkpoint segments, last to first; fills self.grads."""
        S, D = self.nsets, 1 << self.n
        self.g.copy_(self._seed(occ).reshape(-1))
        nck = (self.nsteps + self.ck - 1) // self.ck
        for seg in reversed(range(nck)):
            first = seg * self.ck
            L = min(self.ck, self.nsteps - first)
            start = self.initial if seg == 0 else self.hist.view(-1, S * D)[seg - 1]
            self.work.copy_(start)
            if L > 1:  # the states entering steps first+1 .. first+L-1
                self._launch_f(first, L - 1, self.work, self.rec, 1)
            for k in reversed(range(L)):
                psi = start if k == 0 else self.rec.view(-1, S * D)[k - 1]
                self._launch_a(first + k, psi, self.g, self.g2)
                self.g, self.g2 = self.g2, self.g

    def loss_and_grad(self):
        """(loss [nsets], dL/dOmega_seg [nsets, nseg], dL/ddelta_seg [nsets, nseg],
        dL/dpsi_0 [nsets, 2^n]) as host arrays."""
        self.forward()
        occ = self.occupations()
        loss = ((occ - self.target.to(occ.device)) ** 2).mean(dim=1)
        self.backward(occ)
        st = self.status.cpu().numpy()
        if (st != 0).any():
            s, i = np.argwhere(st != 0)[0]
            _lib.check(int(st[s, i]), f"adjoint of step {s}, set {i}")
        g = self.grads[:, :, :2, : self.n].sum(dim=3)  # [steps, S, 2]: summed over qubits
        g = g.view(self.nseg, self.sps, self.nsets, 2).sum(dim=1)  # [nseg, S, 2]
        return (loss.cpu().numpy(), g[:, :, 0].T.cpu().numpy(), g[:, :, 1].T.cpu().numpy(),
                self.g.view(self.nsets, -1).cpu().numpy())
