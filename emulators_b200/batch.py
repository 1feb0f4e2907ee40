"""Batched time evolution of many registers in one persistent launch.

The reference evolves one register per run of its time loop (emu_sv/sv_backend_impl.py:
197-209: one ``krylov_exp`` per step, emu_base/math/krylov_exp.py:23-131).
:class:`BatchEvolution` evolves a whole list of registers -- uneven atom counts, each with
its own pulse -- through all their steps inside ONE cooperative persistent kernel
(``emusv_batch_launch``), optionally recorded once into a CUDA graph and replayed.  Every
instance follows the same Lanczos/Expokit stopping rule as a single step.

:func:`autotune` picks the launch shape (tile bits x CTAs per SM) by timing short probe
runs of the batch itself and sizes the Krylov basis from the probe's iteration counts;
results are cached per batch signature.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import torch

from . import _lib

TILE_BITS = {_lib.C64: (8, 9, 10), _lib.C128: (8, 9)}


def _pack(workloads, key):
    return np.ascontiguousarray(np.concatenate(
        [np.asarray(getattr(w, key), dtype=np.float64).reshape(-1) for w in workloads]))


@dataclasses.dataclass
class TuneResult:
    tile_bits: int
    blocks_per_sm: int
    capacity: int
    ms: dict
    engine: int = 0  # 0 lock-step rounds, 1 per-register phases (emusv_batch_set_engine)


_tuned: dict = {}


class BatchEvolution:
    """Registers ``workloads`` (objects with ``U [n,n]``, ``dt`` (us), ``omega/delta/phi
    [nsteps, n]`` midpoint samples, ``tolerance``) evolved together from ``states``
    (default: every register in |g...g>).  ``precision`` "c64" (complex64 vectors, FP64
    scalars) or "c128"."""

    def __init__(self, workloads, precision: str = "c64", max_krylov_dim: int = 100,
                 states: torch.Tensor | None = None, device="cuda", tolerance=None):
        if not workloads:
            raise ValueError("empty batch")
        self.workloads = list(workloads)
        self.device = torch.device(device)
        self.dtype = torch.complex64 if precision == "c64" else torch.complex128
        self.code = _lib.dtype_code(self.dtype)
        self.nq = np.array([w.U.shape[0] for w in self.workloads], dtype=np.int32)
        maxq = _lib.load().emusv_batch_max_qubits()
        if self.nq.max() > maxq:
            raise ValueError(f"batched registers are limited to {maxq} qubits")
        self.nsteps = np.array([np.asarray(w.omega).shape[0] for w in self.workloads], dtype=np.int32)
        self.dt = np.array([w.dt for w in self.workloads], dtype=np.float64)
        self.tol = float(tolerance if tolerance is not None else self.workloads[0].tolerance)
        self.max_krylov_dim = int(max_krylov_dim)
        self.omegas, self.deltas, self.phis = (_pack(self.workloads, k) for k in ("omega", "delta", "phi"))
        self.U = _pack(self.workloads, "U")
        self.sizes = (1 << self.nq.astype(np.int64))
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)[:-1]])
        total = int(self.sizes.sum())
        if states is None:
            states = torch.zeros(total, dtype=self.dtype, device=self.device)
            states[torch.as_tensor(self.offsets, device=self.device)] = 1.0
        if states.numel() != total or states.dtype != self.dtype or not states.is_cuda:
            raise ValueError("states must be a packed CUDA vector of the batch's amplitudes")
        self.initial = states.contiguous().clone()
        self.states = self.initial.clone()
        self.ws = None
        self.shape = None
        self.graph = None
        self.iterations = None

    @property
    def max_steps(self) -> int:
        return int(self.nsteps.max())

    def signature(self):
        return (tuple(np.bincount(self.nq).tolist()), self.code, self.max_krylov_dim)

    def state(self, i: int) -> torch.Tensor:
        o = int(self.offsets[i])
        return self.states[o:o + int(self.sizes[i])]

    def reset(self) -> None:
        self.states.copy_(self.initial)

    # ---------------------------------------------------------------- C ABI steps
    def prepare(self, tile_bits: int, capacity: int) -> None:
        L = _lib.load()
        nq, ns = self.nq, self.nsteps
        need = L.emusv_batch_workspace_bytes(len(nq), nq.ctypes.data, ns.ctypes.data, self.code,
                                             tile_bits, capacity)
        if need == 0:
            raise ValueError(f"unsupported batch shape (tile bits {tile_bits})")
        if self.ws is None or self.ws.numel() < need:
            self.ws = None
            self.ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        st = L.emusv_batch_prepare(len(nq), nq.ctypes.data, ns.ctypes.data, self.dt.ctypes.data,
                                   self.code, self.omegas.ctypes.data, self.deltas.ctypes.data,
                                   self.phis.ctypes.data, self.U.ctypes.data,
                                   self.states.data_ptr(), self.tol, self.tol,
                                   self.max_krylov_dim, tile_bits, capacity, self.ws.data_ptr(),
                                   self.ws.numel(), _lib.stream_of(self.states))
        _lib.check(st, "batch prepare")
        self.shape = (tile_bits, capacity)
        self.graph = None

    def set_barrier_test(self, wait_cycles: int = 0, skip_first_arrival: bool = False) -> None:
        """Failure-path test switch of the prepared workspace (off by default; reset by
        :meth:`prepare`): grid-barrier waits give up after ``wait_cycles`` SM clock cycles
        (0: the default, about 1 s) and, with ``skip_first_arrival``, one CTA never arrives
        at a launch's first barrier, so the launch ends with ``TimeoutError`` in
        :meth:`results` and the device stays usable."""
        st = _lib.load().emusv_batch_set_barrier_test(self.ws.data_ptr(), int(wait_cycles),
                                                      1 if skip_first_arrival else 0)
        _lib.check(st, "batch barrier test switch")

    def set_engine(self, engine: int) -> None:
        """Scheduling of the prepared workspace's launches (reset by :meth:`prepare`): 0
        lock-step rounds of the whole batch, 1 every register's own sequence of phases.
        Same results; the autotuner times both."""
        _lib.check(_lib.load().emusv_batch_set_engine(self.ws.data_ptr(), int(engine)),
                   "batch engine")

    def launch(self, blocks_per_sm: int) -> None:
        st = _lib.load().emusv_batch_launch(self.code, self.shape[0], blocks_per_sm,
                                            self.ws.data_ptr(), _lib.stream_of(self.states))
        _lib.check(st, "batch launch")

    def capture(self, blocks_per_sm: int) -> torch.cuda.CUDAGraph:
        """Record the persistent launch into a CUDA graph (replayed by :meth:`replay`)."""
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            st = _lib.load().emusv_batch_launch(self.code, self.shape[0], blocks_per_sm,
                                                self.ws.data_ptr(),
                                                torch.cuda.current_stream().cuda_stream)
        _lib.check(st, "batch launch (graph capture)")
        self.graph = g
        return g

    def replay(self) -> None:
        self.graph.replay()

    def results(self, raise_on_error: bool = True):
        n = len(self.nq)
        status = np.zeros(n, dtype=np.int32)
        iters = np.zeros((n, self.max_steps), dtype=np.int32)
        st = _lib.load().emusv_batch_results(n, self.max_steps, self.ws.data_ptr(),
                                             status.ctypes.data, iters.ctypes.data,
                                             _lib.stream_of(self.states))
        self.iterations = iters
        self.last_code = st
        if raise_on_error and st != _lib.OK:
            _lib.check(st, f"batch ({int((status != 0).sum())} instance(s) failed)")
        return status, iters

    # ---------------------------------------------------------------- one call
    def run(self, tune: bool = True, graph: bool = False, tile_bits: int | None = None,
            blocks_per_sm: int | None = None, capacity: int | None = None,
            engine: int | None = None):
        """Evolve every instance through all its steps from the initial states; returns
        (statuses, iterations [ninst, max_steps])."""
        if tune and tile_bits is None:
            t = autotune(self)
            tile_bits, blocks_per_sm = t.tile_bits, t.blocks_per_sm
            capacity = capacity or t.capacity
            engine = t.engine if engine is None else engine
        tile_bits = tile_bits or default_tile_bits(self)
        blocks_per_sm = blocks_per_sm or 1
        capacity = capacity or self.max_krylov_dim
        while True:
            self.reset()
            self.prepare(tile_bits, capacity)
            if engine:
                self.set_engine(engine)
            if graph:
                self.capture(blocks_per_sm)
                self.replay()
            else:
                self.launch(blocks_per_sm)
            status, iters = self.results(raise_on_error=False)
            if self.last_code != _lib.OK and not status.any():
                # a launch-wide failure (a wait that ran out, a CUDA error): no per-instance
                # status was written
                _lib.check(self.last_code, "batch launch")
            if (status == _lib.WORKSPACE_TOO_SMALL).any() and capacity < self.max_krylov_dim:
                capacity = min(self.max_krylov_dim, 2 * capacity)
                continue
            break
        if (status != 0).any():
            bad = int(np.flatnonzero(status)[0])
            _lib.check(int(status[bad]), f"batch instance {bad}")
        return status, iters


def default_tile_bits(b: BatchEvolution) -> int:
    return max(t for t in TILE_BITS[b.code] if t <= int(b.nq.min()))


def autotune(b: BatchEvolution, probe_steps: int = 3, reps: int = 2) -> TuneResult:
    """Time every launch shape (tile bits x CTAs per SM x scheduling engine) on the first
    ``probe_steps`` steps of the batch (on a copy of its states) and keep the fastest; the
    Krylov capacity is the probe's largest
    iteration count plus a margin.  Cached per batch signature."""
    key = b.signature()
    if key in _tuned:
        return _tuned[key]
    probe_wl = []
    for w in b.workloads:
        k = min(probe_steps, np.asarray(w.omega).shape[0])
        probe_wl.append(dataclasses.replace(w, omega=np.asarray(w.omega)[:k],
                                            delta=np.asarray(w.delta)[:k],
                                            phi=np.asarray(w.phi)[:k]) if dataclasses.is_dataclass(w)
                        else _Slice(w, k))
    probe = BatchEvolution(probe_wl, "c64" if b.code == _lib.C64 else "c128", b.max_krylov_dim,
                           states=b.initial.clone(), device=b.device, tolerance=b.tol)
    L = _lib.load()
    timings = {}
    best = None
    max_iters = 0
    for T in TILE_BITS[b.code]:
        if T > int(b.nq.min()):
            continue
        probe.prepare(T, b.max_krylov_dim)
        cap = L.emusv_batch_max_blocks_per_sm(b.code, T)
        for engine, bps in [(e, k) for e in (0, 1) for k in range(1, max(cap, 1) + 1)]:
            probe.set_engine(engine)
            ms = []
            for _ in range(reps + 1):
                probe.reset()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                probe.launch(bps)
                e1.record()
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
            status, iters = probe.results(raise_on_error=False)
            if probe.last_code != _lib.OK and not status.any():
                _lib.check(probe.last_code, "batch autotune probe")  # a launch-wide failure
            max_iters = max(max_iters, int(iters.max()))
            t = min(ms[1:])
            timings[f"T{T}_b{bps}" + ("_phases" if engine else "")] = round(t, 3)
            if best is None or t < best[0]:
                best = (t, T, bps, engine)
    capacity = min(b.max_krylov_dim, max(16, int(np.ceil(1.5 * max_iters)) + 4))
    res = TuneResult(best[1], best[2], capacity, timings, best[3])
    _tuned[key] = res
    return res


class _Slice:
    """First k steps of a workload-like object."""

    def __init__(self, w, k):
        self.U, self.dt, self.tolerance = w.U, w.dt, w.tolerance
        self.omega = np.asarray(w.omega)[:k]
        self.delta = np.asarray(w.delta)[:k]
        self.phi = np.asarray(w.phi)[:k]
