"""Backend time loop and configuration, the drop-in for emu-sv's SVConfig / SVBackendImpl
(reference emu_sv/sv_config.py:33-155, emu_sv/sv_backend_impl.py:74-262,
emu_sv/sv_backend.py:7-42).

pulser is not a dependency: the loop consumes a :class:`SequenceData` (the reference's
adapter output, emu_base/pulser_adapter.py:259-280) -- per-step midpoint samples of
Omega/delta/phi, the target-time grid in ns and the interaction matrix -- and the
observables are small local classes with pulser's names and evaluation-time semantics.
"""

from __future__ import annotations

import bisect
import dataclasses
import logging
import math
import time
from typing import Callable, Sequence

import numpy as np
import torch

from .hamiltonian import RydbergHamiltonian
from .observables import (correlation_matrix_sv_impl, energy_second_moment_sv_impl,
                          energy_sv_impl, energy_variance_sv_impl, qubit_occupation_sv_impl)
from .state_vector import StateVector
from .density_matrix import (DensityMatrix, correlation_matrix_sv_den_mat_impl,
                             energy_second_moment_den_mat_impl, energy_variance_sv_den_mat_impl,
                             qubit_occupation_sv_den_mat_impl)
from .time_evolution import EvolveDensityMatrix, EvolveMonteCarlo, EvolveStateVector

_TIME_CONVERSION_COEFF = 0.001  # Omega and delta in rad/us, dt in ns (sv_backend_impl.py:29)
logger = logging.getLogger("emulators")

# Relative times closer than this are one time (pulser.backend.observable.TIME_TOLERANCE, a
# third-party constant; 1e-6 is the value the target-time fixtures were generated with).
TIME_TOLERANCE = 1e-6


# ---------------------------------------------------------------- target-time grid
def fuzzy_union(base: Sequence[float], extra, tol: float = TIME_TOLERANCE) -> list[float]:
    """Sorted ``base`` with the sorted ``extra`` times merged in; a time of ``extra`` within
    ``tol`` of one already present is dropped, so ``base`` wins (pulser_adapter.py:80-95)."""
    merged = list(base)
    for t in extra:
        i = bisect.bisect_left(merged, t)
        if i > 0 and t - merged[i - 1] <= tol:
            continue
        if i < len(merged) and merged[i] - t <= tol:
            continue
        merged.insert(i, t)
    return merged


def get_target_times(duration: float, dt: float, observable_times=(),
                     tol: float = TIME_TOLERANCE) -> list[float]:
    """Absolute times (ns) at which a sequence of ``duration`` ns is sampled
    (pulser_adapter.py:130-151): the relative grid i dt / duration for i = 0..floor(duration
    / dt), 1.0 appended unless the grid already ends within ``tol`` of it, the observables'
    relative evaluation times merged in by :func:`fuzzy_union`, all scaled by duration."""
    duration = float(duration)
    n_steps = math.floor(duration / dt)
    rel = [i * float(dt) / duration for i in range(n_steps + 1)]
    if rel[-1] < 1.0 - tol:
        rel.append(1.0)
    rel = fuzzy_union(rel, sorted(set(float(t) for t in observable_times)), tol)
    return [t * duration for t in rel]


# ---------------------------------------------------------------- observables
class Observable:
    tag = "observable"

    def __init__(self, evaluation_times: Sequence[float] | None = None, tag_suffix: str = ""):
        self.evaluation_times = None if evaluation_times is None else [float(t) for t in evaluation_times]
        self.tag_suffix = tag_suffix

    @property
    def name(self) -> str:
        return self.tag + (f"_{self.tag_suffix}" if self.tag_suffix else "")

    def due(self, t: float, default_times: Sequence[float] | None = None) -> bool:
        """Whether relative time ``t`` is one of this observable's evaluation times, to
        TIME_TOLERANCE (pulser_adapter.py:98-127).  An observable without its own times
        takes the config's ``default_times``; with neither, it is due at every step."""
        times = self.evaluation_times if self.evaluation_times is not None else default_times
        if times is None:
            return True
        return any(abs(t - e) <= TIME_TOLERANCE for e in times)

    def apply(self, *, config, state, hamiltonian):  # pragma: no cover - overridden
        raise NotImplementedError


def _dm(state) -> bool:
    return isinstance(state, DensityMatrix)


class Occupation(Observable):
    tag = "occupation"

    def apply(self, *, config, state, hamiltonian):
        f = qubit_occupation_sv_den_mat_impl if _dm(state) else qubit_occupation_sv_impl
        return f(config=config, state=state, hamiltonian=hamiltonian)


class CorrelationMatrix(Observable):
    tag = "correlation_matrix"

    def apply(self, *, config, state, hamiltonian):
        f = correlation_matrix_sv_den_mat_impl if _dm(state) else correlation_matrix_sv_impl
        return f(config=config, state=state, hamiltonian=hamiltonian)


class Energy(Observable):
    tag = "energy"

    def apply(self, *, config, state, hamiltonian):
        if _dm(state):
            return hamiltonian.expect(state).cpu()
        return energy_sv_impl(config=config, state=state, hamiltonian=hamiltonian)


class EnergyVariance(Observable):
    tag = "energy_variance"

    def apply(self, *, config, state, hamiltonian):
        f = energy_variance_sv_den_mat_impl if _dm(state) else energy_variance_sv_impl
        return f(config=config, state=state, hamiltonian=hamiltonian)


class EnergySecondMoment(Observable):
    tag = "energy_second_moment"

    def apply(self, *, config, state, hamiltonian):
        f = energy_second_moment_den_mat_impl if _dm(state) else energy_second_moment_sv_impl
        return f(config=config, state=state, hamiltonian=hamiltonian)


class StateResult(Observable):
    tag = "state"

    def apply(self, *, config, state, hamiltonian):
        if _dm(state):
            return DensityMatrix(state.data.clone())
        return StateVector(state.data.clone())


class BitStrings(Observable):
    tag = "bitstrings"

    def __init__(self, evaluation_times=None, num_shots: int = 1000, tag_suffix: str = ""):
        super().__init__(evaluation_times, tag_suffix)
        self.num_shots = num_shots

    def apply(self, *, config, state, hamiltonian):
        return state.sample(self.num_shots)


class Statistics(Observable):
    """Per-step statistics (sv_backend_impl.py:32-71): the wall time of the step just taken
    and the peak device memory so far (MB, the largest over the GPUs), logged at INFO and
    stored under the tag ``statistics`` at every step of the time loop."""

    tag = "statistics"

    def __init__(self, timestep_count: int):
        super().__init__(None)
        self.durations: list[float] = []
        self.timestep_count = timestep_count

    def apply(self, *, config, state, hamiltonian):
        duration = self.durations[-1]
        if state.data.is_cuda:
            mem = max(torch.cuda.max_memory_allocated(d) * 1e-6 for d in range(torch.cuda.device_count()))
        else:  # pragma: no cover - the package keeps its states on the GPU
            import resource

            mem = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss * 1e-3
        logger.info(f"step = {len(self.durations)}/{self.timestep_count}, RSS = {mem:.3f} MB, "
                    f"\u0394t = {duration:.3f} s")
        return {"RSS": mem, "duration": duration}


class Results:
    """Per-observable time series: ``results.get(tag)`` -> list of values,
    ``results.times(tag)`` -> their normalised times; ``results.statistics`` the
    per-step statistics (tag ``statistics``)."""

    def __init__(self, atom_order: Sequence[str], total_duration: int):
        self.atom_order = tuple(atom_order)
        self.total_duration = total_duration
        self._data: dict[str, list] = {}
        self._times: dict[str, list] = {}

    def _store(self, tag: str, t: float, value) -> None:
        self._data.setdefault(tag, []).append(value)
        self._times.setdefault(tag, []).append(t)

    def get(self, tag: str) -> list:
        return self._data.get(tag, [])

    def times(self, tag: str) -> list:
        return self._times.get(tag, [])

    def __getattr__(self, tag):
        if tag.startswith("_"):
            raise AttributeError(tag)
        if tag in self._data:
            return self._data[tag]
        raise AttributeError(tag)


# ---------------------------------------------------------------- config and data
class SVConfig:
    """sv_config.py:75-122 keyword set, plus the B200 knobs:

    * ``precision``: "c128" (reference) or "c64" (complex64 vectors; FP64 Krylov scalars,
      tridiagonal exponential and norms);
    * ``krylov_dim_hint``: test convergence from the previous step's iteration count on.
    """

    def __init__(self, *, dt: float = 10.0, max_krylov_dim: int = 100,
                 krylov_tolerance: float = 1e-10, gpu: bool | None = None,
                 interaction_cutoff: float = 0.0, log_level: int = logging.INFO,
                 log_file=None, solver: str = "default", observables: Sequence[Observable] = (),
                 initial_state: StateVector | None = None, precision: str = "c128",
                 krylov_dim_hint: bool = True, **kwargs):
        if gpu is False:
            raise ValueError("emulators_b200 runs on the GPU only (gpu=False is not supported)")
        if precision not in ("c128", "c64"):
            raise ValueError("precision must be 'c128' or 'c64'")
        self.dt = dt
        self.max_krylov_dim = max_krylov_dim
        self.krylov_tolerance = krylov_tolerance
        self.gpu = gpu
        self.interaction_cutoff = interaction_cutoff
        self.log_level = log_level
        self.log_file = log_file
        self.solver = solver
        self.observables = tuple(observables)
        self.initial_state = initial_state
        self.precision = precision
        self.krylov_dim_hint = krylov_dim_hint
        # relative times of the observables that have none of their own; "Full" (or none
        # given) evaluates them at every step
        d = kwargs.pop("default_evaluation_times", None)
        self.default_evaluation_times = None if d is None or isinstance(d, str) else \
            tuple(float(t) for t in d)
        self._backend_options = dict(kwargs)

    @property
    def vector_dtype(self) -> torch.dtype:
        return torch.complex128 if self.precision == "c128" else torch.complex64


@dataclasses.dataclass
class SequenceData:
    """emu_base/pulser_adapter.py:259-280: midpoint samples [nsteps, N] (rad/us), the
    target-time grid in ns, and U(t) (a callable returning [1, N, N] like the adapter's
    _InteractionMatrixCallable, or a fixed [N, N] tensor)."""

    omega: torch.Tensor
    delta: torch.Tensor
    phi: torch.Tensor
    target_times: list
    interaction_matrix: Callable | torch.Tensor
    qubit_ids: tuple = ()
    lindblad_ops: list = dataclasses.field(default_factory=list)
    has_stochastic_noise: bool = False
    # state-preparation errors: the atoms of this run that were badly prepared (drawn per
    # run by the sequence sampler) and the error probability
    bad_atoms: tuple = ()
    state_prep_error: float = 0.0

    def U(self, t: float) -> torch.Tensor:
        if callable(self.interaction_matrix):
            return self.interaction_matrix(t)[0]
        return self.interaction_matrix

    @classmethod
    def from_samples(cls, amp, det, phase, duration: float, dt: float, interaction_matrix,
                     observable_times=(), qubit_ids: tuple = (), device=None) -> "SequenceData":
        """From per-qubit drive samples ``[qubits, T]`` on pulser's 1 ns grid: the target-time
        grid of ``duration`` ns with step ``dt`` ns and the observables' relative times
        (:func:`get_target_times`), then the PCHIP midpoint samples of every signal on the
        GPU (:func:`emulators_b200.pchip.midpoint_samples`), as the reference's adapter
        builds its data (pulser_adapter.py:130-231)."""
        from .pchip import midpoint_samples

        times = get_target_times(duration, dt, observable_times)
        om, de, ph = (a.cpu() for a in midpoint_samples(amp, det, phase, times, device))
        return cls(om, de, ph, times, torch.as_tensor(interaction_matrix), tuple(qubit_ids))

    @classmethod
    def from_workload(cls, w) -> "SequenceData":
        times = list(np.round(np.arange(w.nsteps + 1) * w.dt * 1000.0, 9))
        return cls(torch.as_tensor(w.omega), torch.as_tensor(w.delta), torch.as_tensor(w.phi),
                   times, torch.as_tensor(w.U), tuple(f"q{i}" for i in range(w.nqubits)))


# ---------------------------------------------------------------- time loop
class SVBackendImpl:
    """sv_backend_impl.py:74-262: the noiseless state-vector stepper, and with Lindblad
    operators the Monte Carlo stepper or the density-matrix stepper, chosen as the
    reference chooses (sv_backend_impl.py:82-95)."""

    def __init__(self, config: SVConfig, data: SequenceData):
        from . import krylov

        krylov.use_iteration_hint = bool(config.krylov_dim_hint)
        self._config = config
        self._data = data
        state_type = StateVector
        if data.lindblad_ops:
            solver = str(getattr(config.solver, "value", config.solver))
            if (solver == "default" and data.has_stochastic_noise) or solver == "montecarlo":
                self.stepper = EvolveMonteCarlo(config.max_krylov_dim)
            else:
                self.stepper = EvolveDensityMatrix(config.max_krylov_dim)
                state_type = DensityMatrix
        else:
            self.stepper = EvolveStateVector(config.max_krylov_dim)
        self.target_times = data.target_times
        self.omega, self.delta, self.phi = data.omega, data.delta, data.phi
        self.nsteps = data.omega.shape[0]
        self.nqubits = data.omega.shape[1]
        if config.initial_state is not None:
            if config.initial_state.n_qudits != self.nqubits:
                raise ValueError(
                    "Mismatch in number of atoms: initial state has "
                    f"{config.initial_state.n_qudits} and the sequence has {self.nqubits}")
            init = config.initial_state
            if state_type is DensityMatrix and not isinstance(init, DensityMatrix):
                init = DensityMatrix.from_state_vector(init)  # sv_backend_impl.py:143-160
            self.state = state_type(init.data.clone().to(config.vector_dtype))
        elif state_type is DensityMatrix:
            self.state = DensityMatrix(DensityMatrix.make(self.nqubits).data.to(config.vector_dtype))
        else:
            self.state = StateVector.make(self.nqubits, dtype=config.vector_dtype)
        self.results = Results(data.qubit_ids, int(self.target_times[-1]))
        self.statistics = Statistics(self.nsteps)
        self._current_H: RydbergHamiltonian | None = None
        self.init_dark_qubits()
        if config.initial_state is not None and data.state_prep_error > 0.0:
            raise NotImplementedError(
                "an initial state cannot be combined with a state-preparation error")
        self.time = time.time()

    def init_dark_qubits(self) -> None:
        """sv_backend_impl.py:162-184: with a state-preparation error, the badly prepared
        atoms of the run are dark -- their Omega, delta and phi are zero at every step and
        their rows and columns of the interaction matrix are zero (the caller's samples are
        left untouched)."""
        self.dark_qubits = None
        if self._data.state_prep_error > 0.0:
            mask = torch.as_tensor(tuple(bool(b) for b in self._data.bad_atoms), dtype=torch.bool)
            if mask.numel() != self.nqubits:
                raise ValueError(f"bad_atoms has {mask.numel()} entries for {self.nqubits} atoms")
            self.dark_qubits = mask
            self.omega, self.delta, self.phi = (a.clone() for a in (self.omega, self.delta, self.phi))
            for a in (self.omega, self.delta, self.phi):
                a[:, mask] = 0.0

    def _U(self, t: float) -> torch.Tensor:
        U = self._data.U(t)
        if self.dark_qubits is not None:
            U = torch.as_tensor(U).clone()
            U[self.dark_qubits, :] = 0.0
            U[:, self.dark_qubits] = 0.0
        return U

    def step(self, step_idx: int) -> None:
        dt = self.target_times[step_idx + 1] - self.target_times[step_idx]
        self._current_H = None
        torch.cuda.nvtx.range_push(f"step {step_idx + 1}")
        self.state.data, self._current_H = self.stepper.apply(
            dt * _TIME_CONVERSION_COEFF, self.omega[step_idx], self.delta[step_idx],
            self.phi[step_idx], self._U(self.target_times[step_idx]), self.state.data,
            self._config.krylov_tolerance, self._data.lindblad_ops)
        self._apply_observables(step_idx + 1)
        torch.cuda.nvtx.range_pop()
        self._save_statistics(step_idx + 1)

    def _save_statistics(self, step_idx: int) -> None:
        """sv_backend_impl.py:244-255: after every step (not only at observation times)."""
        t = self.target_times[step_idx] / self.target_times[-1]
        self.statistics.durations.append(time.time() - self.time)
        self.results._store(self.statistics.name, t, self.statistics.apply(
            config=self._config, state=self.state, hamiltonian=self._current_H))
        self.time = time.time()

    def _apply_observables(self, step_idx: int) -> None:
        """sv_backend_impl.py:211-242: renormalised state, H of the step just done."""
        t = self.target_times[step_idx] / self.target_times[-1]
        due = [o for o in self._config.observables
               if o.due(t, self._config.default_evaluation_times)]
        if not due:
            return
        norm = self.state.norm()
        if not torch.allclose(norm, torch.tensor(1.0, dtype=torch.float64)):
            state = type(self.state)((1.0 / norm.item()) * self.state.data)
        else:
            state = self.state
        if self._current_H is None:  # t = 0 (sv_backend_impl.py:224-234)
            self._current_H = self.stepper.get_hamiltonian(
                self.omega[0], self.delta[0], self.phi[0], self._data.lindblad_ops, self._U(
                    0.5 * (self.target_times[step_idx] + self.target_times[step_idx + 1])),
                state.data.device)
        for o in due:
            self.results._store(o.name, t, o.apply(config=self._config, state=state,
                                                   hamiltonian=self._current_H))

    def _run(self) -> Results:
        self._apply_observables(0)
        for step in range(self.nsteps):
            self.step(step)
        return self.results


class SVBackend:
    """sv_backend.py:7-42 without pulser: ``SVBackend(sequence_data, config).run()``."""

    def __init__(self, sequence: SequenceData | Sequence[SequenceData], config: SVConfig | None = None):
        self._sequences = [sequence] if isinstance(sequence, SequenceData) else list(sequence)
        self._config = config or SVConfig(observables=[BitStrings(evaluation_times=[1.0])])

    def run(self) -> Results | list[Results]:
        out = [SVBackendImpl(self._config, s)._run() for s in self._sequences]
        return out[0] if len(out) == 1 else out
