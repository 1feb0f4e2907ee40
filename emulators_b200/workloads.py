"""Seeded synthetic registers and pulses for the emu-sv time-evolution workloads.

No pulser sequence is built: the drive amplitudes are sampled analytically at the
step midpoints ``t_k + dt/2``, which is what the reference adapter feeds the
stepper (emu_base/pulser_adapter.py:155-231, midpoints at 193-194).  For the
linear ramps and constant amplitudes used here the reference's PCHIP
interpolation of the 1 ns pulser grid is exact, so the samples coincide.

Units follow the stepper: time in microseconds, Omega and delta in rad/us,
positions in micrometres, ``U_ij = C6 / r_ij**6`` in rad/us.

Workloads (all sizes are the ones the benchmarks and parity tests use):

* ``chain_n10``      N=10 chain, 5 um spacing, Omega=4, delta -10 -> 10 over 1 us,
                     dt=10 ns (100 steps), complex128, tolerance 1e-10.
* ``lattice_n20``    N=20 4x5 square lattice, 6 um spacing, Omega = 2 pi sin^2(pi t/3),
                     delta -15 -> 15 over 3 us, dt=10 ns (300 steps), Krylov dim <= 30.
* ``ladder_n26``     N=26 2x13 ladder, 5.5 um spacing, chain_n10 pulse shapes over
                     2 us, dt=5 ns (400 steps), complex64 vectors / FP64 scalars.
* ``batch_256``      256 registers, N ~ U{12..18}, positions uniform in a 40x40 um box
                     rejection-sampled to a 5 um minimum distance, 10-segment
                     piecewise-linear Omega in [0, 2 pi] and delta in [-20, 20], phi=0,
                     1.5 us at dt=10 ns (150 steps).
* ``noisy_ladder_n22`` N=22 2x11 ladder, 5.5 um spacing, the ladder_n26 pulse shapes over
                     0.5 us at dt=10 ns (50 steps), Lindblad operators: relaxation
                     (rate 0.5/us, sqrt(rate)|g><r|) and dephasing (rate 1/us,
                     sqrt(rate/2) Z), complex128; the Monte Carlo stepper's workload.
* ``lindblad_ladder_n12`` N=12 2x6 ladder, 5.5 um spacing, Omega 4, delta -10 -> 10 over
                     0.2 us at dt=10 ns (20 steps), the noisy ladder's Lindblad operators;
                     a 4^12 density matrix (complex128), the density-matrix stepper's
                     workload.
* ``ring_n16_grad``  N=16 ring of radius 10 um, 20-segment piecewise-constant Omega in
                     [0, 2 pi] and delta in [-20, 20], 64 parameter sets, 2 us at
                     dt=10 ns (200 steps, 10 steps per segment), loss = MSE between the
                     final occupations and the Neel pattern [1, 0, 1, 0, ...].
"""

from __future__ import annotations

import dataclasses

import numpy as np

C6 = 5420158.53  # rad * um^6 / us (Rb 70S, the value pulser's AnalogDevice uses)

BATCH_SEED = 20261203
GRAD_SEED = 16022026


# ----------------------------------------------------------------------------- registers
def chain(n: int, spacing: float) -> np.ndarray:
    return np.stack([np.arange(n) * spacing, np.zeros(n)], axis=1).astype(np.float64)


def square_lattice(rows: int, cols: int, spacing: float) -> np.ndarray:
    ys, xs = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    return np.stack([xs.ravel() * spacing, ys.ravel() * spacing], axis=1).astype(np.float64)


def ladder(rungs: int, spacing: float) -> np.ndarray:
    """2 x ``rungs`` ladder; atom order runs along the first leg, then the second."""
    return square_lattice(2, rungs, spacing)


def ring(n: int, radius: float) -> np.ndarray:
    ang = 2.0 * np.pi * np.arange(n) / n
    return np.stack([radius * np.cos(ang), radius * np.sin(ang)], axis=1)


def random_box(n: int, side: float, min_dist: float, rng: np.random.Generator) -> np.ndarray:
    """Uniform positions in a ``side`` x ``side`` box, each new atom rejection-sampled
    until it is at least ``min_dist`` from every atom already placed."""
    pts: list[np.ndarray] = []
    while len(pts) < n:
        p = rng.uniform(0.0, side, size=2)
        if all(np.hypot(*(p - q)) >= min_dist for q in pts):
            pts.append(p)
    return np.array(pts)


def interaction_matrix(pos: np.ndarray, c6: float = C6) -> np.ndarray:
    """Full symmetric ``U_ij = C6 / r_ij^6`` with a zero diagonal (what pulser's
    ``interaction_matrix`` returns; only the upper triangle enters the Hamiltonian)."""
    d = pos[:, None, :] - pos[None, :, :]
    r2 = np.einsum("ijk,ijk->ij", d, d)
    n = len(pos)
    u = np.zeros((n, n))
    iu = np.triu_indices(n, 1)
    u[iu] = c6 / r2[iu] ** 3
    return u + u.T


# ----------------------------------------------------------------------------- workloads
@dataclasses.dataclass
class Workload:
    name: str
    positions: np.ndarray
    U: np.ndarray
    dt: float  # us
    omega: np.ndarray  # [nsteps, N] float64, rad/us, midpoint samples
    delta: np.ndarray  # [nsteps, N]
    phi: np.ndarray  # [nsteps, N]
    tolerance: float = 1e-10
    max_krylov_dim: int = 100
    precision: str = "c128"
    obs_every: int = 0  # observables every k steps (0: only at the end)

    @property
    def nqubits(self) -> int:
        return self.U.shape[0]

    @property
    def nsteps(self) -> int:
        return self.omega.shape[0]


def midpoints(duration: float, dt: float) -> np.ndarray:
    nsteps = int(round(duration / dt))
    return (np.arange(nsteps) + 0.5) * dt


def _global(vals: np.ndarray, n: int) -> np.ndarray:
    return np.repeat(vals[:, None], n, axis=1).astype(np.float64)


def chain_n10() -> Workload:
    n, T, dt = 10, 1.0, 0.01
    pos = chain(n, 5.0)
    t = midpoints(T, dt)
    return Workload("chain_n10", pos, interaction_matrix(pos), dt,
                    _global(np.full_like(t, 4.0), n), _global(-10.0 + 20.0 * t / T, n),
                    np.zeros((len(t), n)), tolerance=1e-10, obs_every=10)


def lattice_n20() -> Workload:
    n, T, dt = 20, 3.0, 0.01
    pos = square_lattice(4, 5, 6.0)
    t = midpoints(T, dt)
    om = 2.0 * np.pi * np.sin(np.pi * t / T) ** 2
    return Workload("lattice_n20", pos, interaction_matrix(pos), dt, _global(om, n),
                    _global(-15.0 + 30.0 * t / T, n), np.zeros((len(t), n)),
                    tolerance=1e-10, max_krylov_dim=30, obs_every=10)


def ladder_n26(nsteps: int | None = None) -> Workload:
    n, T, dt = 26, 2.0, 0.005
    pos = ladder(13, 5.5)
    t = midpoints(T, dt)
    if nsteps is not None:
        t = t[:nsteps]
    return Workload("ladder_n26", pos, interaction_matrix(pos), dt,
                    _global(np.full_like(t, 4.0), n), _global(-10.0 + 20.0 * t / T, n),
                    np.zeros((len(t), n)), tolerance=1e-10, precision="c64", obs_every=100)


def noisy_ladder_n22(nsteps: int | None = None):
    """(Workload, Lindblad operators as 2x2 complex arrays)."""
    n, T, dt = 22, 0.5, 0.01
    pos = ladder(11, 5.5)
    t = midpoints(T, dt)
    if nsteps is not None:
        t = t[:nsteps]
    w = Workload("noisy_ladder_n22", pos, interaction_matrix(pos), dt,
                 _global(np.full_like(t, 4.0), n), _global(-10.0 + 20.0 * t / T, n),
                 np.zeros((len(t), n)), tolerance=1e-10, precision="c128")
    relax = np.array([[0.0, np.sqrt(0.5)], [0.0, 0.0]], dtype=np.complex128)
    c = np.sqrt(1.0 / 2)
    deph = np.array([[c, 0.0], [0.0, -c]], dtype=np.complex128)
    return w, [relax, deph]


def lindblad_ladder_n12():
    """(Workload, Lindblad operators as 2x2 complex arrays)."""
    n, T, dt = 12, 0.2, 0.01
    pos = ladder(6, 5.5)
    t = midpoints(T, dt)
    w = Workload("lindblad_ladder_n12", pos, interaction_matrix(pos), dt,
                 _global(np.full_like(t, 4.0), n), _global(-10.0 + 20.0 * t / T, n),
                 np.zeros((len(t), n)), tolerance=1e-10, precision="c128")
    return w, noisy_ladder_n22()[1]


def piecewise_linear(knots_t: np.ndarray, knots_v: np.ndarray, t: np.ndarray) -> np.ndarray:
    return np.interp(t, knots_t, knots_v)


def batch_256(count: int = 256, seed: int = BATCH_SEED) -> list[Workload]:
    T, dt, nseg = 1.5, 0.01, 10
    rng = np.random.default_rng(seed)
    t = midpoints(T, dt)
    kt = np.linspace(0.0, T, nseg + 1)
    out = []
    for k in range(count):
        n = int(rng.integers(12, 19))
        pos = random_box(n, 40.0, 5.0, rng)
        om = piecewise_linear(kt, rng.uniform(0.0, 2.0 * np.pi, nseg + 1), t)
        de = piecewise_linear(kt, rng.uniform(-20.0, 20.0, nseg + 1), t)
        out.append(Workload(f"batch_{k}", pos, interaction_matrix(pos), dt, _global(om, n),
                            _global(de, n), np.zeros((len(t), n)), tolerance=1e-10,
                            precision="c64"))
    return out


@dataclasses.dataclass
class GradWorkload:
    positions: np.ndarray
    U: np.ndarray
    dt: float
    steps_per_segment: int
    omega_seg: np.ndarray  # [nsets, nseg]
    delta_seg: np.ndarray  # [nsets, nseg]
    target: np.ndarray  # [N] Neel pattern
    tolerance: float = 1e-10

    @property
    def nqubits(self) -> int:
        return self.U.shape[0]

    @property
    def nsegments(self) -> int:
        return self.omega_seg.shape[1]


def ring_n16_grad(nsets: int = 64, nseg: int = 20, steps_per_segment: int = 10,
                  n: int = 16, seed: int = GRAD_SEED) -> GradWorkload:
    rng = np.random.default_rng(seed)
    pos = ring(n, 10.0)
    om = rng.uniform(0.0, 2.0 * np.pi, (nsets, nseg))
    de = rng.uniform(-20.0, 20.0, (nsets, nseg))
    target = np.array([(i + 1) % 2 for i in range(n)], dtype=np.float64)
    return GradWorkload(pos, interaction_matrix(pos), 0.01, steps_per_segment, om, de, target)


def neel(n: int) -> np.ndarray:
    return np.array([(i + 1) % 2 for i in range(n)], dtype=np.float64)


def state_bytes(nqubits: int, precision: str) -> int:
    return (1 << nqubits) * (16 if precision == "c128" else 8)


def hilbert_dim(nqubits: int) -> int:
    return 1 << nqubits


__all__ = [
    "C6", "Workload", "GradWorkload", "chain", "square_lattice", "ladder", "ring",
    "random_box", "interaction_matrix", "chain_n10", "lattice_n20", "ladder_n26",
    "batch_256", "ring_n16_grad", "neel", "midpoints", "state_bytes", "hilbert_dim",
]
