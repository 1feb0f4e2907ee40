"""GPU parity of the batched persistent evolution (emulators_b200.batch, C ABI
emusv_batch_*) against the oracle's step-by-step chain and the single-register path."""

import dataclasses

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda"


@dataclasses.dataclass
class _Reg:
    U: np.ndarray
    dt: float
    omega: np.ndarray
    delta: np.ndarray
    phi: np.ndarray
    tolerance: float = 1e-10


def _random_batch(sizes, steps, seed, phase=False):
    from emulators_b200 import workloads as wl

    rng = np.random.default_rng(seed)
    regs = []
    for n, k in zip(sizes, steps):
        pos = wl.random_box(n, max(20.0, 7.5 * np.sqrt(n)), 5.0, rng)
        om = rng.uniform(0, 2 * np.pi, (k, 1)) * np.ones((1, n))
        de = rng.uniform(-20, 20, (k, 1)) * np.ones((1, n))
        ph = rng.normal(size=(k, n)) if phase else np.zeros((k, n))
        regs.append(_Reg(wl.interaction_matrix(pos), 0.01, om, de, ph))
    return regs


def _oracle_chain(oracle, r):
    n = r.U.shape[0]
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1.0
    its = []
    for k in range(r.omega.shape[0]):
        s, _, info = oracle.evolve_step(r.dt, r.omega[k], r.delta[k], r.phi[k], r.U, s,
                                        r.tolerance, 100)
        its.append(info.iteration_count)
    return s, its


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("tile_bits", [8, 9])
def test_batch_c128_matches_oracle(oracle, tile_bits, engine):
    """Uneven registers and step counts, complex phases, both scheduling engines (lock-step
    rounds, per-register phases): every instance's final state and every step's Krylov
    iteration count equal the oracle's chain."""
    from emulators_b200.batch import BatchEvolution

    regs = _random_batch([9, 13, 10, 12, 11, 9], [7, 12, 10, 5, 11, 12], seed=3, phase=True)
    b = BatchEvolution(regs, precision="c128", max_krylov_dim=100)
    status, iters = b.run(tune=False, tile_bits=tile_bits, blocks_per_sm=1, capacity=40,
                          engine=engine)
    assert (status == 0).all()
    for i, r in enumerate(regs):
        ref, its = _oracle_chain(oracle, r)
        got = b.state(i).cpu().numpy()
        assert np.abs(got - ref).max() < 1e-10, (i, np.abs(got - ref).max())
        assert list(iters[i, :len(its)]) == its, (i, list(iters[i]), its)


def test_batch_c128_large_registers_match_oracle(oracle):
    """The top of the batched size range (the 256-register batch draws 12-18 qubits; the
    engine takes up to 20): complex128 registers of 14, 16, 18 and 20 qubits with complex phases against
    the oracle's chain, states and every step's Krylov iteration count."""
    from emulators_b200.batch import BatchEvolution

    regs = _random_batch([14, 20, 16, 18], [4, 3, 4, 3], seed=29, phase=True)
    b = BatchEvolution(regs, precision="c128", max_krylov_dim=100)
    status, iters = b.run(tune=False, tile_bits=9, blocks_per_sm=1, capacity=40)
    assert (status == 0).all()
    for i, r in enumerate(regs):
        ref, its = _oracle_chain(oracle, r)
        got = b.state(i).cpu().numpy()
        assert np.abs(got - ref).max() < 1e-10, (i, np.abs(got - ref).max())
        assert list(iters[i, :len(its)]) == its, (i, list(iters[i]), its)


def test_batch_c64_matches_single_register_path():
    """complex64 batch vs the single-register fused step (same precision form)."""
    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian
    from emulators_b200.batch import BatchEvolution
    from emulators_b200.krylov import fused_step

    regs = _random_batch([12, 18, 14, 16], [6, 6, 6, 6], seed=7)
    b = BatchEvolution(regs, precision="c64", max_krylov_dim=100)
    status, _ = b.run(tune=False, tile_bits=10, blocks_per_sm=1, capacity=40)
    assert (status == 0).all()
    for i, r in enumerate(regs):
        n = r.U.shape[0]
        s = torch.zeros(1 << n, dtype=torch.complex64, device=DEV)
        s[0] = 1.0
        for k in range(r.omega.shape[0]):
            H = RydbergHamiltonian(*(torch.as_tensor(a) for a in (r.omega[k], r.delta[k], r.phi[k], r.U)),
                                   DEV)
            s, _, st = fused_step(HamiltonianExpOperator(H, r.dt), s, r.tolerance, r.tolerance, 100)
            assert st == 0
        err = torch.linalg.vector_norm(b.state(i).to(torch.complex128) - s.to(torch.complex128)).item()
        assert err < 2e-5, (i, err)


def test_batch_autotune_graph_replay_and_capacity_retry():
    """The C4 batch shape (first 24 registers, first 15 steps): autotuned launch, the
    same launch replayed from a CUDA graph gives the same bits, and a too-small Krylov
    capacity is retried."""
    from emulators_b200 import workloads as wl
    from emulators_b200.batch import BatchEvolution, autotune

    regs = [dataclasses.replace(w, omega=w.omega[:15], delta=w.delta[:15], phi=w.phi[:15])
            for w in wl.batch_256()[:24]]
    b = BatchEvolution(regs, precision="c64")
    t = autotune(b)
    assert t.tile_bits in (8, 9, 10) and t.blocks_per_sm >= 1 and t.capacity >= 16
    status, iters = b.run(tune=True)
    assert (status == 0).all() and (iters > 0).all()
    direct = b.states.clone()
    b.reset()
    b.capture(t.blocks_per_sm)
    b.replay()
    status2, iters2 = b.results()
    assert (status2 == 0).all()
    assert torch.equal(b.states, direct)
    np.testing.assert_array_equal(iters, iters2)
    # capacity retry: 4 vectors are too few; run() doubles until the steps fit
    status3, _ = b.run(tune=False, tile_bits=t.tile_bits, blocks_per_sm=1, capacity=4)
    assert (status3 == 0).all()
    assert torch.equal(b.states, direct)
