"""Failure paths on the GPU, in forms that fault no GPU.

* A bounded device wait made to run out, under both batch schedulers: the lock-step
  engine's grid barrier with a short wait limit and one CTA that never arrives, and the
  phase engine with one register's first phase never published
  (emusv_batch_set_barrier_test).  Every waiting warp gives up, the launch reports
  EMUSV_TIMEOUT (TimeoutError), and the same workspace then runs the batch and matches the
  oracle.
* A non-finite state, copied in from a host buffer holding a NaN: the Lanczos step, the
  Arnoldi step and the adjoint step report EMUSV_NONFINITE, raised as NonFiniteError -- a
  FloatingPointError and, like the reference's Lanczos loop, which never converges on such a
  state (emu_base/math/krylov_exp.py:126-129, emu_base/math/double_krylov.py:107-110), a
  RecursionError -- and the next step on the same device matches the oracle.
"""

import dataclasses

import numpy as np
import pytest
import torch

from conftest import golden

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


def _batch(sizes, steps, seed):
    from emulators_b200 import workloads as wl

    rng = np.random.default_rng(seed)
    regs = []
    for n in sizes:
        pos = wl.random_box(n, 20.0, 5.0, rng)
        om = rng.uniform(0, 2 * np.pi, (steps, 1)) * np.ones((1, n))
        de = rng.uniform(-20, 20, (steps, 1)) * np.ones((1, n))
        regs.append(_Reg(wl.interaction_matrix(pos), 0.01, om, de, np.zeros((steps, n))))
    return regs


def _oracle_chain(oracle, r):
    s = np.zeros(1 << r.U.shape[0], dtype=np.complex128)
    s[0] = 1.0
    for k in range(r.omega.shape[0]):
        s, _, _ = oracle.evolve_step(r.dt, r.omega[k], r.delta[k], r.phi[k], r.U, s, r.tolerance, 100)
    return s


@pytest.mark.parametrize("engine", [0, 1])
def test_batch_barrier_timeout_then_recovers(oracle, engine):
    """Both schedulers: lock-step rounds (a CTA that never arrives at the first grid
    barrier) and the phase engine (register 0's first phase never published, so the warps
    find no work and their starvation limit runs out)."""
    from emulators_b200.batch import BatchEvolution

    regs = _batch([9, 10, 11, 12], 3, seed=11)
    b = BatchEvolution(regs, precision="c128", max_krylov_dim=100)
    b.reset()
    b.prepare(8, 40)
    b.set_engine(engine)
    # a wait of 2e6 SM cycles (about 1 ms) for an arrival that never comes
    b.set_barrier_test(wait_cycles=2_000_000, skip_first_arrival=True)
    b.launch(1)
    with pytest.raises(TimeoutError):
        b.results()
    # the same workspace with the switch off: the batch runs and matches the oracle
    b.set_barrier_test(0, False)
    b.reset()
    b.prepare(8, 40)
    b.set_engine(engine)
    b.launch(1)
    status, _ = b.results()
    assert (status == 0).all()
    for i, r in enumerate(regs):
        ref = _oracle_chain(oracle, r)
        assert np.abs(b.state(i).cpu().numpy() - ref).max() < 1e-10


def _nan_state(n, dtype, seed=0):
    rng = np.random.default_rng(seed)
    host = (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)) / np.sqrt(2 << n)
    host[(1 << n) // 3] = np.nan
    return host, torch.as_tensor(host).to(DEV, dtype)


def _params(n, seed=1):
    from emulators_b200 import workloads as wl

    rng = np.random.default_rng(seed)
    return (rng.uniform(0, 6, n), rng.uniform(-15, 15, n), rng.normal(size=n),
            wl.interaction_matrix(wl.chain(n, 6.0)))


@pytest.mark.parametrize("n,dtype", [(8, torch.complex128), (13, torch.complex128), (16, torch.complex64)])
def test_krylov_step_nonfinite_state(oracle, n, dtype):
    """Single-pass (n = 8) and multi-pass (H-first) registers."""
    from emulators_b200 import EvolveStateVector, _lib

    om, de, ph, U = _params(n)
    args = (0.01, torch.as_tensor(om), torch.as_tensor(de), torch.as_tensor(ph), torch.as_tensor(U))
    host, psi = _nan_state(n, dtype)
    with pytest.raises(_lib.NonFiniteError) as e:
        EvolveStateVector().apply(*args, psi, 1e-10, None)
    assert isinstance(e.value, FloatingPointError) and isinstance(e.value, RecursionError)
    # the next step on the same device (same cached workspace) is the oracle's
    host[(1 << n) // 3] = 0.0
    host /= np.linalg.norm(host)
    out, _ = EvolveStateVector().apply(*args, torch.as_tensor(host).to(DEV, dtype), 1e-10, None)
    ref, _, _ = oracle.evolve_step(0.01, om, de, ph, U, host, 1e-10)
    tol = 1e-10 if dtype == torch.complex128 else 2e-5
    assert np.abs(out.cpu().to(torch.complex128).numpy() - ref).max() < tol


def test_arnoldi_step_nonfinite_state():
    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian, _lib
    from emulators_b200.krylov import fused_arnoldi_step

    n = 12
    om, de, ph, U = _params(n)
    noise = golden("noisy")["noise"]
    H = RydbergHamiltonian(*(torch.as_tensor(a) for a in (om, de, ph, U)), DEV, noise=torch.as_tensor(noise))
    _, psi = _nan_state(n, torch.complex128)
    with pytest.raises(_lib.NonFiniteError):
        fused_arnoldi_step(HamiltonianExpOperator(H, 0.01), psi, 1e-10, 1e-10, 100)


@pytest.mark.parametrize("which", ["state", "gradient"])
def test_adjoint_step_nonfinite(which):
    from emulators_b200 import RydbergHamiltonian, _lib
    from emulators_b200.adjoint import parameter_gradients

    n = 10
    om, de, ph, U = _params(n)
    H = RydbergHamiltonian(*(torch.as_tensor(a) for a in (om, de, ph, U)), DEV)
    _, bad = _nan_state(n, torch.complex128)
    rng = np.random.default_rng(4)
    good = torch.as_tensor(rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)).to(DEV)
    good /= torch.linalg.vector_norm(good)
    state, grad = (bad, good) if which == "state" else (good, bad)
    with pytest.raises(_lib.NonFiniteError):
        parameter_gradients(H, 0.01, state, grad, 1e-10, 100)
