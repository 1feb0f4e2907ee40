"""GPU parity of the Krylov time step against the reference fixtures and the oracle."""

import numpy as np
import pytest
import torch

from conftest import cases, golden

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.fixture
def no_hint():
    """Test convergence at every iteration, exactly as the reference does."""
    from emulators_b200 import krylov

    old = krylov.use_iteration_hint
    krylov.use_iteration_hint = False
    yield
    krylov.use_iteration_hint = old


def _step(c, dtype=torch.complex128, tol=None):
    from emulators_b200 import EvolveStateVector

    tol = float(c["tol"]) if tol is None else tol
    s = torch.as_tensor(c["state"]).to(DEV, dtype)
    out, H = EvolveStateVector().apply(float(c["dt"]), torch.as_tensor(c["omegas"]),
                                       torch.as_tensor(c["deltas"]), torch.as_tensor(c["phis"]),
                                       torch.as_tensor(c["U"]), s, tol, None)
    return out.cpu().to(torch.complex128).numpy()


def test_step_matches_reference_fixtures(no_hint):
    # reference test_time_evolution.py:58-76: atol = tolerance vs dense expm
    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian, krylov_exp_impl

    for c in cases(golden("krylov_step")):
        out = _step(c)
        np.testing.assert_allclose(out, c["dense"], atol=float(c["tol"]), rtol=0)
        np.testing.assert_allclose(out, c["result"], atol=1e-12, rtol=0)
        H = RydbergHamiltonian(*(torch.as_tensor(c[k]) for k in ("omegas", "deltas", "phis", "U")), DEV)
        r = krylov_exp_impl(HamiltonianExpOperator(H, float(c["dt"])),
                            torch.as_tensor(c["state"]).to(DEV), True, float(c["tol"]),
                            float(c["tol"]), 100)
        assert r.iteration_count == int(c["iters"])
        assert r.happy_breakdown == bool(c["happy"])


def test_step_c64_precision_form():
    """complex64 vectors with FP64 scalars: error vs the complex128 reference ~1e-6."""
    for c in cases(golden("krylov_step")):
        out = _step(c, torch.complex64, tol=max(float(c["tol"]), 1e-10))
        err = np.linalg.norm(out - c["result"])
        assert err < 2e-6, err


def test_chain_n10_run_matches_reference():
    """Full 100-step N=10 run: final-state infidelity <= 1e-10 vs the reference."""
    from emulators_b200 import workloads as wl
    from emulators_b200.runner import run_workload

    g = golden("chain_n10")
    r = run_workload(wl.chain_n10())
    ref = g["final"]
    fid = abs(np.vdot(ref, r["final"])) ** 2 / (np.vdot(ref, ref).real * np.vdot(r["final"], r["final"]).real)
    assert 1 - fid <= 1e-10
    np.testing.assert_allclose(r["final"], ref, atol=1e-9, rtol=0)
    np.testing.assert_allclose(r["occupation"], g["occupation"], atol=1e-9)
    np.testing.assert_allclose(r["energy"], g["energy"], atol=1e-7)


def test_lattice_n20_run_matches_reference():
    """Full 300-step N=20 lattice run (Krylov dim <= 30) vs reference observables."""
    from emulators_b200 import workloads as wl
    from emulators_b200.runner import run_workload

    g = golden("lattice_n20")
    r = run_workload(wl.lattice_n20(), probes=len(g["probe_overlaps"]))
    np.testing.assert_allclose(r["occupation"], g["occupation"], atol=1e-8)
    np.testing.assert_allclose(r["energy"], g["energy"], atol=1e-6)
    np.testing.assert_allclose(r["probe_overlaps"], g["probe_overlaps"], atol=1e-7)
    assert abs(r["final_norm"] - float(g["final_norm"])) < 1e-9


def test_not_converged_raises_recursion_error():
    from emulators_b200 import EvolveStateVector

    c = cases(golden("krylov_step"))[-1]
    s = torch.as_tensor(c["state"]).to(DEV)
    with pytest.raises(RecursionError):
        EvolveStateVector(max_krylov_dim=3).apply(
            float(c["dt"]), *(torch.as_tensor(c[k]) for k in ("omegas", "deltas", "phis", "U")),
            s, 1e-12, None)


def test_in_place_and_unitarity_large():
    """N=22: the step is unitary to 1e-12 and forward(-dt) undoes forward(+dt)."""
    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian
    from emulators_b200 import workloads as wl
    from emulators_b200.krylov import fused_step

    n = 22
    U = torch.as_tensor(wl.interaction_matrix(wl.ladder(11, 5.5)))
    H = RydbergHamiltonian(torch.full((n,), 4.0), torch.full((n,), 3.0), torch.zeros(n), U, DEV)
    g = torch.Generator(device=DEV).manual_seed(5)
    psi = torch.randn(1 << n, dtype=torch.complex128, device=DEV, generator=g)
    psi /= torch.linalg.vector_norm(psi)
    out, info, st = fused_step(HamiltonianExpOperator(H, 0.005), psi, 1e-10, 1e-10, 100)
    assert st == 0 and abs(info.output_norm - 1.0) < 1e-12
    back, _, _ = fused_step(HamiltonianExpOperator(H, -0.005), out, 1e-10, 1e-10, 100)
    assert torch.linalg.vector_norm(back - psi).item() < 1e-9


def test_stale_iteration_hint_keeps_the_stopping_iteration():
    """A hint far above the needed iteration count (left by another problem of the same
    size) must not change the step: the device tests every iteration; the hint only
    delays the host's read of the decision."""
    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian, krylov
    from emulators_b200 import workloads as wl

    w = wl.lattice_n20()
    H = RydbergHamiltonian(*(torch.as_tensor(a) for a in (w.omega[0], w.delta[0], w.phi[0], w.U)),
                           DEV)
    psi = torch.zeros(1 << w.nqubits, dtype=torch.complex128, device=DEV)
    psi[0] = 1.0
    op = HamiltonianExpOperator(H, w.dt)
    outs = []
    for stale in (0, 60):
        krylov.release_workspaces()
        c = krylov._cache(psi.device, w.nqubits, 0)
        c.last_iters = stale
        out, info, st = krylov.fused_step(op, psi, w.tolerance, w.tolerance, 100)
        outs.append((out.cpu().numpy(), info.iterations))
    assert outs[0][1] == outs[1][1]
    np.testing.assert_array_equal(outs[0][0], outs[1][0])


def test_iteration_hint_matches_testing_every_iteration():
    """A chain whose iteration count moves between steps, run three ways: testing every
    iteration, with the previous step's count as the hint, and with a hint above the
    count at every step (the first test then already converges and the skipped
    iterations are tested in order): the same counts and the same bits."""
    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian, krylov
    from emulators_b200 import workloads as wl

    rng = np.random.default_rng(3)
    n, steps = 13, 12
    U = wl.interaction_matrix(wl.random_box(n, 27.0, 5.0, rng))
    om = rng.uniform(0, 2 * np.pi, steps)
    de = rng.uniform(-20, 20, steps)
    ph = rng.normal(size=(steps, n))
    runs = []
    for mode in ("every", "hint", "high"):
        krylov.use_iteration_hint = mode != "every"
        krylov.release_workspaces()
        s = torch.zeros(1 << n, dtype=torch.complex128, device=DEV)
        s[0] = 1.0
        its = []
        for k in range(steps):
            if mode == "high" and its:
                krylov._cache(s.device, n, 0).last_iters = its[-1] + 8
            H = RydbergHamiltonian(torch.full((n,), om[k]), torch.full((n,), de[k]),
                                   torch.as_tensor(ph[k]), torch.as_tensor(U), DEV)
            s, info, st = krylov.fused_step(HamiltonianExpOperator(H, 0.01), s, 1e-10, 1e-10, 100)
            its.append(info.iterations)
        runs.append((s.cpu().numpy(), its))
    krylov.use_iteration_hint = True
    for r in runs[1:]:
        assert r[1] == runs[0][1]
        np.testing.assert_array_equal(r[0], runs[0][0])


def test_generic_arnoldi_matches_reference():
    """krylov_exp_impl(is_hermitian=False) for arbitrary callables (reference
    krylov_exp.py:23-106; its test/emu_base/math/test_krylov_exp.py:194-218 case on a
    256 x 256 tensor, a vector case, and a rank-2 operator's happy breakdown): iteration
    counts, flags and results of the reference."""
    from emulators_b200 import krylov_exp, krylov_exp_impl

    g = golden("krylov_nonhermitian")
    for p in ("m_", "v_", "r_"):
        A = torch.as_tensor(g[p + "op"]).to(DEV)
        x = torch.as_tensor(g[p + "in"]).to(DEV)
        tol = float(g[p + "tol"])
        r = krylov_exp_impl(lambda y: A @ y, x.clone(), False, tol, tol, 100)
        assert r.iteration_count == int(g[p + "iters"]), p
        assert r.happy_breakdown == bool(g[p + "happy"]) and r.converged == bool(g[p + "converged"])
        ref = g[p + "result"]
        assert r.result.shape == x.shape
        np.testing.assert_allclose(r.result.cpu().numpy(), ref, atol=1e-12 * np.abs(ref).max(), rtol=0)
    # the reference test's own check: close to the dense exponential
    A = torch.as_tensor(g["m_op"]).to(DEV)
    X = torch.as_tensor(g["m_in"]).to(DEV)
    out = krylov_exp(lambda y: A @ y, X.clone(), 1e-6, 1e-6, is_hermitian=False, max_krylov_dim=100)
    assert torch.allclose(out, torch.linalg.matrix_exp(A) @ X)


@pytest.mark.parametrize("n,dtype", [(23, torch.complex128), (24, torch.complex64)])
def test_krylov_step_large_vs_oracle(oracle, n, dtype):
    """One time step of a register whose pass H takes two bit groups in one fused launch
    (8 super-tiles), from a random state with complex phases, against the oracle's
    Lanczos step: result and iteration count."""
    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian
    from emulators_b200 import workloads as wl
    from emulators_b200.krylov import fused_step

    rng = np.random.default_rng(40 + n)
    om, de, ph = rng.uniform(0, 2 * np.pi, n), rng.uniform(-20, 20, n), rng.normal(size=n)
    U = wl.interaction_matrix(wl.chain(n, 6.0))
    psi = torch.randn(1 << n, dtype=dtype, device=DEV)
    psi /= torch.linalg.vector_norm(psi)
    host = psi.cpu().to(torch.complex128).numpy()
    H = RydbergHamiltonian(*(torch.as_tensor(a) for a in (om, de, ph, U)), DEV)
    out, info, st = fused_step(HamiltonianExpOperator(H, 0.005), psi.clone(), 1e-10, 1e-10, 100)
    assert st == 0
    ref, _, rinfo = oracle.evolve_step(0.005, om, de, ph, U, host, 1e-10)
    tol = 1e-10 if dtype == torch.complex128 else 5e-6
    assert np.abs(out.cpu().to(torch.complex128).numpy() - ref).max() < tol
    if dtype == torch.complex128:
        assert info.iterations == rinfo.iteration_count


def test_fused_pass_h_kernel_vs_oracle(tmp_path):
    """The fused two-group pass H (EMUSV_FUSED_PASS_H=1, read once per process): the
    large-register steps of test_krylov_step_large_vs_oracle in a child process with the
    switch on."""
    import os
    import subprocess
    import sys

    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, EMUSV_FUSED_PASS_H="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
                        os.path.join(repo, "tests", "test_gpu_krylov.py"), "-k", "large_vs_oracle"],
                       env=env, cwd=repo, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "2 passed" in r.stdout
