"""GPU parity of the Monte Carlo (noisy) path: H*psi with the noise term, the fused
Arnoldi step (emusv_arnoldi_step), expect_batch / apply (emusv_qubit_densities,
emusv_apply_1q) and whole EvolveMonteCarlo steps, against the reference's fixtures
(noisy.npz) and the oracle."""

import random

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _pref(g, p, k):
    q = f"{p}{k}_"
    return {key[len(q):]: g[key] for key in g.files if key.startswith(q)}


def _ham(c, noise):
    from emulators_b200 import RydbergHamiltonian

    return RydbergHamiltonian(*(torch.as_tensor(c[k]) for k in ("omegas", "deltas", "phis", "U")),
                              DEV, noise=torch.as_tensor(noise))


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-6)])
def test_noisy_hpsi_matches_reference(dtype, tol):
    """n = 3..13: the single-pass kernel and (n = 13; complex128 from n = 11) the
    multi-pass kernels with the noise diagonal in pass L."""
    g = golden("noisy")
    for k in range(int(g["hcount"])):
        c = _pref(g, "h", k)
        H = _ham(c, g["noise"])
        out = (H * torch.as_tensor(c["psi"]).to(DEV, dtype)).cpu().numpy()
        ref = c["hpsi"]
        np.testing.assert_allclose(out, ref, atol=tol * np.abs(ref).max(), rtol=0)
        if dtype == torch.complex128:
            np.testing.assert_allclose(H.diag.cpu().numpy(), c["diag"], atol=1e-12, rtol=0)


@pytest.mark.parametrize("n,dtype", [(16, torch.complex64), (17, torch.complex128),
                                     (22, torch.complex64), (24, torch.complex128)])
def test_noisy_hpsi_large_vs_oracle(oracle, n, dtype):
    """Every pass layout (one and two H passes) against the oracle."""
    from emulators_b200 import RydbergHamiltonian
    from emulators_b200 import workloads as wl

    g = golden("noisy")
    rng = np.random.default_rng(n)
    om, de, ph = rng.uniform(0, 6, n), rng.uniform(-20, 20, n), rng.normal(size=n)
    U = wl.interaction_matrix(wl.chain(n, 6.0))
    psi = (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)) / np.sqrt(2 << n)
    ref = oracle.Hamiltonian(om, de, ph, U, noise=g["noise"]).apply(psi)
    H = RydbergHamiltonian(*(torch.as_tensor(a) for a in (om, de, ph, U)), DEV,
                           noise=torch.as_tensor(g["noise"]))
    out = (H * torch.as_tensor(psi).to(DEV, dtype)).cpu().numpy()
    tol = 1e-12 if dtype == torch.complex128 else 1e-6
    np.testing.assert_allclose(out, ref, atol=tol * np.abs(ref).max(), rtol=0)


def _arnoldi(c, noise, dtype, hint=True):
    from emulators_b200 import krylov
    from emulators_b200.krylov import HamiltonianExpOperator, fused_arnoldi_step

    krylov.use_iteration_hint = hint
    try:
        H = _ham(c, noise)
        s = torch.as_tensor(c["state"]).to(DEV, dtype)
        return fused_arnoldi_step(HamiltonianExpOperator(H, float(c["dt"])), s, 1e-10, 1e-10, 100)
    finally:
        krylov.use_iteration_hint = True


def test_arnoldi_matches_reference():
    """krylov_exp(is_hermitian=False) cases: same iteration counts and happy flags, results
    within 1e-12 (complex128) / 2e-6 (complex64)."""
    g = golden("noisy")
    for k in range(int(g["acount"])):
        c = _pref(g, "a", k)
        out, info, st = _arnoldi(c, g["noise"], torch.complex128, hint=False)
        assert st == 0
        assert info.iterations == int(c["iters"]) and bool(info.happy_breakdown) == bool(c["happy"])
        np.testing.assert_allclose(out.cpu().numpy(), c["result"], atol=1e-12, rtol=0)
        out64, _, st64 = _arnoldi(c, g["noise"], torch.complex64, hint=False)
        assert st64 == 0
        np.testing.assert_allclose(out64.cpu().numpy(), c["result"], atol=2e-6, rtol=0)


def test_arnoldi_hint_and_large_register(oracle):
    """N=16: the iteration hint (first test three iterations before the previous count,
    forward scan when it already converges) gives the same bits as testing every
    iteration, and the oracle's iteration count and result."""
    from emulators_b200 import krylov
    from emulators_b200 import workloads as wl

    g = golden("noisy")
    n, dt = 16, 0.02
    rng = np.random.default_rng(5)
    om, de, ph = np.full(n, 5.0), rng.uniform(-10, 10, n), np.zeros(n)
    U = wl.interaction_matrix(wl.ladder(n // 2, 6.0))
    s0 = np.zeros(1 << n, dtype=np.complex128)
    s0[0] = 1.0
    H = oracle.Hamiltonian(om, de, ph, U, noise=g["noise"])
    ref = s0
    for _ in range(3):
        r = oracle.krylov_exp_impl(lambda x: -1j * dt * H.apply(x), ref, False, 1e-10, 1e-10, 100)
        ref = r.result
    c = {"omegas": om, "deltas": de, "phis": ph, "U": U, "dt": dt}
    runs = []
    for hint in (False, True):
        krylov.release_workspaces()
        s = s0.copy()
        for _ in range(3):
            c["state"] = s
            out, info, st = _arnoldi(c, g["noise"], torch.complex128, hint=hint)
            assert st == 0
            s = out.cpu().numpy()
        runs.append((s, info.iterations))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1] == r.iteration_count
    np.testing.assert_allclose(runs[0][0], ref, atol=1e-11, rtol=0)


def test_expect_batch_and_apply_match_reference():
    from emulators_b200.algebra import apply, expect_batch

    g = golden("noisy")
    v = torch.as_tensor(g["alg_vec"]).to(DEV)
    np.testing.assert_allclose(expect_batch(v, torch.as_tensor(g["alg_ops"]), 2).cpu().numpy(),
                               g["alg_expect"], atol=1e-15)
    ops = [torch.as_tensor(g[f"L{k}"]) for k in range(int(g["nops"]))]
    agg = torch.stack([L.mH @ L for L in ops])
    v6 = torch.as_tensor(g["alg_v6"]).to(DEV)
    np.testing.assert_allclose(expect_batch(v6, agg, 6).cpu().numpy(), g["alg_expect6"], atol=1e-12)
    for q in range(6):
        np.testing.assert_allclose(apply(v6, q, ops[q % len(ops)]).cpu().numpy(),
                                   g[f"alg_apply6_{q}"], atol=1e-14)
    for dt in (torch.complex64,):
        got = expect_batch(v6.to(dt), agg, 6).cpu().numpy()
        np.testing.assert_allclose(got, g["alg_expect6"], atol=1e-5 * np.abs(g["alg_expect6"]).max())


def test_monte_carlo_steps_match_reference():
    """EvolveMonteCarlo (N=8, 40 steps, 18-19 quantum jumps per seed) with the reference's
    seeded draws: every jump threshold and the states every 10 steps."""
    from emulators_b200.time_evolution import EvolveMonteCarlo

    g = golden("noisy")
    n, dt, nsteps = int(g["mc_n"]), float(g["mc_dt"]), int(g["mc_nsteps"])
    ops = [torch.as_tensor(g[f"mcL{k}"]) for k in range(int(g["mc_nops"]))]
    U = torch.as_tensor(g["mc_U"])
    for seed in (11, 12):
        random.seed(seed)
        stepper = EvolveMonteCarlo(100)
        st = torch.zeros(1 << n, dtype=torch.complex128, device=DEV)
        st[0] = 1.0
        thr, states = [stepper.jump_threshold], []
        for k in range(nsteps):
            om = torch.full((n,), 2 * np.pi * (0.5 + 0.5 * np.sin(0.3 * k)), dtype=torch.float64)
            de = torch.full((n,), -4.0 + 0.2 * k, dtype=torch.float64)
            st, _ = stepper.apply(dt, om, de, torch.zeros(n, dtype=torch.float64), U, st, 1e-10, ops)
            thr.append(stepper.jump_threshold)
            if (k + 1) % 10 == 0:
                states.append(st.cpu().numpy())
        np.testing.assert_allclose(thr, g[f"mc{seed}_thresholds"], rtol=1e-10, atol=0)
        np.testing.assert_allclose(np.stack(states), g[f"mc{seed}_states"], atol=1e-9, rtol=0)


def test_backend_runs_monte_carlo_solver():
    """SVBackendImpl picks the Monte Carlo stepper for Lindblad operators with
    solver='montecarlo' and the density-matrix stepper with solver='lindblad'
    (sv_backend_impl.py:82-95); the Monte Carlo state's norm stays <= 1."""
    from emulators_b200 import workloads as wl
    from emulators_b200.sv_backend import SequenceData, SVBackendImpl, SVConfig
    from emulators_b200.time_evolution import EvolveMonteCarlo

    g = golden("noisy")
    w = wl.chain_n10()
    data = SequenceData.from_workload(w)
    data.lindblad_ops = [torch.as_tensor(g[f"L{k}"]) for k in range(int(g["nops"]))]
    random.seed(3)
    impl = SVBackendImpl(SVConfig(solver="montecarlo"), data)
    assert isinstance(impl.stepper, EvolveMonteCarlo)
    for k in range(10):
        impl.step(k)
    nrm = float(torch.linalg.vector_norm(impl.state.data))
    assert 0.0 < nrm <= 1.0 + 1e-12
    from emulators_b200.time_evolution import EvolveDensityMatrix

    assert isinstance(SVBackendImpl(SVConfig(solver="lindblad"), data).stepper, EvolveDensityMatrix)
