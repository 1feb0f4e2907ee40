"""The Monte Carlo (noisy) path on the CPU: the oracle's noisy H*psi, Arnoldi exponential,
expect_batch / apply, Brent bracketing and whole EvolveMonteCarlo steps against fixtures
made by running the reference (tests/golden/make_golden.py, noisy.npz), and the package's
host-side pieces (Brent's root finder, the Lindblad operators and the noise term)."""

import random

import numpy as np
import torch

from conftest import golden


def _pref(g, p, k):
    q = f"{p}{k}_"
    return {key[len(q):]: g[key] for key in g.files if key.startswith(q)}


def test_noisy_hamiltonian_matches_reference(oracle):
    g = golden("noisy")
    for k in range(int(g["hcount"])):
        c = _pref(g, "h", k)
        H = oracle.Hamiltonian(c["omegas"], c["deltas"], c["phis"], c["U"], noise=g["noise"])
        ref = c["hpsi"]
        np.testing.assert_allclose(H.apply(c["psi"]), ref, atol=1e-12 * np.abs(ref).max(), rtol=0)
        np.testing.assert_allclose(H.diag + H.noise_diag(), c["diag"], atol=1e-12, rtol=0)


def test_arnoldi_matches_reference(oracle):
    g = golden("noisy")
    for k in range(int(g["acount"])):
        c = _pref(g, "a", k)
        H = oracle.Hamiltonian(c["omegas"], c["deltas"], c["phis"], c["U"], noise=g["noise"])
        dt = float(c["dt"])
        r = oracle.krylov_exp_impl(lambda x: -1j * dt * H.apply(x), c["state"], False, 1e-10,
                                   1e-10, 100)
        assert r.iteration_count == int(c["iters"]) and r.happy_breakdown == bool(c["happy"])
        np.testing.assert_allclose(r.result, c["result"], atol=1e-13, rtol=0)


def test_algebra_matches_reference(oracle):
    g = golden("noisy")
    np.testing.assert_allclose(oracle.expect_batch(g["alg_vec"], g["alg_ops"], 2), g["alg_expect"],
                               atol=1e-15)
    ops = [g[f"L{k}"] for k in range(int(g["nops"]))]
    agg = [L.conj().T @ L for L in ops]
    np.testing.assert_allclose(oracle.expect_batch(g["alg_v6"], agg, 6), g["alg_expect6"], atol=1e-12)
    for q in range(6):
        np.testing.assert_allclose(oracle.apply_1q(g["alg_v6"], q, ops[q % len(ops)]),
                                   g[f"alg_apply6_{q}"], atol=1e-14)
    # the reference's own test values (test/emu_sv/test_algebra.py:5-29)
    had = np.array([[1.0, -1.0], [1.0, 1.0]])
    vec = np.array([0.0, 0.0, 0.5, 1.0])
    np.testing.assert_allclose(oracle.apply_1q(vec, 0, had), [-0.5, -1.0, 0.5, 1.0])
    np.testing.assert_allclose(oracle.apply_1q(vec, 1, had), [0.0, 0.0, -0.5, 1.5])


def _brent_run(make, provide, nxt, conv):
    xs = []
    while not conv():
        x = nxt()
        xs.append(x)
        provide(x, (x + 3) * (x - 1) ** 2)
    return xs


def test_brent_matches_reference(oracle):
    """Same abscissae as the reference on (x+3)(x-1)^2 from [-4, 4/3] (its own test case,
    test/emu_base/math/test_brents_root_finding.py:44-53), for the oracle and the package."""
    from emulators_b200.brents_root_finding import BrentsRootFinder, find_root_brents

    g = golden("noisy")
    f = lambda x: (x + 3) * (x - 1) ** 2  # noqa: E731
    rf = BrentsRootFinder(start=-4.0, end=4 / 3.0, f_start=f(-4.0), f_end=f(4 / 3.0), epsilon=1e-6)
    xs = _brent_run(None, rf.provide_ordinate, rf.get_next_abscissa, lambda: rf.is_converged(1e-6))
    np.testing.assert_array_equal(xs, g["brent_x"])
    assert rf.current_guess == float(g["brent_root"])
    ob = oracle.Brent(-4.0, 4 / 3.0, f(-4.0), f(4 / 3.0), 1e-6)
    xs2 = _brent_run(None, ob.provide, ob.next, lambda: ob.converged(1e-6))
    np.testing.assert_array_equal(xs2, g["brent_x"])
    calls = []
    root = find_root_brents(lambda x: calls.append(x) or f(x), start=-4, end=4 / 3.0)
    assert abs(root + 3) < 1e-10 and len(calls) == 12  # the reference's expected call count


def test_monte_carlo_oracle_matches_reference(oracle):
    """Whole EvolveMonteCarlo steps (N=8, 40 steps, 18-19 jumps) with the same seeded draws
    of Python's random module: thresholds and states every 10 steps."""
    g = golden("noisy")
    n, dt, nsteps = int(g["mc_n"]), float(g["mc_dt"]), int(g["mc_nsteps"])
    ops = [g[f"mcL{k}"] for k in range(int(g["mc_nops"]))]
    for seed in (11, 12):
        rnd = random.Random(seed)
        thr = rnd.uniform(0.0, 1.0)
        st = np.zeros(1 << n, dtype=np.complex128)
        st[0] = 1.0
        thresholds, states = [thr], []
        for k in range(nsteps):
            om = np.full(n, 2 * np.pi * (0.5 + 0.5 * np.sin(0.3 * k)))
            de = np.full(n, -4.0 + 0.2 * k)
            st, thr, _ = oracle.monte_carlo_step(rnd, thr, dt, om, de, np.zeros(n), g["mc_U"], st,
                                                 ops, 1e-10)
            thresholds.append(thr)
            if (k + 1) % 10 == 0:
                states.append(st)
        np.testing.assert_allclose(thresholds, g[f"mc{seed}_thresholds"], rtol=1e-12, atol=0)
        np.testing.assert_allclose(np.stack(states), g[f"mc{seed}_states"], atol=1e-9, rtol=0)


def test_lindblad_operators_and_noise_term():
    """The package's get_lindblad_operators / compute_noise_from_lindbladians give the
    operators and noise term the fixtures were made with (the reference's own)."""
    from emulators_b200.jump_lindblad_operators import (compute_noise_from_lindbladians,
                                                        get_lindblad_operators)

    g = golden("noisy")

    class NM:
        noise_types = ("relaxation", "dephasing", "depolarizing")
        relaxation_rate = 0.9
        dephasing_rate = 0.6
        hyperfine_dephasing_rate = 0.0
        depolarizing_rate = 0.3

    ops = []
    for t in NM.noise_types:
        ops += get_lindblad_operators(noise_type=t, noise_model=NM)
    ops.append(torch.tensor([[0.1, 0.2 + 0.1j], [0.0, -0.3j]], dtype=torch.complex128))
    for k, L in enumerate(ops):
        np.testing.assert_allclose(L.numpy(), g[f"L{k}"], atol=1e-15)
    np.testing.assert_allclose(compute_noise_from_lindbladians(ops).numpy(), g["noise"], atol=1e-15)
