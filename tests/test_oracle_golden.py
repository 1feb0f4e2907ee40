"""Pin the oracle (oracle/oracle.py + oracle/emusv_oracle.c) against fixtures produced by
running the reference emu-sv code itself (tests/golden/make_golden.py).  CPU only."""

import numpy as np
import pytest

from conftest import cases, golden


def test_hamiltonian_matches_reference(oracle):
    # reference test/emu_sv/test_hamiltonian.py:20-85 cases (atol 1e-12) plus larger registers
    for c in cases(golden("hamiltonian")):
        H = oracle.Hamiltonian(c["omegas"], c["deltas"], c["phis"], c["U"])
        assert H.complex == bool(c["complex"])
        np.testing.assert_allclose(H.diag, c["diag"].real, atol=1e-12, rtol=0)
        np.testing.assert_allclose(H.apply(c["state"]), c["hpsi"], atol=1e-12 * max(1.0, np.abs(c["hpsi"]).max()), rtol=0)


def test_krylov_step_matches_reference(oracle):
    # test/emu_sv/test_time_evolution.py:58-76 (atol = tolerance) and identical iteration counts
    for c in cases(golden("krylov_step")):
        r, _, info = oracle.evolve_step(float(c["dt"]), c["omegas"], c["deltas"], c["phis"], c["U"],
                                        c["state"], float(c["tol"]))
        np.testing.assert_allclose(r, c["result"], atol=1e-13, rtol=0)
        np.testing.assert_allclose(r, c["dense"], atol=float(c["tol"]), rtol=0)
        assert info.iteration_count == int(c["iters"])
        assert info.happy_breakdown == bool(c["happy"])


def test_backward_matches_reference(oracle):
    # test/emu_sv/test_time_evolution.py:79-103 gradients, here vs the reference autograd itself
    for c in cases(golden("backward")):
        g = oracle.step_backward(float(c["dt"]), c["omegas"], c["deltas"], c["phis"], c["U"],
                                 c["state"], c["r"], float(c["tol"]))
        for got, name in zip(g, ["g_omegas", "g_deltas", "g_phis", "g_U", "g_state"]):
            ref = c[name]
            np.testing.assert_allclose(got, ref, atol=1e-12 * max(1.0, np.abs(ref).max()), rtol=0)


def test_double_krylov_matches_reference(oracle):
    # test/emu_base/math/test_double_krylov.py:31-87
    for c in cases(golden("double_krylov")):
        H = oracle.Hamiltonian(c["omegas"], c["deltas"], c["phis"], c["U"])
        Vs, dS, Vg = oracle.double_krylov(lambda x: -1j * H.apply(x), c["state"], c["grad"],
                                          float(c["tol"]), 100)
        assert len(Vs) == int(c["len_s"]) and len(Vg) == int(c["len_g"])
        dU = np.stack(Vs).T @ dS @ np.stack(Vg).conj()
        np.testing.assert_allclose(dU, c["dU"], atol=1e-13, rtol=0)


def test_observables_match_reference(oracle):
    for c in cases(golden("observables")):
        s = c["state"]
        H = oracle.Hamiltonian(c["omegas"], c["deltas"], c["phis"], c["U"])
        np.testing.assert_allclose(oracle.occupation(s), c["occupation"], atol=1e-14)
        np.testing.assert_allclose(oracle.correlation(s), c["correlation"], atol=1e-14)
        assert abs(H.expect(s) - float(c["energy"])) < 1e-12
        assert abs(oracle.energy_variance(H, s) - float(c["variance"])) < 1e-10
        assert abs(oracle.energy_second_moment(H, s) - float(c["second_moment"])) < 1e-10


def test_chain_n10_run_matches_reference(oracle):
    from emulators_b200 import workloads as wl

    g = golden("chain_n10")
    r = oracle.run_workload(wl.chain_n10())
    np.testing.assert_allclose(r["final"], g["final"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(r["occupation"], g["occupation"], atol=1e-11)
    np.testing.assert_allclose(r["energy"], g["energy"], atol=1e-9)
    assert list(r["steps_at"]) == list(g["steps_at"])


@pytest.mark.slow
def test_lattice_n20_prefix_matches_reference(oracle):
    """First 30 steps of the N=20 lattice workload vs the reference observables."""
    from emulators_b200 import workloads as wl

    g = golden("lattice_n20")
    r = oracle.run_workload(wl.lattice_n20(), nsteps=30)
    np.testing.assert_allclose(r["occupation"], g["occupation"][:3], atol=1e-10)
    np.testing.assert_allclose(r["energy"], g["energy"][:3], atol=1e-7)


def test_neel_gradient_matches_reference(oracle):
    """Chained adjoint through 20 steps of the N=16 ring vs the reference autograd."""
    from emulators_b200 import workloads as wl

    g = golden("ring_n16_grad")
    gw = wl.ring_n16_grad()
    nseg = int(g["nseg"])
    for p in range(int(g["sets"])):
        loss, go, gd, occ = oracle.neel_loss_and_grad(gw, p, nseg=nseg)
        assert abs(loss - float(g[f"p{p}_loss"])) < 1e-12
        np.testing.assert_allclose(go, g[f"p{p}_g_omega"], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(gd, g[f"p{p}_g_delta"], rtol=1e-9, atol=1e-12)


def test_oracle_happy_breakdown_and_identity(oracle):
    """test/emu_base/math/test_krylov_exp.py:71-131 cases on the oracle's generic Lanczos."""
    import scipy.linalg

    m = np.diag([1.0, 2.0, 3.0, 3.0, 3.0]).astype(np.complex128)
    v = np.ones(5, dtype=np.complex128) / np.sqrt(5)
    r = oracle.krylov_exp_impl(lambda x: m @ x, v, True, 1e-6, 1e-12, 80)
    assert r.happy_breakdown and r.converged and r.iteration_count == 3
    np.testing.assert_allclose(r.result, scipy.linalg.expm(m) @ v, atol=1e-12)
    eye = np.eye(300, dtype=np.complex128)
    v = np.arange(300).astype(np.complex128)
    r = oracle.krylov_exp_impl(lambda x: eye @ x, v, True, 1e-6, 1e-12, 80)
    assert r.happy_breakdown and r.iteration_count == 1
    np.testing.assert_allclose(r.result, np.e * v, atol=1e-9)


def test_oracle_arnoldi_for_callables(oracle):
    """The oracle's krylov_exp_impl(is_hermitian=False) on the reference's fixtures of the
    Arnoldi branch for arbitrary operators (krylov_nonhermitian.npz, including the
    reference's own test_krylov_with_matrix case on a 256 x 256 tensor)."""
    g = golden("krylov_nonhermitian")
    for p in ("m_", "v_", "r_"):
        A, x = g[p + "op"], g[p + "in"]
        shape = x.shape
        r = oracle.krylov_exp_impl(lambda y: (A @ y.reshape(shape)).reshape(-1), x.reshape(-1).copy(),
                                   False, float(g[p + "tol"]), float(g[p + "tol"]), 100)
        assert r.iteration_count == int(g[p + "iters"])
        assert r.happy_breakdown == bool(g[p + "happy"]) and r.converged == bool(g[p + "converged"])
        ref = g[p + "result"].reshape(-1)
        np.testing.assert_allclose(r.result, ref, atol=1e-12 * np.abs(ref).max())


def test_oracle_dark_qubits(oracle):
    """State-preparation errors (sv_backend_impl.py:162-184): the masks the reference applies
    and its 12-step chain on the masked data (dark_qubits.npz)."""
    g = golden("dark_qubits")
    bad = g["bad_atoms"].astype(bool)
    om, de, ph, U = (g[k].copy() for k in ("omega", "delta", "phi", "U"))
    for a in (om, de, ph):
        a[:, bad] = 0.0
    U[bad, :] = 0.0
    U[:, bad] = 0.0
    for k, a in (("omega", om), ("delta", de), ("phi", ph), ("U", U)):
        np.testing.assert_array_equal(a, g[k + "_masked"])
    s = np.zeros(1 << U.shape[0], dtype=np.complex128)
    s[0] = 1.0
    for k in range(om.shape[0]):
        s, _, _ = oracle.evolve_step(float(g["dt"]), om[k], de[k], ph[k], U, s, 1e-10)
    np.testing.assert_allclose(s, g["final"], atol=1e-11)
