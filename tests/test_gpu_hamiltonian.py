"""GPU parity of the fused H*psi, diagonal and observables against the reference fixtures
and the oracle (tolerances written per test)."""

import numpy as np
import pytest
import torch

from conftest import cases, golden

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _ham(c):
    from emulators_b200 import RydbergHamiltonian

    return RydbergHamiltonian(torch.as_tensor(c["omegas"]), torch.as_tensor(c["deltas"]),
                              torch.as_tensor(c["phis"]), torch.as_tensor(c["U"]), DEV)


def test_hpsi_c128_matches_reference_fixtures():
    # reference test_hamiltonian.py uses atol=1e-12 on O(1) values; scale for large |H psi|
    for c in cases(golden("hamiltonian")):
        H = _ham(c)
        assert H.complex == bool(c["complex"])
        psi = torch.as_tensor(c["state"]).to(DEV)
        out = (H * psi).cpu().numpy()
        tol = 1e-12 * max(1.0, np.abs(c["hpsi"]).max())
        np.testing.assert_allclose(out, c["hpsi"], atol=tol, rtol=0)
        np.testing.assert_allclose(H.diag.cpu().numpy(), c["diag"], atol=1e-12 * max(1, np.abs(c["diag"]).max()), rtol=0)


def test_hpsi_c64_matches_reference_fixtures():
    # complex64 storage: relative error bound 1e-6 of the largest amplitude
    for c in cases(golden("hamiltonian")):
        H = _ham(c)
        psi = torch.as_tensor(c["state"]).to(DEV, torch.complex64)
        out = (H * psi).cpu().numpy()
        np.testing.assert_allclose(out, c["hpsi"], atol=1e-6 * np.abs(c["hpsi"]).max(), rtol=0)


C64, C128 = torch.complex64, torch.complex128


@pytest.mark.parametrize("n,phase,dtype", [
    # every layout of the two-pass kernel: single pass L with cluster sizes 1, 2, 4 (c64)
    # and 1, 2, 4, 8 (c128), pass H with 1..11 group bits, and the global fallback bits
    (12, True, C128), (13, False, C64), (13, True, C128), (14, True, C64), (14, False, C128),
    (15, False, C64), (15, True, C128), (16, True, C64), (16, False, C128), (17, False, C64),
    (18, True, C64), (20, True, C128), (21, False, C64), (23, True, C64), (24, False, C128),
    (26, False, C64), (26, True, C128), (27, False, C128)])
def test_hpsi_large_registers_vs_oracle(oracle, n, phase, dtype):
    """H*psi of every kernel layout against the oracle (c128: 1e-13, c64: 1e-6 relative)."""
    from emulators_b200 import RydbergHamiltonian
    from emulators_b200 import workloads as wl

    rng = np.random.default_rng(n)
    om = rng.uniform(0, 2 * np.pi, n)
    de = rng.uniform(-20, 20, n)
    ph = rng.normal(size=n) if phase else np.zeros(n)
    U = wl.interaction_matrix(wl.square_lattice(2, n // 2, 5.5) if n % 2 == 0 else wl.chain(n, 5.0))
    psi = (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)) / np.sqrt(2 << n)
    ref = oracle.Hamiltonian(om, de, ph, U).apply(psi)
    H = RydbergHamiltonian(torch.as_tensor(om), torch.as_tensor(de), torch.as_tensor(ph),
                           torch.as_tensor(U), DEV)
    out = (H * torch.as_tensor(psi).to(DEV, dtype)).cpu().numpy()
    scale = np.abs(ref).max()
    tol = 1e-13 if dtype == torch.complex128 else 1e-6
    np.testing.assert_allclose(out, ref, atol=tol * scale, rtol=0)


def test_observables_match_reference_fixtures():
    from emulators_b200 import StateVector
    from emulators_b200.observables import (correlation_matrix_sv_impl,
                                            energy_second_moment_sv_impl, energy_variance_sv_impl,
                                            qubit_occupation_sv_impl)

    for c in cases(golden("observables")):
        st = StateVector(torch.as_tensor(c["state"]))
        H = _ham(c)
        np.testing.assert_allclose(qubit_occupation_sv_impl(state=st).numpy(), c["occupation"], atol=1e-14)
        np.testing.assert_allclose(correlation_matrix_sv_impl(state=st).numpy(), c["correlation"], atol=1e-14)
        assert abs(H.expect(st).item() - float(c["energy"])) < 1e-12
        assert abs(energy_variance_sv_impl(state=st, hamiltonian=H).item() - float(c["variance"])) < 1e-10
        assert abs(energy_second_moment_sv_impl(state=st, hamiltonian=H).item()
                   - float(c["second_moment"])) < 1e-10


@pytest.mark.parametrize("n,dtype,phase", [(12, torch.complex128, True), (16, torch.complex64, True),
                                           (22, torch.complex128, False), (24, torch.complex64, True),
                                           (26, torch.complex64, False)])
def test_energy_moments_vs_oracle(oracle, n, dtype, phase):
    """Energy, variance and second moment (hamiltonian.py:164-172,
    custom_callback_implementations.py:131-185) through the streaming passes (one and two
    pass H kernels, real and complex drives) against the oracle's H psi of the same state."""
    from emulators_b200 import RydbergHamiltonian, StateVector
    from emulators_b200 import workloads as wl
    from emulators_b200.observables import energy_second_moment_sv_impl, energy_variance_sv_impl

    rng = np.random.default_rng(300 + n)
    om, de = rng.uniform(0, 2 * np.pi, n), rng.uniform(-20, 20, n)
    ph = rng.normal(size=n) if phase else np.zeros(n)
    U = wl.interaction_matrix(wl.ladder(n // 2, 5.5))
    t = torch.randn(1 << n, dtype=dtype, device=DEV)
    t /= torch.linalg.vector_norm(t)
    H = RydbergHamiltonian(*(torch.as_tensor(a) for a in (om, de, ph, U)), DEV)
    st = StateVector(t)
    got = [H.expect(st).item(), energy_variance_sv_impl(state=st, hamiltonian=H).item(),
           energy_second_moment_sv_impl(state=st, hamiltonian=H).item()]
    host = t.cpu().to(torch.complex128).numpy()
    hpsi = oracle.Hamiltonian(om, de, ph, U).apply(host)
    e, m2 = np.vdot(host, hpsi).real, np.vdot(hpsi, hpsi).real
    want = [e, m2 - e * e, m2]
    rtol = 1e-12 if dtype == torch.complex128 else 2e-6
    for g, w in zip(got, want):
        assert abs(g - w) <= rtol * m2 ** 0.5 * max(1.0, m2 ** 0.5), (n, got, want)


@pytest.mark.parametrize("n,dtype", [(12, torch.complex128), (19, torch.complex64), (22, torch.complex128)])
def test_occupation_correlation_vs_oracle(oracle, n, dtype):
    rng = np.random.default_rng(100 + n)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    from emulators_b200.observables import correlation, occupation

    t = torch.as_tensor(psi).to(DEV, dtype)
    ref_psi = t.cpu().to(torch.complex128).numpy()
    tol = 1e-13 if dtype == torch.complex128 else 1e-12
    np.testing.assert_allclose(occupation(t).cpu().numpy(), oracle.occupation(ref_psi), atol=tol)
    np.testing.assert_allclose(correlation(t).cpu().numpy(), oracle.correlation(ref_psi), atol=tol)


def test_empty_and_edge_registers():
    """1- and 2-qubit registers (a single tile smaller than a warp) and zero drives."""
    from emulators_b200 import RydbergHamiltonian

    H = RydbergHamiltonian(torch.tensor([2.0]), torch.tensor([1.0]), torch.tensor([0.0]),
                           torch.zeros(1, 1), DEV)
    psi = torch.tensor([1.0, 2.0j], dtype=torch.complex128, device=DEV)
    # H = X - n : [[0,1],[1,-1]]
    np.testing.assert_allclose((H * psi).cpu().numpy(), [2.0j, 1.0 - 2.0j], atol=1e-15)
    H0 = RydbergHamiltonian(torch.zeros(2), torch.zeros(2), torch.zeros(2), torch.zeros(2, 2), DEV)
    psi = torch.randn(4, dtype=torch.complex128, device=DEV)
    assert torch.count_nonzero(H0 * psi).item() == 0


@pytest.mark.parametrize("n,dtype", [(5, torch.complex128), (13, torch.complex64),
                                     (25, torch.complex128)])
def test_sample_indices_vs_oracle(oracle, n, dtype):
    """emusv_sample equals the inverse-CDF draw of emu_sv/utils.py:40-49 (restated by the
    oracle) for the same uniforms, below and above the reference's 2^24 switch, including
    draws near 0 and 1 and zero-probability amplitudes."""
    from emulators_b200.state_vector import sample_indices

    rng = np.random.default_rng(n)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi[rng.random(1 << n) < 0.3] = 0.0  # zero-probability indices are never drawn
    psi /= np.linalg.norm(psi)
    u = np.concatenate([rng.random(4000), [0.0, 1e-300, 1 - 1e-16]])
    t = torch.as_tensor(psi).to(DEV, dtype)
    got = sample_indices(t, torch.as_tensor(u)).cpu().numpy()
    p = np.abs(t.cpu().numpy().astype(np.complex128)) ** 2
    want = oracle.sample_indices(p, u)
    # identical draws except where u * total falls within rounding of a cumulative boundary
    assert (got != want).sum() <= 2, (got != want).sum()
    assert np.all((p[got] > 0) | (got == (1 << n) - 1))  # the clamp may land anywhere
    with pytest.raises(RuntimeError):
        sample_indices(torch.zeros_like(t), torch.as_tensor(u[:4]))
