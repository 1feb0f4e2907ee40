"""The Lindblad density-matrix path: the oracle's dense restatement of RydbergLindbladian
and EvolveDensityMatrix against fixtures made by running the reference (lindblad.npz), on
the CPU; the GPU kernels (emusv_lindblad_apply, emusv_lindblad_arnoldi_step,
emusv_dm_energy, emusv_dm_diagonal_amplitudes) against the same fixtures and the oracle."""

import numpy as np
import pytest
import torch

from conftest import cases, golden


def _ops(g):
    return [g[f"L{k}"] for k in range(int(g["nops"]))]


def test_oracle_lindbladian_matches_reference(oracle):
    g = golden("lindblad")
    for c in cases(g):
        got = oracle.lindbladian_apply(c["omegas"], c["deltas"], c["phis"], c["U"], _ops(g), c["rho"])
        np.testing.assert_allclose(got, c["Lrho"], atol=1e-12 * np.abs(c["Lrho"]).max(), rtol=0)


def test_oracle_density_matrix_evolution_matches_reference(oracle):
    g = golden("lindblad")
    n, dt = int(g["ev_n"]), float(g["ev_dt"])
    rho = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    rho[0, 0] = 1.0
    snaps = []
    for k in range(int(g["ev_nsteps"])):
        om = np.full(n, 2 * np.pi * (0.6 + 0.4 * np.sin(0.5 * k)))
        de = np.full(n, -3.0 + 0.5 * k)
        ph = np.full(n, 0.1 * k)
        rho, _ = oracle.lindblad_step(dt, om, de, ph, g["ev_U"], _ops(g), rho, 1e-10)
        if (k + 1) % 4 == 0:
            snaps.append(rho)
    np.testing.assert_allclose(np.stack(snaps), g["ev_states"], atol=1e-11, rtol=0)


def _lind(c, g):
    from emulators_b200.density_matrix import RydbergLindbladian

    return RydbergLindbladian(*(torch.as_tensor(c[k]) for k in ("omegas", "deltas", "phis")),
                              [torch.as_tensor(L) for L in _ops(g)], torch.as_tensor(c["U"]), "cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 2e-6)])
def test_gpu_lindbladian_matches_reference(dtype, tol):
    from emulators_b200.density_matrix import DensityMatrix

    g = golden("lindblad")
    for c in cases(g):
        L = _lind(c, g)
        rho = torch.as_tensor(c["rho"]).to("cuda", dtype)
        got = (L @ rho).cpu().numpy()
        np.testing.assert_allclose(got, c["Lrho"], atol=tol * np.abs(c["Lrho"]).max(), rtol=0)
        if dtype == torch.complex128:
            assert abs(float(L.expect(DensityMatrix(rho))) - float(c["energy"])) < 1e-11


@pytest.mark.gpu
def test_gpu_lindbladian_larger_register_vs_oracle(oracle):
    """N=7 (14-bit vector: the multi-pass kernels on both indices) against the oracle."""
    from emulators_b200 import workloads as wl
    from emulators_b200.density_matrix import RydbergLindbladian

    g = golden("lindblad")
    n = 7
    rng = np.random.default_rng(7)
    om, de, ph = rng.uniform(0, 6, n), rng.uniform(-10, 10, n), rng.normal(size=n)
    U = wl.interaction_matrix(wl.chain(n, 6.0))
    a = rng.normal(size=(1 << n, 4)) + 1j * rng.normal(size=(1 << n, 4))
    rho = a @ a.conj().T
    rho /= np.trace(rho).real
    ref = oracle.lindbladian_apply(om, de, ph, U, _ops(g), rho)
    L = RydbergLindbladian(*(torch.as_tensor(x) for x in (om, de, ph)),
                           [torch.as_tensor(x) for x in _ops(g)], torch.as_tensor(U), "cuda")
    got = (L @ torch.as_tensor(rho).cuda()).cpu().numpy()
    np.testing.assert_allclose(got, ref, atol=1e-12 * np.abs(ref).max(), rtol=0)


@pytest.mark.gpu
def test_gpu_density_matrix_evolution_and_observables():
    """EvolveDensityMatrix (12 steps of 50 ns, N=4) and the density-matrix observables of
    the final state against the reference's values."""
    from emulators_b200.density_matrix import (DensityMatrix, correlation_matrix_sv_den_mat_impl,
                                               energy_second_moment_den_mat_impl,
                                               energy_variance_sv_den_mat_impl,
                                               qubit_occupation_sv_den_mat_impl)
    from emulators_b200.time_evolution import EvolveDensityMatrix

    g = golden("lindblad")
    n, dt = int(g["ev_n"]), float(g["ev_dt"])
    ops = [torch.as_tensor(L) for L in _ops(g)]
    stepper = EvolveDensityMatrix(100)
    rho = DensityMatrix.make(n).data
    snaps = []
    for k in range(int(g["ev_nsteps"])):
        om = torch.full((n,), 2 * np.pi * (0.6 + 0.4 * np.sin(0.5 * k)), dtype=torch.float64)
        de = torch.full((n,), -3.0 + 0.5 * k, dtype=torch.float64)
        ph = torch.full((n,), 0.1 * k, dtype=torch.float64)
        rho, ham = stepper.apply(dt, om, de, ph, torch.as_tensor(g["ev_U"]), rho, 1e-10, ops)
        if (k + 1) % 4 == 0:
            snaps.append(rho.cpu().numpy())
    np.testing.assert_allclose(np.stack(snaps), g["ev_states"], atol=1e-11, rtol=0)
    st = DensityMatrix(rho)
    assert abs(float(st.norm()) - 1.0) < 1e-10
    np.testing.assert_allclose(qubit_occupation_sv_den_mat_impl(state=st).numpy(), g["ev_occupation"],
                               atol=1e-12)
    np.testing.assert_allclose(correlation_matrix_sv_den_mat_impl(state=st).numpy(),
                               g["ev_correlation"], atol=1e-12)
    assert abs(float(ham.expect(st)) - float(g["ev_energy"])) < 1e-10
    assert abs(float(energy_variance_sv_den_mat_impl(state=st, hamiltonian=ham))
               - float(g["ev_variance"])) < 1e-8
    assert abs(float(energy_second_moment_den_mat_impl(state=st, hamiltonian=ham))
               - float(g["ev_second_moment"])) < 1e-8


@pytest.mark.gpu
def test_gpu_backend_density_matrix_solver():
    """SVBackendImpl picks the density-matrix stepper for Lindblad operators with the
    default solver and no stochastic noise (sv_backend_impl.py:85-93); the trace stays 1."""
    from emulators_b200 import workloads as wl
    from emulators_b200.density_matrix import DensityMatrix
    from emulators_b200.sv_backend import Energy, Occupation, SequenceData, SVBackendImpl, SVConfig
    from emulators_b200.time_evolution import EvolveDensityMatrix

    g = golden("lindblad")
    w = wl.chain_n10()
    n = 5
    data = SequenceData(torch.as_tensor(w.omega[:20, :n]), torch.as_tensor(w.delta[:20, :n]),
                        torch.as_tensor(w.phi[:20, :n]), [10.0 * k for k in range(21)],
                        torch.as_tensor(w.U[:n, :n]), tuple(f"q{i}" for i in range(n)))
    data.lindblad_ops = [torch.as_tensor(L) for L in _ops(g)]
    impl = SVBackendImpl(SVConfig(observables=[Occupation(), Energy()]), data)
    assert isinstance(impl.stepper, EvolveDensityMatrix) and isinstance(impl.state, DensityMatrix)
    res = impl._run()
    assert abs(float(impl.state.norm()) - 1.0) < 1e-9
    occ = res.get("occupation")
    assert len(occ) == 21 and all((o >= -1e-12).all() and (o <= 1 + 1e-12).all() for o in occ)
