"""GPU parity of the adjoint step (emulators_b200.adjoint, C ABI emusv_adjoint_step)
against the reference's gradients (torch.py:223-378, double_krylov.py:5-113), the oracle
and central finite differences."""

import numpy as np
import pytest
import torch

from conftest import cases, golden

pytestmark = pytest.mark.gpu
DEV = "cuda"
NAMES = ["g_omegas", "g_deltas", "g_phis", "g_U", "g_state"]


def _grads_through_autograd(c, dtype=torch.complex128):
    """Re<r|exp(-i dt H) s> differentiated as test_time_evolution.py:79-103 does."""
    from emulators_b200 import DifferentiableStateVectorEvolution as DSE

    params = [torch.tensor(c[nm], device=DEV, requires_grad=True)
              for nm in ("omegas", "deltas", "phis", "U")]
    s_in = torch.tensor(c["state"], device=DEV).to(dtype).requires_grad_(True)
    r = torch.tensor(c["r"], device=DEV).to(dtype)
    so, _ = DSE.apply(float(c["dt"]), *params, s_in, float(c["tol"]), 100)
    scalar = torch.vdot(r, so).real
    return [g.detach().cpu().to(torch.complex128 if g.is_complex() else torch.float64).numpy()
            for g in torch.autograd.grad(scalar, (*params, s_in))]


def test_backward_matches_reference():
    # test_time_evolution.py:79-103 bar: allclose(rtol=tol) (torch's default atol 1e-8);
    # here against the reference's own gradients, plus a tighter absolute check.
    for c in cases(golden("backward")):
        tol = float(c["tol"])
        got = _grads_through_autograd(c)
        for g, nm in zip(got, NAMES):
            ref = c[nm]
            assert np.allclose(g, ref, rtol=tol, atol=1e-8), (nm, int(c["n"]), tol)
            scale = max(1.0, np.abs(ref).max())
            assert np.abs(g - ref).max() <= max(10 * tol, 1e-11) * scale, \
                (nm, int(c["n"]), tol, np.abs(g - ref).max())


def test_backward_complex64_state():
    """complex64 vectors with FP64 Lanczos scalars: gradients within 1e-5 relative."""
    for c in cases(golden("backward")):
        if float(c["tol"]) != 1e-8:
            continue
        got = _grads_through_autograd(c, torch.complex64)
        for g, nm in zip(got, NAMES):
            ref = c[nm]
            err = np.abs(g - ref).max() / max(1.0, np.abs(ref).max())
            assert err < 1e-5, (nm, int(c["n"]), err)


def _dense_flip(n, i, alpha):
    """Dense alpha sigma+_i + conj(alpha) sigma-_i (qubit i = bit n-1-i)."""
    D = 1 << n
    p = n - 1 - i
    A = np.zeros((D, D), dtype=np.complex128)
    for x in range(D):
        y = x ^ (1 << p)
        A[x, y] = alpha if (x >> p) & 1 else np.conj(alpha)
    return A


def _grads_from_frechet(c):
    """Re(-i dt Tr(dH/dtheta dU)) from the reference's Frechet derivative dU
    (torch.py:324-353 with dU = Vs^T dS Vg*, dt = 1)."""
    n = int(c["n"])
    dU = c["dU"]
    D = 1 << n
    x = np.arange(D)
    bits = [(x >> (n - 1 - i)) & 1 for i in range(n)]
    om, ph = c["omegas"], c["phis"]
    g_om = np.array([(-1j * np.trace(_dense_flip(n, i, 0.5 * np.exp(1j * ph[i])) @ dU)).real
                     for i in range(n)])
    g_ph = np.array([(-1j * np.trace(_dense_flip(n, i, 0.5 * om[i] * np.exp(1j * (ph[i] + np.pi / 2)))
                                     @ dU)).real for i in range(n)])
    dd = np.diag(dU)
    g_de = np.array([(-1j * np.sum(-bits[i] * dd)).real for i in range(n)])
    g_U = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1, n):
            g_U[i, j] = (-1j * np.sum(bits[i] * bits[j] * dd)).real
    return g_om, g_de, g_ph, g_U


def test_double_krylov_matches_reference():
    # test_double_krylov.py:31-87: the derivative along |state><grad| to atol = tol; the GPU
    # path never forms dU, so it is compared through the traces the gradients take of it.
    from emulators_b200 import RydbergHamiltonian
    from emulators_b200.adjoint import parameter_gradients

    for c in cases(golden("double_krylov")):
        n, tol = int(c["n"]), float(c["tol"])
        ham = RydbergHamiltonian(*(torch.as_tensor(c[k]) for k in ("omegas", "deltas", "phis", "U")),
                                 device=DEV)
        s = torch.tensor(c["state"], device=DEV)
        g = torch.tensor(c["grad"], device=DEV)
        got = parameter_gradients(ham, 1.0, s, g, tol, 100)
        want = _grads_from_frechet(c)
        # |Tr(A dE)| <= ||A||_2 * sum|dE| <= ||A||_2 * D * ||dE||_max with ||A||_2 <= |Omega|
        for gv, wv, nm in zip(got, want, ["omega", "delta", "phi", "U"]):
            bound = 10 * tol * (1 << n) * max(1.0, np.abs(c["omegas"]).max())
            assert np.abs(gv - wv).max() <= bound, (nm, n, tol, np.abs(gv - wv).max())


def test_double_krylov_max_dim_plumbing():
    # test_double_krylov.py:73-87: a basis of L vectors took at least L - 1 iterations, so a
    # cap of L - 2 must raise RecursionError.
    from emulators_b200 import RydbergHamiltonian
    from emulators_b200.adjoint import parameter_gradients

    for c in cases(golden("double_krylov")):
        longest = max(int(c["len_s"]), int(c["len_g"]))
        ham = RydbergHamiltonian(*(torch.as_tensor(c[k]) for k in ("omegas", "deltas", "phis", "U")),
                                 device=DEV)
        s = torch.tensor(c["state"], device=DEV)
        g = torch.tensor(c["grad"], device=DEV)
        parameter_gradients(ham, 1.0, s, g, float(c["tol"]), longest)
        with pytest.raises(RecursionError):
            parameter_gradients(ham, 1.0, s, g, float(c["tol"]), longest - 2)


@pytest.mark.parametrize("n,dtype", [(12, torch.complex128), (18, torch.complex128),
                                     (18, torch.complex64), (20, torch.complex128)])
def test_adjoint_matches_oracle_large(oracle, n, dtype):
    """Registers that take every contraction variant (12, 16 < n <= 20 bits) and the
    pair-sum kernel with low bits per thread, against the oracle's adjoint."""
    from emulators_b200.adjoint import step_adjoint

    rng = np.random.default_rng(n)
    om, de, ph = rng.normal(size=n) * 3, rng.normal(size=n) * 5, rng.normal(size=n)
    U = np.triu(rng.uniform(0.5, 4.0, size=(n, n)), 1)
    s = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    s /= np.linalg.norm(s)
    # a gradient of the form a loss of the occupations produces: sum_i w_i x_i psi
    x = np.arange(1 << n)
    w = rng.normal(size=n)
    g = sum(w[i] * ((x >> (n - 1 - i)) & 1) for i in range(n)) * s
    dt, tol = 0.02, 1e-10
    ref = oracle.step_backward(dt, om, de, ph, U, s, g, tol)
    args = [torch.tensor(a, device=DEV) for a in (om, de, ph, U)]
    got = step_adjoint(dt, *args, torch.tensor(s, device=DEV).to(dtype),
                       torch.tensor(g, device=DEV).to(dtype), tol, 100, (True,) * 5)
    bound = 1e-9 if dtype == torch.complex128 else 1e-5
    for gv, rv, nm in zip(got, ref, NAMES):
        gv = gv.detach().cpu().to(torch.complex128 if gv.is_complex() else torch.float64).numpy()
        err = np.abs(gv - rv).max() / np.abs(rv).max()
        assert err < bound, (nm, n, dtype, err)


def test_zero_gradient_gives_zero():
    from emulators_b200.adjoint import step_adjoint

    n = 6
    args = [torch.ones(n, dtype=torch.float64, device=DEV) for _ in range(3)]
    U = torch.triu(torch.ones(n, n, dtype=torch.float64, device=DEV), 1)
    s = torch.zeros(1 << n, dtype=torch.complex128, device=DEV)
    s[0] = 1
    g = torch.zeros_like(s)
    # parameter gradients of a zero incoming gradient are zero (the reference's lanczos
    # would divide by the zero norm); the state gradient is not requested
    out = step_adjoint(0.01, *args, U, s, g, 1e-10, 100, (True,) * 4 + (False,))
    for t in out[:4]:
        assert torch.count_nonzero(t) == 0
    assert out[4] is None


def _neel_chain(gw, p, nseg, om=None, de=None, dtype=torch.complex128):
    """Loss and per-segment gradients through the autograd.Function chain, as the reference
    computes them (tests/golden/make_golden.py gen_ring_n16_grad)."""
    from emulators_b200 import DifferentiableStateVectorEvolution as DSE

    n = gw.nqubits
    om = torch.tensor(gw.omega_seg[p, :nseg] if om is None else om, device=DEV,
                      requires_grad=True)
    de = torch.tensor(gw.delta_seg[p, :nseg] if de is None else de, device=DEV,
                      requires_grad=True)
    U = torch.tensor(gw.U, device=DEV)
    zeros = torch.zeros(n, dtype=torch.float64, device=DEV)
    s = torch.zeros(1 << n, dtype=dtype, device=DEV)
    s[0] = 1.0
    for seg in range(nseg):
        for _ in range(gw.steps_per_segment):
            s, _ = DSE.apply(gw.dt, om[seg].expand(n), de[seg].expand(n), zeros, U, s,
                             gw.tolerance, 100)
    occ = torch.stack([torch.linalg.vector_norm(s.view(2**i, 2, -1)[:, 1]) ** 2
                       for i in range(n)])
    loss = torch.mean((occ.to(torch.float64) - torch.tensor(gw.target, device=DEV)) ** 2)
    go, gd = torch.autograd.grad(loss, (om, de))
    return float(loss.detach()), go.cpu().numpy(), gd.cpu().numpy()


def test_neel_gradient_matches_reference():
    from emulators_b200 import workloads as wl

    g = golden("ring_n16_grad")
    gw = wl.ring_n16_grad()
    nseg = int(g["nseg"])
    for p in range(int(g["sets"])):
        loss, go, gd = _neel_chain(gw, p, nseg)
        assert abs(loss - float(g[f"p{p}_loss"])) < 1e-11
        np.testing.assert_allclose(go, g[f"p{p}_g_omega"], rtol=1e-7, atol=1e-11)
        np.testing.assert_allclose(gd, g[f"p{p}_g_delta"], rtol=1e-7, atol=1e-11)


def test_neel_gradient_central_differences():
    """dL/dOmega_seg and dL/ddelta_seg vs central differences, h = 1e-4."""
    from emulators_b200 import workloads as wl

    gw = wl.ring_n16_grad()
    nseg, p, h = 2, 3, 1e-4
    om0, de0 = gw.omega_seg[p, :nseg].copy(), gw.delta_seg[p, :nseg].copy()
    _, go, gd = _neel_chain(gw, p, nseg)
    for which, base, grad in (("om", om0, go), ("de", de0, gd)):
        for k in range(nseg):
            plus, minus = base.copy(), base.copy()
            plus[k] += h
            minus[k] -= h
            kw_p = {"om": plus} if which == "om" else {"de": plus}
            kw_m = {"om": minus} if which == "om" else {"de": minus}
            lp = _neel_chain(gw, p, nseg, **kw_p)[0]
            lm = _neel_chain(gw, p, nseg, **kw_m)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - grad[k]) <= 1e-5 * max(abs(grad[k]), 1e-3), (which, k, fd, grad[k])
