"""ORACLE -- test infrastructure only.

CPU restatement of the reference emu-sv time-evolution hot path, used as the checker by
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``.  The
product (``emulators_b200``) never imports this module.

The 2^N-sized arithmetic runs in ``emusv_oracle.c`` (OpenMP, float64) through ctypes;
the Lanczos control flow and the small matrix exponentials run here in numpy/scipy.
Every function cites the reference lines it restates.  Parity of this oracle with the
reference is pinned by fixtures produced by running the reference itself
(tests/golden/make_golden.py, checked in tests/test_oracle_golden.py).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np
import scipy.linalg
from threadpoolctl import threadpool_limits

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD, "libemusv_oracle.so")
SRC = os.path.join(HERE, "emusv_oracle.c")

_lib = None


def build(force: bool = False) -> str:
    """Compile emusv_oracle.c with gcc into oracle/_build/ (idempotent)."""
    os.makedirs(BUILD, exist_ok=True)
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-shared", "-fPIC",
                               "-o", LIB_PATH, SRC, "-lm"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        P, I, I64, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
        L.or_diag.argtypes = [I, P, P, P]
        L.or_hpsi.argtypes = [I, P, P, P, P]
        L.or_vdot.argtypes = [I64, P, P, P]
        L.or_norm2.argtypes = [I64, P]
        L.or_norm2.restype = D
        L.or_axpy.argtypes = [I64, D, D, P, P]
        L.or_scale.argtypes = [I64, D, D, P]
        L.or_combine.argtypes = [I64, I, P, P, P]
        L.or_occupation.argtypes = [I, P, P]
        L.or_correlation.argtypes = [I, P, P]
        L.or_grad_contract.argtypes = [I, I, P, P, P, P]
        L.or_set_threads.argtypes = [I]
        L.or_num_threads.restype = I
        _lib = L
    return _lib


def set_threads(t: int) -> None:
    lib().or_set_threads(int(t))


def num_threads() -> int:
    return lib().or_num_threads()


def expm(a: np.ndarray) -> np.ndarray:
    """Small dense exponential (Pade scaling and squaring), single-threaded: the matrices
    are at most (max_krylov_dim+2)^2 and BLAS threading only adds overhead."""
    with threadpool_limits(1):
        return scipy.linalg.expm(a)


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.complex128)


def _real(a) -> np.ndarray:
    a = np.asarray(a)
    return np.ascontiguousarray(a.real if np.iscomplexobj(a) else a, dtype=np.float64)


# ----------------------------------------------------------------------- vector helpers
def vdot(a: np.ndarray, b: np.ndarray) -> complex:
    r = np.zeros(2)
    lib().or_vdot(a.size, _p(a), _p(b), _p(r))
    return complex(r[0], r[1])


def norm(a: np.ndarray) -> float:
    return float(np.sqrt(lib().or_norm2(a.size, _p(a))))


def axpy(alpha: complex, x: np.ndarray, y: np.ndarray) -> None:
    lib().or_axpy(x.size, alpha.real, alpha.imag, _p(x), _p(y))


def combine(coef: np.ndarray, V: list[np.ndarray]) -> np.ndarray:
    """sum_k coef[k] V[k] (krylov_exp.py:88-90); large bases are accumulated vector by
    vector so no stacked copy of the basis is made."""
    c = _c128(coef)
    out = np.zeros(V[0].size, dtype=np.complex128)
    if V[0].size * len(V) <= (1 << 24):
        M = np.ascontiguousarray(np.stack(V))
        lib().or_combine(V[0].size, len(V), _p(c), _p(M), _p(out))
        return out
    for ck, vk in zip(c, V):
        axpy(complex(ck), vk, out)
    return out


# ----------------------------------------------------------------------- Hamiltonian
class Hamiltonian:
    """Matrix-free Rydberg Hamiltonian, restating emu_sv/hamiltonian.py:42-172.

    H = sum_j Omega_j/2 (cos phi_j X_j + sin phi_j Y_j) - sum_j delta_j n_j
        + sum_{i<j} U_ij n_i n_j
    """

    def __init__(self, omegas, deltas, phis, U, noise=None):
        self.n = len(omegas)
        self.omegas = _real(omegas) / 2.0  # hamiltonian.py:52
        self.deltas = _real(deltas)
        self.phis = _real(phis)
        self.U = _real(U).reshape(self.n, self.n)
        self.noise = None if noise is None else np.asarray(noise, dtype=np.complex128).reshape(2, 2)
        self.complex = bool(np.any(self.phis != 0.0)) or noise is not None  # hamiltonian.py:61
        up = self.omegas * np.exp(1j * self.phis)  # hamiltonian.py:62-64
        dn = np.conj(up)
        if self.noise is not None:  # hamiltonian.py:65-67
            up = up + self.noise[1, 0]
            dn = dn + self.noise[0, 1]
        self.coef = np.ascontiguousarray(
            np.stack([up.real, up.imag, dn.real, dn.imag], axis=1), dtype=np.float64)
        self._diag = None
        self._noise_diag = None

    @property
    def diag(self) -> np.ndarray:
        """hamiltonian.py:139-162 (real float64 here; the reference stores complex128)."""
        if self._diag is None:
            d = np.empty(1 << self.n, dtype=np.float64)
            lib().or_diag(self.n, _p(self.deltas), _p(np.ascontiguousarray(self.U)), _p(d))
            self._diag = d
        return self._diag

    def noise_diag(self) -> np.ndarray:
        """The noise part of the diagonal: noise[0,0] on every qubit in |g>, noise[1,1] on
        every qubit in |r> (hamiltonian.py:147-151)."""
        if self._noise_diag is None:
            x = np.arange(1 << self.n)
            pop = np.zeros(1 << self.n, dtype=np.int64)
            for p in range(self.n):
                pop += (x >> p) & 1
            self._noise_diag = (self.n - pop) * self.noise[0, 0] + pop * self.noise[1, 1]
        return self._noise_diag

    def apply(self, psi: np.ndarray) -> np.ndarray:
        """H * psi (hamiltonian.py:69-91)."""
        psi = _c128(psi)
        out = np.empty_like(psi)
        lib().or_hpsi(self.n, _p(self.coef), _p(self.diag), _p(psi), _p(out))
        if self.noise is not None:
            out += self.noise_diag() * psi
        return out

    __mul__ = apply

    def expect(self, psi: np.ndarray) -> float:
        """Re <psi|H|psi> (hamiltonian.py:164-172; the real part also with noise)."""
        return vdot(_c128(psi), self.apply(psi)).real


# ----------------------------------------------------------------------- Krylov
@dataclass
class KrylovResult:
    result: np.ndarray
    converged: bool
    happy_breakdown: bool
    iteration_count: int


def krylov_exp_impl(op, v: np.ndarray, is_hermitian: bool, exp_tolerance: float,
                    norm_tolerance: float, max_krylov_dim: int = 100) -> KrylovResult:
    """Lanczos/Arnoldi exp(op) v with the Expokit extended-T error estimate,
    restating emu_base/math/krylov_exp.py:23-106 (the input is not modified here)."""
    v = _c128(v).copy()
    initial_norm = norm(v)  # 43
    v /= initial_norm  # 44
    V = [v]
    T = np.zeros((max_krylov_dim + 2, max_krylov_dim + 2), dtype=np.complex128)  # 47
    expd = None
    for j in range(max_krylov_dim):  # 49
        w = _c128(op(V[-1]))  # 50
        n = norm(w)  # 52
        k_start = max(0, j - 1) if is_hermitian else 0  # 54
        for k in range(k_start, j + 1):  # 55-58
            ov = vdot(V[k], w)
            T[k, j] = ov
            axpy(-ov, V[k], w)
        n2 = norm(w)  # 60
        T[j + 1, j] = n2  # 61
        if n2 < norm_tolerance:  # 63-71 happy breakdown
            e = expm(T[: j + 1, : j + 1])
            return KrylovResult(initial_norm * combine(e[:, 0], V), True, True, j + 1)
        w /= n2  # 73
        V.append(w)
        T[j + 2, j + 1] = 1  # 77
        expd = expm(T[: j + 3, : j + 3])  # 78
        err1 = abs(expd[j + 1, 0])  # 81
        err2 = abs(expd[j + 2, 0] * n)  # 82
        err = err1 if err1 < err2 else (err1 * err2 / (err1 - err2))  # 84
        if err < exp_tolerance:  # 86-96
            return KrylovResult(initial_norm * combine(expd[: len(V), 0], V), True, False, j + 1)
    return KrylovResult(initial_norm * combine(expd[: len(V), 0], V), False, False,
                        max_krylov_dim)  # 98-106


def krylov_exp(op, v, exp_tolerance, norm_tolerance, is_hermitian=True, max_krylov_dim=100):
    """krylov_exp.py:109-131: raises RecursionError when not converged."""
    r = krylov_exp_impl(op, v, is_hermitian, exp_tolerance, norm_tolerance, max_krylov_dim)
    if not r.converged:
        raise RecursionError("exponentiation algorithm did not converge to precision in "
                             "allotted number of steps.")
    return r.result


def lanczos(op, v: np.ndarray, tolerance: float, max_krylov_dim: int):
    """emu_base/math/double_krylov.py:61-113."""
    v = _c128(v)
    V = [v / norm(v)]
    T = np.zeros((max_krylov_dim + 2, max_krylov_dim + 2), dtype=np.complex128)
    converged = False
    for j in range(max_krylov_dim):
        w = _c128(op(V[-1])).copy()
        n = norm(w)
        for k in range(max(0, j - 1), j + 1):
            ov = vdot(V[k], w)
            T[k, j] = ov
            axpy(-ov, V[k], w)
        n2 = norm(w)
        T[j + 1, j] = n2
        if n2 < tolerance:
            converged = True
            break
        V.append(w / n2)
        T[j + 2, j + 1] = 1
        expd = expm(T[: j + 3, : j + 3])
        err1 = abs(expd[j + 1, 0])
        err2 = abs(expd[j + 2, 0] * n)
        err = err1 if err1 < err2 else (err1 * err2 / (err1 - err2))
        if err < tolerance:
            converged = True
            break
    if not converged:
        raise RecursionError("Lanczos iteration did not converge to precision in allotted "
                             "number of steps.")
    size = len(V)
    return V, T[:size, :size].copy()


def double_krylov(op, state, grad, tolerance, max_krylov_dim):
    """emu_base/math/double_krylov.py:5-58: dU(op, |state><grad|) = Vs^T dS Vg*."""
    Vs, Ts = lanczos(op, state, tolerance, max_krylov_dim)
    Vg, Tg = lanczos(op, grad, tolerance, max_krylov_dim)
    ss = len(Vs)
    big = scipy.linalg.block_diag(Ts, Tg).astype(np.complex128)
    big[0, ss] = norm(_c128(state)) * norm(_c128(grad))
    dS = expm(big)[:ss, ss:]
    return Vs, dS, Vg


# ----------------------------------------------------------------------- time step
def evolve_step(dt, omegas, deltas, phis, U, state, tol, max_krylov_dim=100):
    """One step exp(-i dt H) psi (emu_sv/time_evolution/torch.py:143-172)."""
    H = Hamiltonian(omegas, deltas, phis, U)
    r = krylov_exp_impl(lambda x: -1j * dt * H.apply(x), state, True, tol, tol, max_krylov_dim)
    if not r.converged:
        raise RecursionError("exponentiation algorithm did not converge to precision in "
                             "allotted number of steps.")
    return r.result, H, r


def step_backward(dt, omegas, deltas, phis, U, state, grad_out, tol, max_krylov_dim=100,
                  needs=(True, True, True, True, True)):
    """Adjoint of one step, restating emu_sv/time_evolution/torch.py:223-378.

    Returns (g_omegas, g_deltas, g_phis, g_U, g_state); entries not requested are None.
    """
    H = Hamiltonian(omegas, deltas, phis, U)
    n = H.n
    om_full = _real(omegas)
    ph = _real(phis)
    g_om = g_de = g_ph = g_U = g_st = None
    if any(needs[:4]):
        op = lambda x: -1j * dt * H.apply(x)  # noqa: E731
        Vs, dS, Vg = double_krylov(op, state, grad_out, tol, max_krylov_dim)  # 314-316
        Vs_m = np.stack(Vs)
        Vg_m = np.ascontiguousarray(np.stack(Vg))
        e_l = np.ascontiguousarray(dS.T @ Vs_m)  # 322
        m = e_l.shape[0]
        S = np.zeros((n, n), dtype=np.complex128)
        F = np.zeros((n, 2), dtype=np.complex128)
        lib().or_grad_contract(n, m, _p(Vg_m), _p(e_l), _p(S), _p(F))
        pre = -1j * dt
        if needs[0]:  # 324-331, DHDOmegaSparse 36-58
            a = 0.5 * np.exp(1j * ph)
            g_om = np.real(pre * (a * F[:, 0] + np.conj(a) * F[:, 1]))
        if needs[1]:  # 333-338, DHDDeltaSparse 87-101
            g_de = np.real(pre * (-np.diag(S)))
        if needs[2]:  # 340-345, DHDPhiSparse 61-84
            a = 0.5 * om_full * np.exp(1j * (ph + np.pi / 2))
            g_ph = np.real(pre * (a * F[:, 0] + np.conj(a) * F[:, 1]))
        if needs[3]:  # 347-353, DHDUSparse 104-119: upper triangle only
            g_U = np.triu(np.real(pre * S), 1)
    if needs[4]:  # 355-366
        g_st = krylov_exp(lambda x: 1j * dt * H.apply(x), grad_out, tol, tol,
                          max_krylov_dim=max_krylov_dim)
    return g_om, g_de, g_ph, g_U, g_st


# ----------------------------------------------------------------------- sampling
def sample_indices(p: np.ndarray, uniforms: np.ndarray) -> np.ndarray:
    """emu_sv/utils.py:40-49: cdf = cumsum(p) in FP64, normalised by its last value,
    searchsorted(cdf, u, right=True), clamped to the last index."""
    cdf = np.cumsum(np.asarray(p, dtype=np.float64))
    total = cdf[-1]
    if not total > 0:
        raise RuntimeError("invalid multinomial distribution (sum of probabilities <= 0)")
    idx = np.searchsorted(cdf / total, np.asarray(uniforms, dtype=np.float64), side="right")
    return np.minimum(idx, len(cdf) - 1)


# ----------------------------------------------------------------------- observables
def occupation(psi: np.ndarray) -> np.ndarray:
    """custom_callback_implementations.py:30-47."""
    psi = _c128(psi)
    n = int(round(np.log2(psi.size)))
    out = np.zeros(n)
    lib().or_occupation(n, _p(psi), _p(out))
    return out


def correlation(psi: np.ndarray) -> np.ndarray:
    """custom_callback_implementations.py:77-102."""
    psi = _c128(psi)
    n = int(round(np.log2(psi.size)))
    out = np.zeros((n, n))
    lib().or_correlation(n, _p(psi), _p(out))
    return out


def energy(H: Hamiltonian, psi) -> float:
    return H.expect(psi)


def energy_second_moment(H: Hamiltonian, psi) -> float:
    """custom_callback_implementations.py:170-185."""
    h = H.apply(psi)
    return vdot(h, h).real


def energy_variance(H: Hamiltonian, psi) -> float:
    """custom_callback_implementations.py:131-147."""
    psi = _c128(psi)
    h = H.apply(psi)
    return vdot(h, h).real - vdot(psi, h).real ** 2


# ----------------------------------------------------------------------- workloads
def run_workload(w, nsteps: int | None = None, state: np.ndarray | None = None,
                 observe: bool = True, probes: int = 0):
    """Step a workload the way SVBackendImpl does (emu_sv/sv_backend_impl.py:186-242):
    midpoint samples per step, observables on the renormalised state with the H of the
    step just completed.  Returns a dict like tests/golden/make_golden.py:run_reference."""
    n = w.nqubits
    if state is None:
        state = np.zeros(1 << n, dtype=np.complex128)
        state[0] = 1.0
    steps = w.nsteps if nsteps is None else nsteps
    occ, en, at, iters = [], [], [], []
    for k in range(steps):
        state, H, info = evolve_step(w.dt, w.omega[k], w.delta[k], w.phi[k], w.U, state,
                                     w.tolerance, w.max_krylov_dim)
        iters.append(info.iteration_count)
        if observe and ((w.obs_every and (k + 1) % w.obs_every == 0) or k + 1 == steps):
            nrm = norm(state)
            s = state / nrm if not np.isclose(nrm, 1.0) else state
            occ.append(occupation(s))
            en.append(H.expect(s))
            at.append(k + 1)
    out = {"final": state, "occupation": np.array(occ), "energy": np.array(en),
           "steps_at": np.array(at), "iters": np.array(iters)}
    if probes:
        P = probe_vectors(n, probes)
        out["probe_overlaps"] = P.conj() @ state
    return out


def probe_vectors(n: int, count: int) -> np.ndarray:
    """The seeded probe vectors of tests/golden/make_golden.py (torch CPU generator 123)."""
    import torch

    g = torch.Generator().manual_seed(123)
    return torch.randn(count, 2**n, dtype=torch.complex128, generator=g).numpy()


def neel_loss_and_grad(gw, set_index: int, nseg: int | None = None):
    """Loss MSE(occupation, Neel) after the piecewise-constant pulse and its gradient
    with respect to the per-segment global Omega and delta, by the reference's adjoint
    chain (every step's input state kept, as torch.py:215 does)."""
    n = gw.nqubits
    nseg = gw.nsegments if nseg is None else nseg
    om = gw.omega_seg[set_index, :nseg]
    de = gw.delta_seg[set_index, :nseg]
    zeros = np.zeros(n)
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1.0
    states = []
    for seg in range(nseg):
        for _ in range(gw.steps_per_segment):
            states.append((seg, s))
            s, _, _ = evolve_step(gw.dt, np.full(n, om[seg]), np.full(n, de[seg]), zeros,
                                  gw.U, s, gw.tolerance)
    occ = occupation(s)
    diff = occ - gw.target
    loss = float(np.mean(diff**2))
    # d loss / d psi* in torch's convention: 2 * dL/docc_i * x_i * psi
    w_bits = 2.0 * diff / n
    x = np.arange(1 << n)
    fac = np.zeros(1 << n)
    for i in range(n):
        fac += w_bits[i] * ((x >> (n - 1 - i)) & 1)
    g = 2.0 * fac * s
    g_om = np.zeros(nseg)
    g_de = np.zeros(nseg)
    for seg, s_in in reversed(states):
        go, gd, _, _, g = step_backward(gw.dt, np.full(n, om[seg]), np.full(n, de[seg]), zeros,
                                        gw.U, s_in, g, gw.tolerance,
                                        needs=(True, True, False, False, True))
        g_om[seg] += go.sum()
        g_de[seg] += gd.sum()
    return loss, g_om, g_de, occ


# ----------------------------------------------------------------------- Monte Carlo
def noise_from_lindbladians(lindbladians) -> np.ndarray:
    """-0.5i sum L^dag L (emu_base/jump_lindblad_operators.py:79-93)."""
    acc = np.zeros((2, 2), dtype=np.complex128)
    for L in lindbladians:
        L = np.asarray(L, dtype=np.complex128)
        acc += L.conj().T @ L
    return -0.5j * acc


def expect_batch(psi: np.ndarray, ops: np.ndarray, n: int) -> np.ndarray:
    """T[q, i] = Tr(ops_i rho_q) with rho_q[a][b] = sum psi[.,a,.] conj(psi[.,b,.])
    (emu_sv/algebra.py:4-25)."""
    psi = _c128(psi)
    out = np.empty((n, len(ops)), dtype=np.complex128)
    for q in range(n):
        v = psi.reshape(2 ** q, 2, -1)
        rho = np.einsum("iaj,ibj->ab", v, v.conj())
        for i, O in enumerate(ops):
            out[q, i] = np.trace(np.asarray(O) @ rho)
    return out


def apply_1q(psi: np.ndarray, q: int, op) -> np.ndarray:
    """op on qubit q (emu_sv/algebra.py:28-37)."""
    psi = _c128(psi)
    return np.einsum("ab,ibj->iaj", np.asarray(op, dtype=np.complex128),
                     psi.reshape(2 ** q, 2, -1)).reshape(-1)


class Brent:
    """emu_base/math/brents_root_finding.py:4-94, one abscissa at a time."""

    def __init__(self, start, end, f_start, f_end, epsilon):
        self.eps = epsilon
        self.a, self.b, self.fa, self.fb = start, end, f_start, f_end
        assert self.fa * self.fb < 0
        if abs(self.fa) < abs(self.fb):
            self.a, self.b, self.fa, self.fb = self.b, self.a, self.fb, self.fa
        self.c, self.fc, self.d = self.a, self.fa, self.a
        self.bis = True
        self.nxt = None

    def next(self):
        a, b, c, fa, fb, fc = self.a, self.b, self.c, self.fa, self.fb, self.fc
        if abs(fc - fa) < self.eps or abs(fc - fb) < self.eps:
            dx = fb * (b - a) / (fa - fb)
        else:
            s_, r_, t_ = fb / fa, fb / fc, fa / fc
            dx = s_ * (t_ * (r_ - t_) * (c - b) + (r_ - 1) * (b - a)) / ((t_ - 1) * (s_ - 1) * (r_ - 1))
        delta = abs(2 * self.eps * b)
        ref = abs(b - c) if self.bis else abs(c - self.d)
        if abs(dx) >= abs(3 * (a - b) / 4) or dx * (a - b) < 0 or abs(dx) >= ref / 2 or ref < delta:
            dx, self.bis = (a - b) / 2, True
        else:
            self.bis = False
        self.nxt = b + dx
        self.d = c
        self.c, self.fc = b, fb
        return self.nxt

    def provide(self, x, fx):
        assert x == self.nxt
        if self.fa * fx < 0:
            self.b, self.fb = x, fx
        else:
            self.a, self.fa = x, fx
        if abs(self.fa) < abs(self.fb):
            self.a, self.b, self.fa, self.fb = self.b, self.a, self.fb, self.fa

    def converged(self, tol):
        return abs(self.b - self.a) < tol


def monte_carlo_step(rnd, threshold, dt, omegas, deltas, phis, U, state, lindblads, tol,
                     max_krylov_dim=100):
    """One EvolveMonteCarlo.apply (emu_sv/time_evolution/implementations.py:192-250) with
    the random draws taken from ``rnd`` (a ``random.Random`` or the module) in the
    reference's order.  Returns (state, new threshold, number of jumps)."""
    H = Hamiltonian(omegas, deltas, phis, U, noise_from_lindbladians(lindblads))
    n = H.n

    def evolve(t, psi):
        return krylov_exp(lambda x: -1j * t * H.apply(x), psi, tol, tol, is_hermitian=False,
                          max_krylov_dim=max_krylov_dim)

    ops = [np.asarray(L, dtype=np.complex128) for L in lindblads]
    agg = [L.conj().T @ L for L in ops]
    cur, jtol, jumps = 0.0, dt * 0.1, 0
    new = norm(state) ** 2 - threshold
    while abs(dt - cur) > 1e-5:
        old = new
        state = evolve(dt - cur, state)
        new = norm(state) ** 2 - threshold
        if new > 0.0:
            break
        rf = Brent(cur, dt, old, new, jtol)
        cur = dt
        while not rf.converged(jtol):
            t = rf.next()
            state = evolve(t - cur, state)
            cur = t
            new = norm(state) ** 2 - threshold
            rf.provide(cur, new)
        w = expect_batch(state, agg, n).real  # do_quantum_jump, 168-190
        q, L = rnd.choices([(q, L) for q in range(n) for L in ops], weights=w.reshape(-1).tolist())[0]
        state = apply_1q(state, q, L)
        state = state / norm(state)
        threshold = rnd.uniform(0.0, norm(state) ** 2)
        jumps += 1
        new = norm(state) ** 2 - threshold
    return state, threshold, jumps


# ----------------------------------------------------------------------- PCHIP
def pchip(x, y, xq) -> np.ndarray:
    """PCHIP1D(x, y)(xq), restating emu_base/math/pchip_torch.py:97-269 in numpy (the same
    operation order: secants, weighted harmonic interior slopes, limited one-sided end
    slopes, Hermite coefficients, Horner)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    xq = np.asarray(xq, dtype=np.float64)
    n = x.size
    h = x[1:] - x[:-1]
    delta = (y[1:] - y[:-1]) / h
    d = np.zeros(n)
    if n == 2:
        d[:] = delta[0]
    else:
        dl, dr, hl, hr = delta[:-1], delta[1:], h[:-1], h[1:]
        wl, wr = hl + 2.0 * hr, 2.0 * hl + hr
        with np.errstate(divide="ignore", invalid="ignore"):
            dh = (wl + wr) / (wl / dl + wr / dr)
        d[1:-1] = np.where(dl * dr > 0, dh, 0.0)

        def end(a, b, ha, hb):
            e = ((2.0 * ha + hb) * a - ha * b) / (ha + hb)
            if e * a < 0:
                e = 0.0
            if a * b < 0 and abs(e) > 3.0 * abs(a):
                e = 3.0 * a
            return e

        d[0] = end(delta[0], delta[1], h[0], h[1])
        d[-1] = end(delta[-1], delta[-2], h[-1], h[-2])
    p2 = (3.0 * delta - 2.0 * d[:-1] - d[1:]) / h
    p3 = (d[:-1] + d[1:] - 2.0 * delta) / (h * h)
    i = np.clip(np.searchsorted(x, xq, side="right") - 1, 0, n - 2)
    t = xq - x[i]
    return y[:-1][i] + t * (d[:-1][i] + t * (p2[i] + t * p3[i]))


# ----------------------------------------------------------------------- Lindblad
def _row_op(op, rho, q, n):
    """op on the row index of qubit q (qubit 0 = most significant bit): op @ rho there."""
    A = rho.reshape(2 ** q, 2, 2 ** (n - q - 1), 2 ** n)
    return np.einsum("ab,ibjc->iajc", np.asarray(op, dtype=np.complex128), A).reshape(rho.shape)


def _col_op_conj(op, rho, q, n):
    """rho @ op^dag on the column index of qubit q."""
    B = rho.reshape(2 ** n, 2 ** q, 2, 2 ** (n - q - 1))
    return np.einsum("ab,kibj->kiaj", np.conj(np.asarray(op, dtype=np.complex128)), B).reshape(rho.shape)


def lindbladian_apply(omegas, deltas, phis, U, lindblads, rho) -> np.ndarray:
    """RydbergLindbladian @ rho, restating emu_sv/lindblad_operator.py:96-211 with the same
    per-qubit views: Heff = H - 0.5i sum L^dag L on every qubit (H on the row index column
    by column); res = Heff rho - (Heff rho)^dag + i sum_kq L_kq rho L_kq^dag; returns
    0.5 (res - res^dag)."""
    n = len(omegas)
    rho = np.asarray(rho, dtype=np.complex128)
    H = Hamiltonian(omegas, deltas, phis, U)
    hr = np.stack([H.apply(np.ascontiguousarray(rho[:, c])) for c in range(rho.shape[1])], axis=1)
    noise = noise_from_lindbladians(lindblads)
    for q in range(n):
        hr = hr + _row_op(noise, rho, q, n)
    res = hr - hr.conj().T
    for q in range(n):
        for L in lindblads:
            res = res + 1j * _col_op_conj(L, _row_op(L, rho, q, n), q, n)
    return 0.5 * (res - res.conj().T)


def lindblad_step(dt, omegas, deltas, phis, U, lindblads, rho, tol, max_krylov_dim=100):
    """EvolveDensityMatrix.apply (emu_sv/time_evolution/implementations.py:87-120):
    krylov_exp(-1j dt (L @ rho), is_hermitian=False) on the flattened matrix."""
    D = np.asarray(rho).shape[0]

    def op(x):
        return -1j * dt * lindbladian_apply(omegas, deltas, phis, U, lindblads,
                                            x.reshape(D, D)).reshape(-1)

    r = krylov_exp_impl(op, np.asarray(rho).reshape(-1), False, tol, tol, max_krylov_dim)
    if not r.converged:
        raise RecursionError("exponentiation algorithm did not converge to precision in "
                             "allotted number of steps.")
    return r.result.reshape(D, D), r
