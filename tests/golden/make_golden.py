"""Generate the golden fixtures under tests/golden/ by running the REFERENCE emu-sv code.

This script is the only place that executes the reference implementation.  It runs in
the build container where the reference checkout is readable (its path is the required
``--reference`` argument) and writes small ``.npz`` fixtures that the
test suite reads on any machine.  Nothing else in the repository imports it.

The reference's package ``__init__`` files pull in ``pulser``, which is not installed,
so the four hot-path modules are loaded one by one behind package shells:

* emu_base/math/krylov_exp.py       (krylov_exp_impl, krylov_exp)
* emu_base/math/double_krylov.py    (double_krylov, lanczos)
* emu_sv/hamiltonian.py             (RydbergHamiltonian)
* emu_sv/time_evolution/torch.py    (DifferentiableStateVectorEvolution)
* emu_sv/custom_callback_implementations.py (occupation / correlation / energy moments)
* emu_base/math/pchip_torch.py, emu_base/math/brents_root_finding.py,
  emu_base/jump_lindblad_operators.py,
  emu_sv/algebra.py, emu_sv/lindblad_operator.py, emu_sv/time_evolution/interface.py and
  implementations.py (the Monte Carlo and density-matrix steppers)

``pulser.*`` and ``pyparsing`` imports are served by a meta-path finder that fabricates
empty placeholder classes; none of them is called on the paths exercised here.
``emu_sv.state_vector.StateVector`` is replaced by a minimal holder of ``.data`` (all the
hot path reads from it).

Fixtures (inputs and reference outputs, all complex128/float64):

* hamiltonian.npz      H*psi and the diagonal: the reference's own test cases
                       (test/emu_sv/test_hamiltonian.py:20-85) plus larger registers.
* krylov_step.npz      one time step (test/emu_sv/test_time_evolution.py:58-76 cases)
                       with the reference's Krylov iteration counts.
* backward.npz         gradients of Re<r|psi_out> (test_time_evolution.py:79-103 cases).
* double_krylov.npz    Frechet derivative blocks (test/emu_base/math/test_double_krylov.py).
* observables.npz      occupation, correlation, energy, variance, second moment.
* chain_n10.npz        the N=10 chain workload, 100 steps, observables every 10 steps.
* lattice_n20.npz      the N=20 lattice workload: occupations/energy every 10 steps,
                       final-state probes (inner products with seeded vectors).
* ring_n16_grad.npz    reference autograd gradient of the Neel loss for 2 parameter sets
                       of the N=16 ring over the first 2 segments (20 steps).
* lindblad.npz         RydbergLindbladian @ rho, EvolveDensityMatrix steps and the
                       density-matrix observables (emu_sv/lindblad_operator.py).
* pchip.npz            PCHIP1D (emu_base/math/pchip_torch.py): the reference's test data,
                       random knots with extrapolated queries, drive-like 1 ns signals.
* krylov_nonhermitian.npz  the Arnoldi krylov_exp_impl for arbitrary callables (the
                       reference's test_krylov_with_matrix case and two more).
* dark_qubits.npz      state-preparation errors: the reference's init_dark_qubits on a
                       9-atom chain and 12 stepper steps on the masked data.
* noisy.npz            the Monte Carlo path: H*psi with the noise term, Arnoldi
                       krylov_exp (is_hermitian=False), expect_batch / apply, Brent's
                       abscissae, and EvolveMonteCarlo steps (N=8, 40 steps, two seeds of
                       Python's random module).

Usage:  python tests/golden/make_golden.py [--reference PATH] [--only NAME ...]
"""

from __future__ import annotations

import argparse
import importlib.abc
import importlib.machinery
import importlib.util
import os
import sys
import time
import types
import typing

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

import torch  # noqa: E402

from emulators_b200 import workloads as wl  # noqa: E402

torch.set_default_dtype(torch.float64)


# --------------------------------------------------------------------------- ref loader
class _Placeholder:
    """Generic stand-in for any pulser class (subscriptable, constructible)."""

    def __init__(self, *a, **k):
        pass

    def __class_getitem__(cls, item):
        return cls


class _FakeModule(types.ModuleType):
    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        if name == "TIME_TOLERANCE":
            return 1e-6
        cls = type(name, (_Placeholder,), {})
        setattr(self, name, cls)
        return cls


class _FakeFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    prefixes = ("pulser", "pyparsing")

    def find_spec(self, fullname, path, target=None):
        if fullname.split(".")[0] in self.prefixes:
            return importlib.machinery.ModuleSpec(fullname, self, is_package=True)
        return None

    def create_module(self, spec):
        m = _FakeModule(spec.name)
        m.__path__ = []
        if spec.name == "pyparsing":
            m.Any = typing.Any
        return m

    def exec_module(self, module):
        pass


class StateVector:
    """Minimal replacement for emu_sv.state_vector.StateVector (holds ``data``)."""

    def __init__(self, data, gpu=False, eigenstates=("r", "g")):
        self.data = data

    @property
    def n_qudits(self):
        return int(round(np.log2(self.data.shape[0])))


def load_reference(ref: str) -> dict:
    sys.meta_path.insert(0, _FakeFinder())
    for pkg, sub in [("emu_base", "emu_base"), ("emu_base.math", "emu_base/math"),
                     ("emu_sv", "emu_sv"), ("emu_sv.time_evolution", "emu_sv/time_evolution")]:
        m = types.ModuleType(pkg)
        m.__path__ = [os.path.join(ref, sub)]
        sys.modules[pkg] = m
    sv = types.ModuleType("emu_sv.state_vector")
    sv.StateVector = StateVector
    sys.modules["emu_sv.state_vector"] = sv
    for name in ["emu_sv.density_matrix_state", "emu_sv.dense_operator",
                 "emu_sv.lindblad_operator"]:
        m = _FakeModule(name)
        sys.modules[name] = m

    def load(name, rel):
        spec = importlib.util.spec_from_file_location(name, os.path.join(ref, rel))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
        return mod

    mods = {
        "krylov": load("emu_base.math.krylov_exp", "emu_base/math/krylov_exp.py"),
        "double": load("emu_base.math.double_krylov", "emu_base/math/double_krylov.py"),
        "ham": load("emu_sv.hamiltonian", "emu_sv/hamiltonian.py"),
    }
    mods["torch"] = load("emu_sv.time_evolution.torch", "emu_sv/time_evolution/torch.py")
    mods["brent"] = load("emu_base.math.brents_root_finding", "emu_base/math/brents_root_finding.py")
    mods["pchip"] = load("emu_base.math.pchip_torch", "emu_base/math/pchip_torch.py")
    mods["jump"] = load("emu_base.jump_lindblad_operators", "emu_base/jump_lindblad_operators.py")
    mods["algebra"] = load("emu_sv.algebra", "emu_sv/algebra.py")
    # the real Lindbladian (its package-level imports served from the loaded modules)
    sys.modules["emu_base"].compute_noise_from_lindbladians = mods["jump"].compute_noise_from_lindbladians
    sys.modules["emu_base"].matmul_2x2_with_batched = None  # GPU-only branch, not taken on CPU
    mods["lindblad"] = load("emu_sv.lindblad_operator", "emu_sv/lindblad_operator.py")
    # density matrices: the same minimal holder of ``data`` as the state vectors
    mods["lindblad"].DensityMatrix = StateVector
    iface = load("emu_sv.time_evolution.interface", "emu_sv/time_evolution/interface.py")
    sys.modules["emu_sv.time_evolution"].BaseStepper = iface.BaseStepper
    mods["impl"] = load("emu_sv.time_evolution.implementations",
                        "emu_sv/time_evolution/implementations.py")
    mods["cb"] = load("emu_sv.custom_callback_implementations",
                      "emu_sv/custom_callback_implementations.py")
    mods["cb"].DensityMatrix = StateVector
    mods["adapter"] = load("emu_base.pulser_adapter", "emu_base/pulser_adapter.py")
    return mods


# --------------------------------------------------------------------------- helpers
def nn_interaction_matrix(n):
    u = torch.zeros(n, n)
    for i in range(n - 1):
        u[i, i + 1] = u[i + 1, i] = 1.0
    return u


def randn_interaction_matrix(n):
    u = torch.zeros(n, n)
    for i in range(n):
        for j in range(i + 1, n):
            t = torch.rand(1)
            u[i, j] = u[j, i] = t
    return u


def dense_h(omegas, deltas, phis, U):
    """Kronecker-product dense Hamiltonian (same operator as the reference's
    test/utils_testing/utils_dense_hamiltonians.py:37-67), for the dense oracle."""
    n = U.shape[0]
    c = torch.complex128
    sx = torch.tensor([[0, 1], [1, 0]], dtype=c)
    sy = torch.tensor([[0, -1j], [1j, 0]], dtype=c)
    pn = torch.tensor([[0, 0], [0, 1]], dtype=c)
    eye = torch.eye(2, dtype=c)

    def op(ops):
        m = torch.ones(1, 1, dtype=c)
        for o in ops:
            m = torch.kron(m, o)
        return m

    h = torch.zeros(2**n, 2**n, dtype=c)
    for i in range(n):
        base = [eye] * n
        b = list(base); b[i] = sx
        h = h + omegas[i] * torch.cos(phis[i]) * op(b) / 2
        b = list(base); b[i] = sy
        h = h + omegas[i] * torch.sin(phis[i]) * op(b) / 2
        b = list(base); b[i] = pn
        h = h - deltas[i] * op(b)
        for j in range(i + 1, n):
            b = list(base); b[i] = pn; b[j] = pn
            h = h + U[i, j] * op(b)
    return h


def np_(t):
    t = t.detach()
    return t.cpu().numpy()


# --------------------------------------------------------------------------- generators
def gen_hamiltonian(R):
    Ham = R["ham"].RydbergHamiltonian
    cases = []
    for n in [3, 5, 7, 8]:  # test_hamiltonian.py:20-49
        torch.manual_seed(1337)
        om, de, ph = torch.randn(n), torch.randn(n), torch.zeros(n)
        cases.append((n, om, de, ph, nn_interaction_matrix(n), "nophase"))
    for n in [2, 4, 7, 9]:  # test_hamiltonian.py:52-85
        torch.manual_seed(1337)
        om, de, ph = torch.randn(n), torch.randn(n), torch.randn(n)
        cases.append((n, om, de, ph, randn_interaction_matrix(n), "phase"))
    g = torch.Generator().manual_seed(7)
    for n, phase in [(10, False), (10, True), (12, False), (13, True)]:
        om = torch.rand(n, generator=g) * 2 * np.pi
        de = torch.randn(n, generator=g) * 10
        ph = torch.randn(n, generator=g) if phase else torch.zeros(n)
        U = torch.as_tensor(wl.interaction_matrix(wl.chain(n, 5.0 + 0.5 * torch.rand(1, generator=g).item())))
        cases.append((n, om, de, ph, U, "phase" if phase else "nophase"))
    # complex128 parameter tensors, as the pulser adapter passes them
    n = 6
    om = (torch.rand(n, generator=g) * 4).to(torch.complex128)
    de = torch.randn(n, generator=g).to(torch.complex128)
    ph = torch.zeros(n, dtype=torch.complex128)
    cases.append((n, om, de, ph, torch.as_tensor(wl.interaction_matrix(wl.ring(n, 6.0))), "complexparams"))

    out = {}
    for k, (n, om, de, ph, U, tag) in enumerate(cases):
        torch.manual_seed(1000 + k)
        state = torch.randn(2**n, dtype=torch.complex128)
        H = Ham(omegas=om, deltas=de, phis=ph, interaction_matrix=U, device="cpu", noise=None)
        hpsi = H * state
        if n <= 9:
            hd = dense_h(om.real if om.is_complex() else om, de.real if de.is_complex() else de,
                         ph.real if ph.is_complex() else ph, U)
            assert torch.allclose(hd @ state, hpsi, atol=1e-10)
        pre = f"c{k}_"
        out[pre + "n"] = np.array(n)
        out[pre + "tag"] = np.array(tag)
        out[pre + "omegas"] = np_(om)
        out[pre + "deltas"] = np_(de)
        out[pre + "phis"] = np_(ph)
        out[pre + "U"] = np_(U)
        out[pre + "state"] = np_(state)
        out[pre + "diag"] = np_(H.diag)
        out[pre + "hpsi"] = np_(hpsi)
        out[pre + "complex"] = np.array(bool(H.complex))
    out["count"] = np.array(len(cases))
    return out


def get_randn_ham_params(n, with_phase):
    om, de = torch.randn(n), torch.randn(n)
    ph = torch.randn(n) if with_phase else torch.zeros(n)
    return om, de, ph, randn_interaction_matrix(n)


def gen_krylov_step(R):
    DSE = R["torch"].DifferentiableStateVectorEvolution
    Ham = R["ham"].RydbergHamiltonian
    kimpl = R["krylov"].krylov_exp_impl
    out, k = {}, 0
    for n in [3, 5, 8]:  # test_time_evolution.py:58-76
        for tol in [1e-8, 1e-10, 1e-12]:
            for wp in [False, True]:
                torch.manual_seed(1337)
                p = get_randn_ham_params(n, wp)
                s = torch.randn(2**n, dtype=torch.complex128)
                s = s / s.norm()
                dt = 1.0
                expected = torch.linalg.matrix_exp(-1j * dt * dense_h(*p)) @ s
                res, _ = DSE.apply(dt, *p, s.clone(), tol, 100)
                H = Ham(*p, device="cpu", noise=None)
                kr = kimpl(lambda x: -1j * dt * (H * x), s.clone(), True, tol, tol, 100)
                pre = f"c{k}_"
                for nm, v in zip(["omegas", "deltas", "phis", "U"], p):
                    out[pre + nm] = np_(v)
                out[pre + "n"] = np.array(n)
                out[pre + "tol"] = np.array(tol)
                out[pre + "dt"] = np.array(dt)
                out[pre + "state"] = np_(s)
                out[pre + "result"] = np_(res)
                out[pre + "dense"] = np_(expected)
                out[pre + "iters"] = np.array(kr.iteration_count)
                out[pre + "happy"] = np.array(kr.happy_breakdown)
                k += 1
    # a few physical steps: the chain_n10 drive at its first midpoint, several dt
    w = wl.chain_n10()
    for dt in [0.005, 0.01, 0.02]:
        p = [torch.as_tensor(w.omega[0]), torch.as_tensor(w.delta[0]),
             torch.as_tensor(w.phi[0]), torch.as_tensor(w.U)]
        torch.manual_seed(42)
        s = torch.randn(2**w.nqubits, dtype=torch.complex128)
        s = s / s.norm()
        res, _ = DSE.apply(dt, *p, s.clone(), 1e-10, 100)
        H = Ham(*p, device="cpu", noise=None)
        kr = kimpl(lambda x: -1j * dt * (H * x), s.clone(), True, 1e-10, 1e-10, 100)
        pre = f"c{k}_"
        for nm, v in zip(["omegas", "deltas", "phis", "U"], p):
            out[pre + nm] = np_(v)
        out[pre + "n"] = np.array(w.nqubits)
        out[pre + "tol"] = np.array(1e-10)
        out[pre + "dt"] = np.array(dt)
        out[pre + "state"] = np_(s)
        out[pre + "result"] = np_(res)
        out[pre + "dense"] = np_(res)
        out[pre + "iters"] = np.array(kr.iteration_count)
        out[pre + "happy"] = np.array(kr.happy_breakdown)
        k += 1
    out["count"] = np.array(k)
    return out


def gen_backward(R):
    DSE = R["torch"].DifferentiableStateVectorEvolution
    out, k = {}, 0
    for n in [3, 5, 8]:  # test_time_evolution.py:79-103
        for tol in [1e-8, 1e-10, 1e-12]:
            torch.manual_seed(1337)
            om, de, ph = torch.randn(n), torch.randn(n), torch.randn(n)
            U = randn_interaction_matrix(n)
            s = torch.randn(2**n, dtype=torch.complex128)
            s = s / s.norm()
            params = [x.clone().requires_grad_(True) for x in (om, de, ph, U)]
            s_in = s.clone().requires_grad_(True)
            dt = 1.0
            r = torch.randn(2**n, dtype=torch.complex128)
            r = r * (0.71 / r.norm())
            so, _ = DSE.apply(dt, *params, s_in, tol, 100)
            scalar = torch.vdot(r, so).real
            grads = torch.autograd.grad(scalar, (*params, s_in))
            pre = f"c{k}_"
            for nm, v in zip(["omegas", "deltas", "phis", "U", "state"], (om, de, ph, U, s)):
                out[pre + nm] = np_(v)
            out[pre + "r"] = np_(r)
            out[pre + "n"] = np.array(n)
            out[pre + "tol"] = np.array(tol)
            out[pre + "dt"] = np.array(dt)
            for nm, g in zip(["g_omegas", "g_deltas", "g_phis", "g_U", "g_state"], grads):
                out[pre + nm] = np_(g)
            k += 1
    out["count"] = np.array(k)
    return out


def gen_double_krylov(R):
    Ham = R["ham"].RydbergHamiltonian
    dk = R["double"].double_krylov
    out, k = {}, 0
    for n in [3, 4, 5, 7]:  # test_double_krylov.py:31-87
        for tol in [1e-8, 1e-10, 1e-12]:
            torch.manual_seed(1337)
            om, de, ph = torch.randn(n), torch.randn(n), torch.randn(n)
            U = randn_interaction_matrix(n)
            s = torch.randn(2**n, dtype=torch.complex128)
            s = s / s.norm()
            g = torch.randn(2**n, dtype=torch.complex128)
            H = Ham(om, de, ph, U, device="cpu", noise=None)
            Vs, dS, Vg = dk(lambda x: -1j * 1.0 * (H * x), s, g, tol, 100)
            dU = torch.stack(Vs).mT @ dS @ torch.stack(Vg).conj()
            pre = f"c{k}_"
            for nm, v in zip(["omegas", "deltas", "phis", "U", "state", "grad"], (om, de, ph, U, s, g)):
                out[pre + nm] = np_(v)
            out[pre + "n"] = np.array(n)
            out[pre + "tol"] = np.array(tol)
            out[pre + "dU"] = np_(dU)
            out[pre + "len_s"] = np.array(len(Vs))
            out[pre + "len_g"] = np.array(len(Vg))
            k += 1
    out["count"] = np.array(k)
    return out


def gen_observables(R):
    cb = R["cb"]
    Ham = R["ham"].RydbergHamiltonian
    out, k = {}, 0
    g = torch.Generator().manual_seed(99)
    torch.manual_seed(98)  # randn_interaction_matrix draws from the global generator
    for n in [1, 2, 3, 5, 8, 11]:
        s = torch.randn(2**n, dtype=torch.complex128, generator=g)
        s = s / s.norm()
        om = torch.rand(n, generator=g) * 5
        de = torch.randn(n, generator=g) * 5
        ph = torch.randn(n, generator=g) if n % 2 else torch.zeros(n)
        U = randn_interaction_matrix(n) * 10
        H = Ham(om, de, ph, U, device="cpu", noise=None)
        st = StateVector(s)
        pre = f"c{k}_"
        out[pre + "n"] = np.array(n)
        out[pre + "state"] = np_(s)
        for nm, v in zip(["omegas", "deltas", "phis", "U"], (om, de, ph, U)):
            out[pre + nm] = np_(v)
        out[pre + "occupation"] = np_(cb.qubit_occupation_sv_impl(None, config=None, state=st, hamiltonian=None))
        out[pre + "correlation"] = np_(cb.correlation_matrix_sv_impl(None, config=None, state=st, hamiltonian=None))
        out[pre + "energy"] = np_(H.expect(st))
        out[pre + "variance"] = np_(cb.energy_variance_sv_impl(None, config=None, state=st, hamiltonian=H))
        out[pre + "second_moment"] = np_(cb.energy_second_moment_sv_impl(None, config=None, state=st, hamiltonian=H))
        k += 1
    out["count"] = np.array(k)
    return out


def run_reference(R, w: wl.Workload, probes: int = 0, store_final: bool = True):
    """Step the reference chain exactly as SVBackendImpl does (sv_backend_impl.py:186-242):
    one DifferentiableStateVectorEvolution.apply per step with that step's midpoint
    samples; observables on the (renormalised) state with the H of the step just done."""
    DSE = R["torch"].DifferentiableStateVectorEvolution
    cb = R["cb"]
    n = w.nqubits
    U = torch.as_tensor(w.U)
    s = torch.zeros(2**n, dtype=torch.complex128)
    s[0] = 1.0
    occ, en, steps_at, iters = [], [], [], []
    t0 = time.time()
    for k in range(w.nsteps):
        om, de, ph = (torch.as_tensor(a[k]).to(torch.complex128) for a in (w.omega, w.delta, w.phi))
        s, H = DSE.apply(w.dt, om, de, ph, U, s, w.tolerance, w.max_krylov_dim)
        if (w.obs_every and (k + 1) % w.obs_every == 0) or k + 1 == w.nsteps:
            nrm = torch.linalg.vector_norm(s)
            st = StateVector(s / nrm if not torch.allclose(nrm, torch.tensor(1.0)) else s)
            occ.append(np_(cb.qubit_occupation_sv_impl(None, config=None, state=st, hamiltonian=None)))
            en.append(float(H.expect(st)))
            steps_at.append(k + 1)
    out = {"occupation": np.array(occ), "energy": np.array(en), "steps_at": np.array(steps_at),
           "seconds": np.array(time.time() - t0)}
    if store_final:
        out["final"] = np_(s)
    if probes:
        g = torch.Generator().manual_seed(123)
        P = torch.randn(probes, 2**n, dtype=torch.complex128, generator=g)
        out["probe_overlaps"] = np_(P.conj() @ s)
        out["final_norm"] = np.array(float(torch.linalg.vector_norm(s)))
    return out


def gen_chain_n10(R):
    return run_reference(R, wl.chain_n10())


def gen_lattice_n20(R):
    return run_reference(R, wl.lattice_n20(), probes=4, store_final=False)


def gen_ring_n16_grad(R):
    """Reference autograd through the per-step autograd.Function for the first 2 segments
    (20 steps) of 2 parameter sets of the N=16 ring workload."""
    DSE = R["torch"].DifferentiableStateVectorEvolution
    g = wl.ring_n16_grad()
    n = g.nqubits
    nseg, sets = 2, 2
    U = torch.as_tensor(g.U)
    out = {}
    for p in range(sets):
        om = torch.as_tensor(g.omega_seg[p, :nseg]).clone().requires_grad_(True)
        de = torch.as_tensor(g.delta_seg[p, :nseg]).clone().requires_grad_(True)
        s = torch.zeros(2**n, dtype=torch.complex128)
        s[0] = 1.0
        for seg in range(nseg):
            for _ in range(g.steps_per_segment):
                oms = om[seg].expand(n)
                des = de[seg].expand(n)
                s, _ = DSE.apply(g.dt, oms, des, torch.zeros(n), U, s, g.tolerance, 100)
        occ = torch.stack([torch.linalg.vector_norm(s.view(2**i, 2, -1)[:, 1]) ** 2 for i in range(n)])
        loss = torch.mean((occ - torch.as_tensor(g.target)) ** 2)
        go, gd = torch.autograd.grad(loss, (om, de))
        out[f"p{p}_omega"] = np_(om)
        out[f"p{p}_delta"] = np_(de)
        out[f"p{p}_loss"] = np.array(float(loss))
        out[f"p{p}_g_omega"] = np_(go)
        out[f"p{p}_g_delta"] = np_(gd)
        out[f"p{p}_occupation"] = np_(occ)
    out["nseg"] = np.array(nseg)
    out["sets"] = np.array(sets)
    return out


GENERATORS = {
    "hamiltonian": gen_hamiltonian,
    "krylov_step": gen_krylov_step,
    "backward": gen_backward,
    "double_krylov": gen_double_krylov,
    "observables": gen_observables,
    "chain_n10": gen_chain_n10,
    "lattice_n20": gen_lattice_n20,
    "ring_n16_grad": gen_ring_n16_grad,
}


def _lindblads(R, scale=1.0):
    """relaxation, dephasing and depolarizing operators of the reference's own
    get_lindblad_operators, plus one effective-noise style operator."""
    class NM:
        noise_types = ("relaxation", "dephasing", "depolarizing")
        relaxation_rate = 0.9 * scale
        dephasing_rate = 0.6 * scale
        hyperfine_dephasing_rate = 0.0
        depolarizing_rate = 0.3 * scale

    ops = []
    for t in NM.noise_types:
        ops += R["jump"].get_lindblad_operators(noise_type=t, noise_model=NM)
    ops.append(torch.tensor([[0.1, 0.2 + 0.1j], [0.0, -0.3j]], dtype=torch.complex128) * scale ** 0.5)
    return ops


def gen_noisy(R):
    """Noisy (non-Hermitian) H*psi, Arnoldi krylov_exp, expect_batch / apply, Brent's root
    finder and EvolveMonteCarlo steps with seeded random draws."""
    import random

    Ham = R["ham"].RydbergHamiltonian
    kimpl = R["krylov"].krylov_exp_impl
    out = {}
    ops = _lindblads(R)
    noise = R["jump"].compute_noise_from_lindbladians(ops)
    out["noise"] = np_(noise)
    for k, L in enumerate(ops):
        out[f"L{k}"] = np_(L)
    out["nops"] = np.array(len(ops))
    # H*psi with noise
    for k, (n, wp) in enumerate([(3, False), (5, True), (8, False), (11, True), (13, True)]):
        torch.manual_seed(100 + k)
        p = get_randn_ham_params(n, wp)
        psi = torch.randn(2 ** n, dtype=torch.complex128)
        H = Ham(*p, device="cpu", noise=noise)
        pre = f"h{k}_"
        for nm, v in zip(["omegas", "deltas", "phis", "U"], p):
            out[pre + nm] = np_(v)
        out[pre + "psi"] = np_(psi)
        out[pre + "hpsi"] = np_(H * psi)
        out[pre + "diag"] = np_(H.diag)
    out["hcount"] = np.array(5)
    # Arnoldi exponential (is_hermitian=False)
    k = 0
    for n in [5, 8, 10]:
        for dt in [0.01, 0.05, 0.2]:
            torch.manual_seed(200 + k)
            p = get_randn_ham_params(n, k % 2 == 1)
            s0 = torch.randn(2 ** n, dtype=torch.complex128)
            s0 = s0 / s0.norm()
            H = Ham(*p, device="cpu", noise=noise)
            kr = kimpl(lambda x: -1j * dt * (H * x), s0.clone(), False, 1e-10, 1e-10, 100)
            pre = f"a{k}_"
            for nm, v in zip(["omegas", "deltas", "phis", "U"], p):
                out[pre + nm] = np_(v)
            out[pre + "n"] = np.array(n)
            out[pre + "dt"] = np.array(dt)
            out[pre + "state"] = np_(s0)
            out[pre + "result"] = np_(kr.result)
            out[pre + "iters"] = np.array(kr.iteration_count)
            out[pre + "happy"] = np.array(kr.happy_breakdown)
            k += 1
    out["acount"] = np.array(k)
    # algebra: the reference test vectors (test/emu_sv/test_algebra.py) and a random state
    vec = torch.tensor([0.0, 0.0, 0.5j, 1.0], dtype=torch.complex128)
    nops = torch.tensor([[[0.0, 0.0], [0.0, 1.0j]], [[1.0, 0.0], [0.0, 0.0]],
                         [[0.0, 1.0j], [0.0, 0.0]]], dtype=torch.complex128)
    out["alg_vec"] = np_(vec)
    out["alg_ops"] = np_(nops)
    out["alg_expect"] = np_(R["algebra"].expect_batch(vec, nops, 2))
    torch.manual_seed(7)
    v6 = torch.randn(64, dtype=torch.complex128)
    agg = torch.stack([L.mH @ L for L in ops])
    out["alg_v6"] = np_(v6)
    out["alg_expect6"] = np_(R["algebra"].expect_batch(v6, agg, 6))
    for q in range(6):
        out[f"alg_apply6_{q}"] = np_(R["algebra"].apply(v6, q, ops[q % len(ops)]))
    # Brent: abscissae asked for on (x+3)(x-1)^2 (test_brents_root_finding.py:44-53)
    rf = R["brent"].BrentsRootFinder(start=-4.0, end=4 / 3.0, f_start=(-4 + 3) * 25.0,
                                     f_end=(4 / 3 + 3) * (1 / 3) ** 2, epsilon=1e-6)
    xs = []
    while not rf.is_converged(1e-6):
        x = rf.get_next_abscissa()
        xs.append(x)
        rf.provide_ordinate(x, (x + 3) * (x - 1) ** 2)
    out["brent_x"] = np.array(xs)
    out["brent_root"] = np.array(rf.current_guess)
    # Monte Carlo steps: N=8 chain, strong noise so that jumps happen
    w = wl.chain_n10()
    n, dt, nsteps = 8, 0.05, 40
    U = torch.as_tensor(w.U[:n, :n])
    mc_ops = _lindblads(R, scale=3.0)
    for seed in [11, 12]:
        random.seed(seed)
        stepper = R["impl"].EvolveMonteCarlo(100)
        st = torch.zeros(2 ** n, dtype=torch.complex128)
        st[0] = 1.0
        thr, states = [stepper.jump_threshold], []
        for k in range(nsteps):
            om = torch.full((n,), 2 * np.pi * (0.5 + 0.5 * np.sin(0.3 * k)), dtype=torch.float64)
            de = torch.full((n,), -4.0 + 0.2 * k, dtype=torch.float64)
            ph = torch.zeros(n, dtype=torch.float64)
            st, _ = stepper.apply(dt, om, de, ph, U, st, 1e-10, mc_ops)
            thr.append(stepper.jump_threshold)
            if (k + 1) % 10 == 0:
                states.append(np_(st).copy())  # krylov_exp normalises its input in place
        out[f"mc{seed}_thresholds"] = np.array(thr)
        out[f"mc{seed}_states"] = np.stack(states)
    out["mc_n"] = np.array(n)
    out["mc_dt"] = np.array(dt)
    out["mc_nsteps"] = np.array(nsteps)
    out["mc_nops"] = np.array(len(mc_ops))
    for k, L in enumerate(mc_ops):
        out[f"mcL{k}"] = np_(L)
    out["mc_U"] = np_(U)
    return out


GENERATORS["noisy"] = gen_noisy


def gen_pchip(R):
    """PCHIP1D on the reference's own test data, random non-uniform knots (2, 3, 5 and 50
    knots, queries inside and outside the knot range) and drive-like signals on a 1 ns grid
    evaluated at 10 ns midpoints."""
    P = R["pchip"].PCHIP1D
    out, k = {}, 0
    rng = np.random.default_rng(2024)

    def add(x, y, xq):
        nonlocal k
        out[f"c{k}_x"] = np.asarray(x, dtype=np.float64)
        out[f"c{k}_y"] = np.asarray(y, dtype=np.float64)
        out[f"c{k}_xq"] = np.asarray(xq, dtype=np.float64)
        out[f"c{k}_yq"] = np_(P(torch.as_tensor(x, dtype=torch.float64),
                                torch.as_tensor(y, dtype=torch.float64))(
            torch.as_tensor(xq, dtype=torch.float64)))
        k += 1

    add([0.0, 1.0, 2.5, 4.0], [0.0, 2.0, 1.0, 3.0], [0.0, 1.0, 2.5, 4.0, 0.3, 3.9])  # test_pchip.py
    add([0.0, 1.0, 2.0, 3.0], [0.0, 1.0, 1.5, 2.0], np.linspace(0.0, 3.0, 301))
    for n in [2, 3, 5, 50]:
        x = np.cumsum(rng.uniform(0.1, 2.0, n))
        y = rng.normal(size=n)
        if n == 50:
            y[10:20] = y[10]  # flat run (zero secants)
        xq = rng.uniform(x[0] - 1.0, x[-1] + 1.0, 200)
        add(x, y, xq)
    # drive-like signals: 1 ns grid, smooth ramps with kinks, midpoints of a 10 ns grid
    T = 800
    t = np.arange(T, dtype=np.float64)
    tt = np.arange(0, T + 1, 10, dtype=np.float64)
    tmid = 0.5 * (tt[:-1] + tt[1:])
    for j in range(4):
        knots = np.sort(rng.uniform(0, T, 6))
        vals = rng.uniform(-15, 15, 6)
        y = np.interp(t, knots, vals) + 0.05 * np.sin(0.37 * t * (j + 1))
        add(t, y, tmid)
    out["count"] = np.array(k)
    return out


GENERATORS["pchip"] = gen_pchip


def gen_lindblad(R):
    """RydbergLindbladian @ rho (n = 3, 4, 5; real and complex drives), EvolveDensityMatrix
    steps (n = 4, 12 steps of 50 ns) and the density-matrix observables of the final state."""
    Lop = R["lindblad"].RydbergLindbladian
    cb = R["cb"]
    ops = _lindblads(R, scale=2.0)
    out = {"nops": np.array(len(ops))}
    for k, L in enumerate(ops):
        out[f"L{k}"] = np_(L)

    def rand_rho(n, seed):
        g = torch.Generator().manual_seed(seed)
        a = torch.randn(2 ** n, 3, dtype=torch.complex128, generator=g)
        r = a @ a.mH
        return r / torch.trace(r).real

    for k, (n, wp) in enumerate([(3, False), (4, True), (5, False)]):
        torch.manual_seed(300 + k)
        p = get_randn_ham_params(n, wp)
        rho = rand_rho(n, 400 + k)
        L = Lop(*p[:3], ops, p[3], device="cpu")
        pre = f"c{k}_"
        for nm, v in zip(["omegas", "deltas", "phis", "U"], p):
            out[pre + nm] = np_(v)
        out[pre + "rho"] = np_(rho)
        out[pre + "Lrho"] = np_(L @ rho.clone())
        out[pre + "energy"] = np_(L.expect(StateVector(rho.clone())))
    out["count"] = np.array(3)
    # EvolveDensityMatrix: N=4 chain, time-dependent drive
    n, dt, nsteps = 4, 0.05, 12
    U = torch.as_tensor(wl.interaction_matrix(wl.chain(n, 6.0)))
    stepper = R["impl"].EvolveDensityMatrix(100)
    rho = torch.zeros(2 ** n, 2 ** n, dtype=torch.complex128)
    rho[0, 0] = 1.0
    snaps = []
    for k in range(nsteps):
        om = torch.full((n,), 2 * np.pi * (0.6 + 0.4 * np.sin(0.5 * k)), dtype=torch.float64)
        de = torch.full((n,), -3.0 + 0.5 * k, dtype=torch.float64)
        ph = torch.full((n,), 0.1 * k, dtype=torch.float64)
        rho, ham = stepper.apply(dt, om, de, ph, U, rho, 1e-10, ops)
        if (k + 1) % 4 == 0:
            snaps.append(np_(rho).copy())
    out["ev_states"] = np.stack(snaps)
    out["ev_n"] = np.array(n)
    out["ev_dt"] = np.array(dt)
    out["ev_nsteps"] = np.array(nsteps)
    out["ev_U"] = np_(U)
    st = StateVector(rho.clone())
    out["ev_occupation"] = np_(cb.qubit_occupation_sv_den_mat_impl(None, config=None, state=st,
                                                                    hamiltonian=None))
    out["ev_correlation"] = np_(cb.correlation_matrix_sv_den_mat_impl(None, config=None, state=st,
                                                                       hamiltonian=None))
    out["ev_energy"] = np_(ham.expect(st))
    out["ev_variance"] = np_(cb.energy_variance_sv_den_mat_impl(None, config=None, state=st,
                                                                 hamiltonian=ham))
    out["ev_second_moment"] = np_(cb.energy_second_moment_den_mat_impl(None, config=None, state=st,
                                                                        hamiltonian=ham))
    return out


GENERATORS["lindblad"] = gen_lindblad


def gen_target_times(R):
    """The reference's target-time grid (emu_base/pulser_adapter.py:130-151): a uniform
    dt grid over the sequence duration merged with the observables' evaluation times,
    near-duplicates (TIME_TOLERANCE, 1e-6 under the pulser stand-in above) dropped.  Cases:
    the two of test/emu_base/test_adapter.py:905-966 plus seeded ones (durations that dt
    does not divide, times within and just outside the tolerance of grid points)."""
    from types import SimpleNamespace

    ad = R["adapter"]
    rng = np.random.default_rng(2024)
    cases = [
        (20.0, 5.5, [[0.0, 0.9 / 20, 11.9 / 20, 18.1 / 20]], None),
        (20.0, 5.5, [None], [0.5]),
        (2000.0, 10.0, [[0.05 * k for k in range(1, 21)]], None),
        (100.0, 30.0, [[0.5]], None),
        (100.0, 33.3333333, [[0.25, 0.75]], None),
        (100.0, 100.0, [[0.5], [0.5, 0.25]], None),
    ]
    g = 7.0 / 1237.0  # grid of case 6: near-duplicates of grid points and of each other
    near = [3 * g + 4e-7, 5 * g - 9e-7, 8 * g + 2e-6, 0.5, 0.5 + 5e-7, 0.5 + 3e-6, 1.0 - 4e-7]
    cases.append((1237.0, 7.0, [list(rng.uniform(0, 1, 6)) + near], None))
    cases.append((3000.0, 5.0, [[1 / 3, 2 / 3, 0.9999999, 1.0], [0.0, 1 / 3]], None))
    cases.append((1500.0, 4.9, [list(rng.uniform(0, 1, 25))], [0.1, 0.2]))
    out = {}
    for k, (dur, dt, obs_times, default) in enumerate(cases):
        seq = SimpleNamespace(get_duration=lambda include_fall_time=False, d=dur: d)
        cfg = SimpleNamespace(
            observables=[SimpleNamespace(evaluation_times=t) for t in obs_times],
            default_evaluation_times=np.asarray(default if default is not None else [1.0]),
            with_modulation=False)
        tt = ad._get_target_times(seq, cfg, dt)
        union = sorted(ad._unique_observable_times(cfg))
        out[f"c{k}_duration"] = np.array(dur)
        out[f"c{k}_dt"] = np.array(dt)
        out[f"c{k}_obs"] = np.array(union, dtype=np.float64)
        out[f"c{k}_expected"] = np.array(tt, dtype=np.float64)
    out["count"] = np.array(len(cases))
    out["tolerance"] = np.array(float(ad.TIME_TOLERANCE))
    return out


GENERATORS["target_times"] = gen_target_times


def load_backend_impl(R, ref: str):
    """emu_sv/sv_backend_impl.py with stand-ins for what it imports besides the hot-path
    modules already loaded (emu_base's adapter helpers, the config and state classes)."""
    import emu_base  # the package shell of load_reference

    for name in ("SequenceData", "get_max_rss_cpu", "get_max_rss_gpu"):
        setattr(emu_base, name, getattr(R["adapter"], name, _Placeholder))
    emu_base.is_evaluation_time = R["adapter"].is_evaluation_time
    for name in ("emu_sv.dense_state", "emu_sv.sv_config"):
        sys.modules[name] = _FakeModule(name)
    spec = importlib.util.spec_from_file_location("emu_sv.solver", os.path.join(ref, "emu_sv/solver.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["emu_sv.solver"] = mod
    spec.loader.exec_module(mod)
    te = sys.modules["emu_sv.time_evolution"]
    for name in ("EvolveStateVector", "EvolveDensityMatrix", "EvolveMonteCarlo"):
        setattr(te, name, getattr(R["impl"], name))
    spec = importlib.util.spec_from_file_location("emu_sv.sv_backend_impl",
                                                  os.path.join(ref, "emu_sv/sv_backend_impl.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["emu_sv.sv_backend_impl"] = mod
    spec.loader.exec_module(mod)
    return mod


def gen_dark_qubits(R):
    """State-preparation errors: the reference's SVBackendImpl.init_dark_qubits
    (sv_backend_impl.py:162-184) on a 9-atom chain with atoms 0, 4 and 7 badly prepared
    (Omega, delta, phi of those atoms zeroed, their interaction rows and columns zeroed),
    then 12 steps of the reference stepper chain on the masked data."""
    impl = load_backend_impl(R, R["ref_path"])
    n, steps = 9, 12
    rng = np.random.default_rng(21)
    pos = wl.chain(n, 6.0)
    U0 = torch.as_tensor(wl.interaction_matrix(pos))
    om = torch.as_tensor(rng.uniform(1.0, 6.0, (steps, n)))
    de = torch.as_tensor(rng.uniform(-10.0, 10.0, (steps, n)))
    ph = torch.as_tensor(rng.normal(size=(steps, n)))
    bad = (True, False, False, False, True, False, False, True, False)
    ns = types.SimpleNamespace(
        _data=types.SimpleNamespace(state_prep_error=0.1, bad_atoms=bad),
        interaction_matrix=lambda t: U0.unsqueeze(0), omega=om.clone(), delta=de.clone(),
        phi=ph.clone())
    impl.SVBackendImpl.init_dark_qubits(ns)
    U = ns.interaction_matrix(0.0)[0]
    DSE = R["torch"].DifferentiableStateVectorEvolution
    s = torch.zeros(2**n, dtype=torch.complex128)
    s[0] = 1.0
    dt = 0.01
    for k in range(steps):
        s, _ = DSE.apply(dt, ns.omega[k], ns.delta[k], ns.phi[k], U, s, 1e-10, 100)
    return {"omega": np_(om), "delta": np_(de), "phi": np_(ph), "U": np_(U0),
            "bad_atoms": np.array(bad), "dt": np.array(dt),
            "omega_masked": np_(ns.omega), "delta_masked": np_(ns.delta),
            "phi_masked": np_(ns.phi), "U_masked": np_(U), "final": np_(s)}


GENERATORS["dark_qubits"] = gen_dark_qubits


def gen_krylov_nonhermitian(R):
    """The Arnoldi branch of krylov_exp_impl (is_hermitian=False) for arbitrary callables:
    the reference's own test_krylov_with_matrix case (test/emu_base/math/test_krylov_exp.py:
    194-218: seed 1211, a random 256 x 256 operator of unit norm applied to a random 256 x
    256 tensor, tolerances 1e-6), a random non-Hermitian operator on a vector at 1e-10, and
    a rank-2 operator (happy breakdown)."""
    K = R["krylov"]
    c = torch.complex128
    out = {}

    def run(pre, A, x, tol):
        r = K.krylov_exp_impl(lambda y: A @ y, x.clone(), is_hermitian=False, exp_tolerance=tol,
                              norm_tolerance=tol, max_krylov_dim=100)
        out[pre + "op"], out[pre + "in"], out[pre + "result"] = np_(A), np_(x), np_(r.result)
        out[pre + "iters"] = np.array(r.iteration_count)
        out[pre + "happy"] = np.array(r.happy_breakdown)
        out[pre + "converged"] = np.array(r.converged)
        out[pre + "tol"] = np.array(tol)

    torch.random.manual_seed(1211)
    A = torch.rand(256, 256, dtype=c)
    A = A / A.norm()
    X = torch.rand(256, 256, dtype=c)
    run("m_", A, X, 1e-6)
    g = torch.Generator().manual_seed(17)
    B = (torch.rand(128, 128, dtype=c, generator=g) - (0.5 + 0.5j)) * 0.4
    v = torch.rand(128, dtype=c, generator=g) - (0.5 + 0.5j)
    run("v_", B, v, 1e-10)
    u = torch.rand(64, 2, dtype=c, generator=g)
    w = torch.rand(2, 64, dtype=c, generator=g)
    run("r_", u @ w, torch.rand(64, dtype=c, generator=g), 1e-10)
    return out


GENERATORS["krylov_nonhermitian"] = gen_krylov_nonhermitian


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="checkout of the reference repository (read only)")
    ap.add_argument("--only", nargs="*", default=None)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    a = ap.parse_args()
    torch.set_num_threads(a.threads)
    R = load_reference(a.reference)
    R["ref_path"] = a.reference
    for name, fn in GENERATORS.items():
        if a.only and name not in a.only:
            continue
        t = time.time()
        data = fn(R)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
        print(f"{name}: {len(data)} arrays, {time.time() - t:.1f}s", flush=True)


if __name__ == "__main__":
    main()
