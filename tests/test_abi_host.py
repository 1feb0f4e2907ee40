"""C ABI and host-side logic, CPU only: the library loads, exports every symbol the
header declares, validates arguments before touching the GPU, and the Python layer maps
status codes to the reference's exceptions."""

import os
import re

import numpy as np
import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "emusv_b200.h")


def header_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|size_t|const char \*)\s*(emusv_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    from emulators_b200 import _lib

    L = _lib.load()
    declared = header_functions()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    assert set(_lib.SIGNATURES) == set(declared)
    assert L.emusv_build_arch() == 100


def test_status_strings_and_exception_mapping():
    from emulators_b200 import _lib

    assert _lib.status_message(0) == "ok"
    _lib.check(0, "x")
    with pytest.raises(RecursionError):
        _lib.check(_lib.NOT_CONVERGED, "step")
    with pytest.raises(ValueError):
        _lib.check(_lib.BAD_ARGUMENT, "step")
    with pytest.raises(FloatingPointError):
        _lib.check(_lib.NONFINITE, "step")
    with pytest.raises(_lib.WorkspaceTooSmall):
        _lib.check(_lib.WORKSPACE_TOO_SMALL, "step")
    with pytest.raises(TimeoutError):
        _lib.check(_lib.TIMEOUT, "step")
    with pytest.raises(RuntimeError):
        _lib.check(_lib.CUDA_ERROR, "step")


def test_argument_validation_happens_before_any_device_work():
    """Bad arguments are rejected on the host (no GPU in this process)."""
    from emulators_b200 import _lib

    L = _lib.load()
    n = 4
    om = np.ones(n)
    z = np.zeros(n)
    U = np.zeros((n, n))
    P = (om.ctypes.data, z.ctypes.data, z.ctypes.data, U.ctypes.data)
    # null vector pointers
    assert L.emusv_hpsi(n, 0, *P, None, None, None) == _lib.BAD_ARGUMENT
    # qubit count out of range
    assert L.emusv_hpsi(0, 0, *P, 16, 32, None) == _lib.BAD_ARGUMENT
    assert L.emusv_hpsi(31, 0, *P, 16, 32, None) == _lib.BAD_ARGUMENT
    # non-finite parameters
    bad = np.array([np.nan, 1, 1, 1.0])
    assert L.emusv_hpsi(n, 0, bad.ctypes.data, *P[1:], 16, 32, None) == _lib.BAD_ARGUMENT
    # unknown dtype
    info = _lib.KrylovInfo()
    assert L.emusv_krylov_step(n, 7, 0.1, *P, 256, 256, 1e-10, 1e-10, 10, 0, 256, 1 << 20, info,
                               None) == _lib.BAD_ARGUMENT
    # max_krylov_dim out of range
    assert L.emusv_krylov_step(n, 0, 0.1, *P, 256, 256, 1e-10, 1e-10, 0, 0, 256, 1 << 20, info,
                               None) == _lib.BAD_ARGUMENT
    # misaligned workspace
    assert L.emusv_krylov_step(n, 0, 0.1, *P, 256, 256, 1e-10, 1e-10, 10, 0, 257, 1 << 20, info,
                               None) == _lib.BAD_ARGUMENT
    # too small workspace (header does not fit)
    assert L.emusv_krylov_step(n, 0, 0.1, *P, 256, 256, 1e-10, 1e-10, 10, 0, 256, 64, info,
                               None) == _lib.WORKSPACE_TOO_SMALL
    assert L.emusv_tridiag_expm_col(0, None, None, None, None, None, 0, None) == _lib.BAD_ARGUMENT


def test_workspace_sizes():
    from emulators_b200 import _lib

    L = _lib.load()
    a = L.emusv_krylov_workspace_bytes(20, 0, 10)
    b = L.emusv_krylov_workspace_bytes(20, 0, 11)
    assert b - a == (1 << 20) * 16
    c = L.emusv_krylov_workspace_bytes(20, 1, 11) - L.emusv_krylov_workspace_bytes(20, 1, 10)
    assert c == (1 << 20) * 8
    assert L.emusv_krylov_workspace_bytes(31, 0, 1) == 0
    assert L.emusv_scratch_bytes(10, 0) > 0


def test_host_parameter_conversion():
    import torch

    from emulators_b200 import _lib

    t = torch.tensor([1.0, 2.0], dtype=torch.complex128)
    a = _lib.host_f64(t, 2)
    assert a.dtype == np.float64 and list(a) == [1.0, 2.0]
    with pytest.raises(ValueError):
        _lib.host_f64(t, 3)
    with pytest.raises(RuntimeError):
        _lib.require_cuda_vector(torch.zeros(4, dtype=torch.complex128))
    with pytest.raises(TypeError):
        _lib.dtype_code(torch.float32)


def test_product_refuses_cpu_tensors():
    """No CPU fallback: the drop-in classes refuse host tensors."""
    import torch

    from emulators_b200 import RydbergHamiltonian

    H = RydbergHamiltonian(torch.ones(3), torch.zeros(3), torch.zeros(3), torch.zeros(3, 3), "cpu")
    with pytest.raises(RuntimeError, match="CUDA"):
        H * torch.zeros(8, dtype=torch.complex128)
    Hn = RydbergHamiltonian(torch.ones(3), torch.zeros(3), torch.zeros(3), torch.zeros(3, 3), "cpu",
                            noise=torch.zeros(2, 2, dtype=torch.complex128))
    assert Hn.complex
    with pytest.raises(RuntimeError, match="CUDA"):
        Hn * torch.zeros(8, dtype=torch.complex128)
    with pytest.raises(ValueError):
        RydbergHamiltonian(torch.ones(3), torch.zeros(3), torch.zeros(3), torch.zeros(3, 3), "cpu",
                           noise=torch.zeros(3, 3))


def test_workloads_match_their_specification():
    from emulators_b200 import workloads as wl

    w = wl.chain_n10()
    assert w.nqubits == 10 and w.nsteps == 100 and abs(w.dt - 0.01) < 1e-15
    assert np.isclose(w.U[0, 1], wl.C6 / 5.0**6) and w.U[0, 1] == w.U[1, 0]
    assert np.isclose(w.delta[0, 0], -10 + 20 * 0.005) and np.allclose(w.omega, 4.0)
    w = wl.lattice_n20()
    assert w.nqubits == 20 and w.nsteps == 300 and w.max_krylov_dim == 30
    assert np.isclose(w.U[0, 1], wl.C6 / 6.0**6)
    w = wl.ladder_n26()
    assert w.nqubits == 26 and w.nsteps == 400 and w.precision == "c64"
    assert np.isclose(w.U[0, 13], wl.C6 / 5.5**6)  # rung
    b = wl.batch_256(count=16)
    for x in b:
        assert 12 <= x.nqubits <= 18 and x.nsteps == 150
        d = np.hypot(*(x.positions[:, None, :] - x.positions[None, :, :]).transpose(2, 0, 1))
        assert d[np.triu_indices(x.nqubits, 1)].min() >= 5.0
        assert x.positions.min() >= 0 and x.positions.max() <= 40
        assert (x.omega >= 0).all() and (x.omega <= 2 * np.pi).all()
        assert (np.abs(x.delta) <= 20).all() and (x.phi == 0).all()
    b2 = wl.batch_256(count=16)
    assert all(np.array_equal(p.U, q.U) for p, q in zip(b, b2))  # seeded
    g = wl.ring_n16_grad()
    assert g.omega_seg.shape == (64, 20) and g.nqubits == 16
    assert list(g.target[:4]) == [1, 0, 1, 0]
    assert np.isclose(np.hypot(*(g.positions[0] - g.positions[1])), 2 * 10 * np.sin(np.pi / 16))
