"""GPU check of emusv_expect_noalloc, the energy-moments entry point that allocates
nothing: its reduction scratch is a static device array inside the library, for callers
that cannot allocate device memory where they call (graph-recording code, external
memory managers, host runtimes without a device allocator).

It is compared through the C ABI with emusv_expect (which takes a caller scratch
buffer) on the same state, twice in a row, so that reusing the shared static array is
covered too, and with the oracle's energy and ||H psi||^2 of the same state.  The larger
registers (n = 22, 26) launch as many blocks as the static array holds and walk the state
grid-stride.  This file is collected last on purpose."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,dtype,rtol", [(12, torch.complex128, 1e-12), (18, torch.complex64, 1e-6),
                                          (22, torch.complex64, 1e-6), (26, torch.complex64, 1e-6)])
def test_expect_noalloc_matches_expect(oracle, n, dtype, rtol):
    from emulators_b200 import _lib
    from emulators_b200 import workloads as wl

    L = _lib.load()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(7 + n)
    om = rng.uniform(0, 2 * np.pi, n)
    de = rng.uniform(-20, 20, n)
    ph = rng.normal(size=n)
    U = np.ascontiguousarray(wl.interaction_matrix(wl.chain(n, 5.5)))
    params = [om.ctypes.data, de.ctypes.data, ph.ctypes.data, U.ctypes.data]
    code = _lib.dtype_code(dtype)
    stream = torch.cuda.current_stream(dev).cuda_stream
    ref = torch.empty(3, dtype=torch.float64, device=dev)
    scratch = torch.empty(L.emusv_scratch_bytes(n, code), dtype=torch.uint8, device=dev)
    for call in range(2):
        psi = torch.randn(1 << n, dtype=dtype, device=dev)
        psi /= torch.linalg.vector_norm(psi)
        _lib.check(L.emusv_expect(n, code, *params, psi.data_ptr(), ref.data_ptr(), scratch.data_ptr(),
                                  scratch.numel(), stream), "expect")
        got = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
        _lib.check(L.emusv_expect_noalloc(n, code, *params, psi.data_ptr(), got.data_ptr(), stream),
                   "expect_noalloc")
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        scale = max(abs(r[0]), np.sqrt(abs(r[2])))
        np.testing.assert_allclose(g, r, rtol=rtol, atol=rtol * scale, err_msg=f"call {call}")
        if call == 0:  # the oracle's moments of the same (stored) state, in FP64
            host = psi.cpu().to(torch.complex128).numpy()
            hpsi = oracle.Hamiltonian(om, de, ph, U).apply(host)
            e = np.vdot(host, hpsi)
            want = np.array([e.real, e.imag, np.vdot(hpsi, hpsi).real])
            tol = max(rtol, 2e-6 if dtype == torch.complex64 else rtol)
            np.testing.assert_allclose(g, want, rtol=tol, atol=tol * scale, err_msg="oracle")
            del host, hpsi


def test_expect_noalloc_rejects_bad_sizes():
    from emulators_b200 import _lib

    L = _lib.load()
    z = np.zeros(32)
    U = np.zeros(32 * 32)
    p = [z.ctypes.data, z.ctypes.data, z.ctypes.data, U.ctypes.data]
    dev = torch.device("cuda", 0)
    buf = torch.zeros(4, dtype=torch.float64, device=dev)
    psi = torch.zeros(2, dtype=torch.complex128, device=dev)
    assert L.emusv_expect_noalloc(_lib.MAX_QUBITS + 1, 0, *p, psi.data_ptr(), buf.data_ptr(), None) \
        == _lib.BAD_ARGUMENT
    assert L.emusv_expect_noalloc(0, 0, *p, psi.data_ptr(), buf.data_ptr(), None) == _lib.BAD_ARGUMENT
