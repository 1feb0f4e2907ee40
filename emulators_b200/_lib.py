"""ctypes binding of ``libemusv_b200.so`` (the C ABI declared in include/emusv_b200.h).

The product path has no CPU fallback: every entry point needs the compiled library and a
CUDA tensor, and fails loudly otherwise.  Status codes map to the exceptions the
reference raises for the same conditions (RecursionError for a Krylov iteration that
does not converge, krylov_exp.py:126-129; ValueError for bad arguments).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

PKG = os.path.dirname(os.path.abspath(__file__))
# EMUSV_LIB selects another build of the same library (e.g. an instrumented one)
LIB_PATH = os.environ.get("EMUSV_LIB") or os.path.join(PKG, "libemusv_b200.so")

OK, NOT_CONVERGED, NONFINITE, BAD_ARGUMENT, WORKSPACE_TOO_SMALL, CUDA_ERROR, TIMEOUT = range(7)
C128, C64 = 0, 1
MAX_QUBITS = 30

# every symbol include/emusv_b200.h declares, with (restype, argtypes)
_P, _I, _I64, _D, _SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_size_t


class KrylovInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("happy_breakdown", ctypes.c_int),
                ("converged", ctypes.c_int), ("basis_vectors", ctypes.c_int),
                ("error_estimate", ctypes.c_double), ("input_norm", ctypes.c_double),
                ("output_norm", ctypes.c_double), ("second_rounds", ctypes.c_int)]


SIGNATURES: dict[str, tuple] = {
    "emusv_build_arch": (_I, []),
    "emusv_status_string": (ctypes.c_char_p, [_I]),
    "emusv_device_error": (_I, [_P]),
    "emusv_hamiltonian_diag": (_I, [_I, _P, _P, _P, _P]),
    "emusv_hpsi": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "emusv_scratch_bytes": (_SZ, [_I, _I]),
    "emusv_expect": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "emusv_expect_noalloc": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "emusv_occupation": (_I, [_I, _I, _P, _P, _P, _SZ, _P]),
    "emusv_correlation": (_I, [_I, _I, _P, _P, _P, _SZ, _P]),
    "emusv_krylov_workspace_bytes": (_SZ, [_I, _I, _I]),
    "emusv_krylov_step": (_I, [_I, _I, _D, _P, _P, _P, _P, _P, _P, _D, _D, _I, _I, _P, _SZ,
                               ctypes.POINTER(KrylovInfo), _P]),
    "emusv_adjoint_workspace_bytes": (_SZ, [_I, _I, _I]),
    "emusv_adjoint_step": (_I, [_I, _I, _D, _P, _P, _P, _P, _P, _P, _D, _I, _P, _P, _P, _P, _P, _SZ,
                                _P]),
    "emusv_hpsi_noisy": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "emusv_arnoldi_workspace_bytes": (_SZ, [_I, _I, _I]),
    "emusv_arnoldi_step": (_I, [_I, _I, _D, _P, _P, _P, _P, _P, _P, _P, _D, _D, _I, _I, _P, _SZ,
                                ctypes.POINTER(KrylovInfo), _P]),
    "emusv_qubit_densities_scratch_bytes": (_SZ, [_I]),
    "emusv_qubit_densities": (_I, [_I, _I, _P, _P, _P, _SZ, _P]),
    "emusv_apply_1q": (_I, [_I, _I, _P, _I, _P, _P]),
    "emusv_pchip_eval": (_I, [_I, _P, _I, _P, _I64, _I, _P, _P, _I64, _P]),
    "emusv_lindblad_apply": (_I, [_I, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P]),
    "emusv_lindblad_workspace_bytes": (_SZ, [_I, _I, _I]),
    "emusv_lindblad_arnoldi_step": (_I, [_I, _I, _D, _P, _P, _P, _P, _I, _P, _P, _P, _D, _D, _I, _I,
                                         _P, _SZ, ctypes.POINTER(KrylovInfo), _P]),
    "emusv_dm_scratch_bytes": (_SZ, [_I, _I]),
    "emusv_dm_energy": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "emusv_dm_diagonal_amplitudes": (_I, [_I, _I, _P, _P, _P]),
    "emusv_sample_scratch_bytes": (_SZ, [_I]),
    "emusv_sample": (_I, [_I, _I, _P, _I, _P, _P, _P, _SZ, _P]),
    "emusv_batch_max_qubits": (_I, []),
    "emusv_batch_workspace_bytes": (_SZ, [_I, _P, _P, _I, _I, _I]),
    "emusv_batch_prepare": (_I, [_I, _P, _P, _P, _I, _P, _P, _P, _P, _P, _D, _D, _I, _I, _I, _P,
                                 _SZ, _P]),
    "emusv_batch_launch": (_I, [_I, _I, _I, _P, _P]),
    "emusv_batch_launch_steps": (_I, [_I, _I, _I, _I, _I, _P, _P, _I, _P, _P]),
    "emusv_batch_set_engine": (_I, [_P, _I]),
    "emusv_batch_adjoint_workspace_bytes": (_SZ, [_I, _P, _P, _I, _I, _I]),
    "emusv_batch_adjoint_prepare": (_I, [_I, _P, _P, _P, _I, _P, _P, _P, _P, _D, _I, _I, _I, _P,
                                         _SZ, _P]),
    "emusv_batch_adjoint_launch": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "emusv_batch_adjoint_iterations": (_I, [_I, _P, _P, _P]),
    "emusv_batch_set_barrier_test": (_I, [_P, ctypes.c_longlong, _I]),
    "emusv_batch_max_blocks_per_sm": (_I, [_I, _I]),
    "emusv_batch_results": (_I, [_I, _I, _P, _P, _P, _P]),
    "emusv_vec_dot": (_I, [_I64, _I, _P, _P, _P, _P, _SZ, _P]),
    "emusv_vec_axpy": (_I, [_I64, _I, _P, _P, _P, _P]),
    "emusv_vec_combine": (_I, [_I64, _I, _I, _P, _P, _P, _P]),
    "emusv_dense_expm_scratch_bytes": (_SZ, [_I]),
    "emusv_dense_expm_col": (_I, [_I, _P, _P, _P, _SZ, _P]),
    "emusv_tridiag_scratch_bytes": (_SZ, []),
    "emusv_tridiag_expm_col": (_I, [_I, _P, _P, _P, _P, _P, _SZ, _P]),
    "emusv_profile_begin": (None, [_I]),
    "emusv_profile_end": (_I, [_P, _P, _I]),
}

_lib = None


class WorkspaceTooSmall(Exception):
    """Raised internally when the Krylov basis outgrew its workspace (then retried)."""


class NonFiniteError(FloatingPointError, RecursionError):
    """A NaN or infinity met in a reduction (EMUSV_NONFINITE).  The reference's Lanczos loop
    (emu_base/math/krylov_exp.py:49-131) never converges on a non-finite state and raises
    RecursionError once it reaches max_krylov_dim; the device detects the value at once, so
    this error is both a FloatingPointError and, for callers written against the
    reference, a RecursionError."""


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the library (no GPU needed) and declare every exported signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError(
                f"emulators_b200: CUDA library {path} is missing; build it with "
                "`python -m emulators_b200.build` (there is no CPU fallback)")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def status_message(code: int) -> str:
    return load().emusv_status_string(code).decode()


def check(code: int, what: str) -> None:
    if code == OK:
        return
    msg = f"{what}: {status_message(code)}"
    if code == NOT_CONVERGED:
        raise RecursionError("exponentiation algorithm did not converge to precision in "
                             "allotted number of steps.")
    if code == BAD_ARGUMENT:
        raise ValueError(msg)
    if code == NONFINITE:
        raise NonFiniteError(msg)
    if code == WORKSPACE_TOO_SMALL:
        raise WorkspaceTooSmall(msg)
    if code == TIMEOUT:
        raise TimeoutError(msg)
    raise RuntimeError(msg)


# ---------------------------------------------------------------- tensor helpers
def dtype_code(dt: torch.dtype) -> int:
    if dt == torch.complex128:
        return C128
    if dt == torch.complex64:
        return C64
    raise TypeError(f"emulators_b200 vectors must be complex128 or complex64, got {dt}")


def require_cuda_vector(v: torch.Tensor, name: str = "vector") -> torch.Tensor:
    if not isinstance(v, torch.Tensor) or not v.is_cuda:
        raise RuntimeError(
            f"emulators_b200: {name} must be a CUDA tensor; this implementation runs on the "
            "GPU only (no CPU fallback)")
    dtype_code(v.dtype)
    if not v.is_contiguous():
        v = v.contiguous()
    return v


def nqubits_of(v: torch.Tensor) -> int:
    n = v.numel().bit_length() - 1
    if v.dim() != 1 or n < 1 or (1 << n) != v.numel():
        raise ValueError(f"state vector length must be a power of two >= 2, got {tuple(v.shape)}")
    if n > MAX_QUBITS:
        raise ValueError(f"at most {MAX_QUBITS} qubits are supported, got {n}")
    return n


def host_f64(t, n: int | None = None, name: str = "parameter") -> np.ndarray:
    """Real float64 host copy of a parameter tensor/array (complex inputs: real part,
    as the pulser adapter passes real values in complex128 tensors)."""
    if isinstance(t, torch.Tensor):
        t = t.detach()
        if t.is_complex():
            t = t.real
        a = t.to("cpu", torch.float64).contiguous().numpy()
    else:
        a = np.asarray(t)
        if np.iscomplexobj(a):
            a = a.real
        a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.size != n:
        raise ValueError(f"{name}: expected {n} values, got {a.size}")
    return a


def ptr(a) -> int:
    if isinstance(a, torch.Tensor):
        return a.data_ptr()
    return a.ctypes.data


def stream_of(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


_scratch: dict = {}


def scratch(device: torch.device, nbytes: int) -> torch.Tensor:
    """Per-device reduction scratch (grown on demand, reused across calls on the same
    stream order)."""
    key = (device.type, device.index)
    buf = _scratch.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=device)
        _scratch[key] = buf
    return buf
