"""Krylov exponential exp(op) v, the drop-in for ``emu_base.math.krylov_exp``
(reference emu_base/math/krylov_exp.py:1-131).

Two routes behind the reference signature:

* ``op`` is a :class:`HamiltonianExpOperator` (what the steppers of this package build):
  the whole Lanczos step runs in ``emusv_krylov_step`` -- fused H*psi with FP64 reductions,
  Gram-Schmidt, and the exponential of the extended Krylov matrix with the Expokit error
  estimate computed on the GPU.
* any other callable: the reference's Lanczos (Hermitian) or Arnoldi loop driven from
  Python, with the vector arithmetic in this package's kernels (FP64-accumulated dots,
  axpy, multi-vector combination) and the small exponential (tridiagonal, or dense for
  Arnoldi) on the GPU.
* ``is_hermitian=False`` with a :class:`HamiltonianExpOperator` (the Monte Carlo stepper's
  noisy Hamiltonian): the whole Arnoldi step runs in ``emusv_arnoldi_step``.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import torch

from . import _lib
from .hamiltonian import RydbergHamiltonian

DEFAULT_MAX_KRYLOV_DIM: int = 100
_MAX_SUPPORTED_DIM = 126


class KrylovExpResult:
    """krylov_exp.py:7-20."""

    def __init__(self, result, converged, happy_breakdown, iteration_count):
        assert (not happy_breakdown) or converged
        self.converged = converged
        self.happy_breakdown = happy_breakdown
        self.iteration_count = iteration_count
        self.result = result


class HamiltonianExpOperator:
    """``op(x) = -1j * dt * (H * x)`` -- the operator the reference steppers pass to
    krylov_exp (emu_sv/time_evolution/torch.py:161-162, 308-309, 358-359).  Callable like
    the reference closure; krylov_exp recognises it and runs the fused GPU step."""

    def __init__(self, ham: RydbergHamiltonian, dt: float):
        self.ham = ham
        self.dt = float(dt)

    def __call__(self, x: torch.Tensor) -> torch.Tensor:
        return (-1j * self.dt) * (self.ham * x)


# ------------------------------------------------------------------ fused step
@dataclasses.dataclass
class _StepCache:
    buf: torch.Tensor | None = None
    capacity: int = 0
    last_iters: int = 0
    last_dt: float = 0.0


_caches: dict = {}
# When true, the host first reads the device's convergence decision three iterations
# before the previous step's count (the device tests every iteration), so the hint saves
# host synchronisations without moving the stopping iteration.
use_iteration_hint: bool = True


def _cache(device, n, code, kind: str = "lanczos") -> _StepCache:
    key = (device.index, n, code, kind)
    c = _caches.get(key)
    if c is None:
        c = _caches[key] = _StepCache()
    return c


def release_workspaces() -> None:
    _caches.clear()


def fused_step(op: HamiltonianExpOperator, v: torch.Tensor, exp_tolerance: float,
               norm_tolerance: float, max_krylov_dim: int, out: torch.Tensor | None = None):
    """exp(-i dt H) v in one C-ABI call.  Returns (result, KrylovInfo)."""
    v = _lib.require_cuda_vector(v, "state")
    n = _lib.nqubits_of(v)
    if n != op.ham.nqubits:
        raise ValueError(f"state has {n} qubits, Hamiltonian {op.ham.nqubits}")
    if not 1 <= max_krylov_dim <= _MAX_SUPPORTED_DIM:
        raise ValueError(f"max_krylov_dim must be in 1..{_MAX_SUPPORTED_DIM}")
    code = _lib.dtype_code(v.dtype)
    L = _lib.load()
    c = _cache(v.device, n, code)
    out = torch.empty_like(v) if out is None else out
    info = _lib.KrylovInfo()
    hint = max(0, c.last_iters - 3) if use_iteration_hint else 0
    if c.buf is None:
        c.capacity = min(max_krylov_dim + 1, 32)
    while True:
        need = L.emusv_krylov_workspace_bytes(n, code, c.capacity)
        if c.buf is None or c.buf.numel() < need:
            c.buf = None
            # zeroed once: the step's state block carries the energy shift between steps
            c.buf = torch.zeros(need, dtype=torch.uint8, device=v.device)
        st = L.emusv_krylov_step(n, code, op.dt, *op.ham._params(), v.data_ptr(), out.data_ptr(),
                                 float(exp_tolerance), float(norm_tolerance), int(max_krylov_dim),
                                 hint, c.buf.data_ptr(), c.buf.numel(), info,
                                 _lib.stream_of(v))
        if st == _lib.WORKSPACE_TOO_SMALL:
            if c.capacity >= max_krylov_dim + 1:
                _lib.check(st, "krylov step")
            c.capacity = min(2 * c.capacity, max_krylov_dim + 1)
            continue
        break
    c.last_iters = info.iterations
    if st not in (_lib.OK, _lib.NOT_CONVERGED):
        _lib.check(st, "krylov step")
    return out, info, st


_MAX_ARNOLDI_DIM = 100


def fused_arnoldi_step(op: HamiltonianExpOperator, v: torch.Tensor, exp_tolerance: float,
                       norm_tolerance: float, max_krylov_dim: int, out: torch.Tensor | None = None):
    """exp(-i dt H) v for the (noisy, non-Hermitian) Hamiltonian of ``op`` by Arnoldi in
    one C-ABI call (krylov_exp.py:23-106 with is_hermitian=False)."""
    v = _lib.require_cuda_vector(v, "state")
    n = _lib.nqubits_of(v)
    if n != op.ham.nqubits:
        raise ValueError(f"state has {n} qubits, Hamiltonian {op.ham.nqubits}")
    if not 1 <= max_krylov_dim <= _MAX_ARNOLDI_DIM:
        raise ValueError(f"max_krylov_dim must be in 1..{_MAX_ARNOLDI_DIM} for Arnoldi")
    code = _lib.dtype_code(v.dtype)
    L = _lib.load()
    c = _cache(v.device, n, code, "arnoldi")
    out = torch.empty_like(v) if out is None else out
    info = _lib.KrylovInfo()
    # the device tests convergence from the hint on; the previous count predicts this
    # one only for the same step length (the Monte Carlo stepper's bracketing steps vary)
    same_dt = abs(op.dt) == c.last_dt
    hint = max(0, c.last_iters - 3) if (use_iteration_hint and same_dt) else 0
    if c.buf is None:
        c.capacity = min(max_krylov_dim + 1, 32)
    noise = op.ham._noise_ptr()
    while True:
        need = L.emusv_arnoldi_workspace_bytes(n, code, c.capacity)
        if c.buf is None or c.buf.numel() < need:
            c.buf = None
            # zeroed once: the state block carries the energy shift between steps
            c.buf = torch.zeros(need, dtype=torch.uint8, device=v.device)
        st = L.emusv_arnoldi_step(n, code, op.dt, *op.ham._params(), noise, v.data_ptr(),
                                  out.data_ptr(), float(exp_tolerance), float(norm_tolerance),
                                  int(max_krylov_dim), hint, c.buf.data_ptr(), c.buf.numel(), info,
                                  _lib.stream_of(v))
        if st == _lib.WORKSPACE_TOO_SMALL:
            if c.capacity >= max_krylov_dim + 1:
                _lib.check(st, "arnoldi step")
            c.capacity = min(2 * c.capacity, max_krylov_dim + 1)
            continue
        break
    c.last_iters = info.iterations
    c.last_dt = abs(op.dt)
    if st not in (_lib.OK, _lib.NOT_CONVERGED):
        _lib.check(st, "arnoldi step")
    return out, info, st


def fused_lindblad_step(ham, dt: float, rho: torch.Tensor, exp_tolerance: float,
                        norm_tolerance: float, max_krylov_dim: int):
    """exp(-i dt L) rho for a RydbergLindbladian by Arnoldi over the 4^N vector in one
    C-ABI call (EvolveDensityMatrix: implementations.py:87-120)."""
    rho = ham._check(rho)
    n = ham.nqubits
    if not 1 <= max_krylov_dim <= _MAX_ARNOLDI_DIM:
        raise ValueError(f"max_krylov_dim must be in 1..{_MAX_ARNOLDI_DIM} for Arnoldi")
    code = _lib.dtype_code(rho.dtype)
    L = _lib.load()
    c = _cache(rho.device, n, code, "lindblad")
    out = torch.empty_like(rho)
    info = _lib.KrylovInfo()
    same_dt = abs(dt) == c.last_dt
    hint = max(0, c.last_iters - 3) if (use_iteration_hint and same_dt) else 0
    if c.buf is None:
        c.capacity = min(max_krylov_dim + 1, 32)
    while True:
        need = L.emusv_lindblad_workspace_bytes(n, code, c.capacity)
        if c.buf is None or c.buf.numel() < need:
            c.buf = None
            c.buf = torch.zeros(need, dtype=torch.uint8, device=rho.device)
        st = L.emusv_lindblad_arnoldi_step(n, code, float(dt), *ham._params(),
                                           len(ham.pulser_lindblads), _lib.ptr(ham._ops),
                                           rho.data_ptr(), out.data_ptr(), float(exp_tolerance),
                                           float(norm_tolerance), int(max_krylov_dim), hint,
                                           c.buf.data_ptr(), c.buf.numel(), info, _lib.stream_of(rho))
        if st == _lib.WORKSPACE_TOO_SMALL:
            if c.capacity >= max_krylov_dim + 1:
                _lib.check(st, "lindblad step")
            c.capacity = min(2 * c.capacity, max_krylov_dim + 1)
            continue
        break
    c.last_iters = info.iterations
    c.last_dt = abs(dt)
    if st not in (_lib.OK, _lib.NOT_CONVERGED):
        _lib.check(st, "lindblad step")
    return out, info, st


# ------------------------------------------------------------------ generic Lanczos
def _dot(a: torch.Tensor, b: torch.Tensor, res: torch.Tensor, sc: torch.Tensor) -> None:
    _lib.check(_lib.load().emusv_vec_dot(a.numel(), _lib.dtype_code(a.dtype), a.data_ptr(),
                                         b.data_ptr(), res.data_ptr(), sc.data_ptr(), sc.numel(),
                                         _lib.stream_of(a)), "dot")


def _axpy(alpha: complex, x: torch.Tensor, y: torch.Tensor) -> None:
    al = np.array([alpha.real, alpha.imag], dtype=np.float64)
    _lib.check(_lib.load().emusv_vec_axpy(x.numel(), _lib.dtype_code(x.dtype), al.ctypes.data,
                                          x.data_ptr(), y.data_ptr(), _lib.stream_of(x)), "axpy")


def tridiag_expm_col(d: np.ndarray, up: np.ndarray, lo: np.ndarray, device) -> torch.Tensor:
    """exp(A) e_0 for a complex tridiagonal A on the GPU (device complex128 [m])."""
    m = len(d)
    L = _lib.load()
    dd, uu, ll = (np.ascontiguousarray(a, dtype=np.complex128) for a in (d, up, lo))
    x = torch.empty(m, dtype=torch.complex128, device=device)
    sc = _lib.scratch(device, L.emusv_tridiag_scratch_bytes())
    _lib.check(L.emusv_tridiag_expm_col(m, dd.ctypes.data, uu.ctypes.data, ll.ctypes.data,
                                        x.data_ptr(), sc.data_ptr(), sc.numel(),
                                        torch.cuda.current_stream(device).cuda_stream),
               "tridiagonal exponential")
    return x


def _combine(coef: torch.Tensor, V: list[torch.Tensor]) -> torch.Tensor:
    M = torch.stack(V)
    out = torch.empty_like(V[0])
    c = coef.to(torch.complex128).contiguous()
    _lib.check(_lib.load().emusv_vec_combine(V[0].numel(), _lib.dtype_code(V[0].dtype), len(V),
                                             c.data_ptr(), M.data_ptr(), out.data_ptr(),
                                             _lib.stream_of(V[0])), "combine")
    return out


def dense_expm_col(T: np.ndarray, device) -> torch.Tensor:
    """exp(T) e_0 for a small dense complex matrix on the GPU (device complex128 [m])."""
    m = T.shape[0]
    L = _lib.load()
    a = np.ascontiguousarray(T, dtype=np.complex128)
    x = torch.empty(m, dtype=torch.complex128, device=device)
    nb = L.emusv_dense_expm_scratch_bytes(m)
    if nb == 0:
        raise ValueError(f"dense exponential of a {m} x {m} matrix: at most "
                         f"{_MAX_ARNOLDI_DIM + 2} rows")
    sc = _lib.scratch(device, nb)
    _lib.check(L.emusv_dense_expm_col(m, a.ctypes.data, x.data_ptr(), sc.data_ptr(), sc.numel(),
                                      torch.cuda.current_stream(device).cuda_stream),
               "dense exponential")
    return x


def _tri_parts(T: np.ndarray, m: int):
    d = np.array([T[k, k] for k in range(m)], dtype=np.complex128)
    up = np.array([T[k - 1, k] if k > 0 else 0 for k in range(m)], dtype=np.complex128)
    lo = np.array([T[k + 1, k] if k < m - 1 else 0 for k in range(m)], dtype=np.complex128)
    return d, up, lo


def _generic_krylov(op, v: torch.Tensor, is_hermitian: bool, exp_tolerance, norm_tolerance,
                    max_krylov_dim):
    """krylov_exp.py:23-106 for any callable ``op`` (a vector or tensor of any shape):
    Lanczos (Gram-Schmidt against the last two vectors) for a Hermitian op, Arnoldi (against
    every vector, T upper Hessenberg) otherwise; the vector arithmetic and the small
    exponentials (tridiagonal, or dense for Arnoldi) on the GPU."""
    v = _lib.require_cuda_vector(v, "vector")
    shape = v.shape
    v = v.reshape(-1)
    L = _lib.load()
    sc = _lib.scratch(v.device, L.emusv_scratch_bytes(1, 0))
    res = torch.empty(2, dtype=torch.float64, device=v.device)

    def dot(a, b) -> complex:
        _dot(a, b, res, sc)
        r = res.cpu()
        return complex(r[0].item(), r[1].item())

    def expm(m: int) -> torch.Tensor:  # exp(T[:m, :m]) e_0
        if is_hermitian:
            return tridiag_expm_col(*_tri_parts(T, m), v.device)
        return dense_expm_col(T[:m, :m], v.device)

    initial_norm = np.sqrt(dot(v, v).real)  # 43
    v = v / initial_norm  # 44
    V = [v]
    T = np.zeros((max_krylov_dim + 2, max_krylov_dim + 2), dtype=np.complex128)  # 47
    expd = None
    for j in range(max_krylov_dim):
        w = _lib.require_cuda_vector(op(V[-1].reshape(shape)), "op(v)").reshape(-1).clone()  # 50
        n = np.sqrt(dot(w, w).real)  # 52
        k_start = max(0, j - 1) if is_hermitian else 0  # 54
        for k in range(k_start, j + 1):  # 55-58
            ov = dot(V[k], w)
            T[k, j] = ov
            _axpy(-ov, V[k], w)
        n2 = np.sqrt(dot(w, w).real)  # 60
        T[j + 1, j] = n2
        if n2 < norm_tolerance:  # 63-71
            e = expm(j + 1)
            r = initial_norm * _combine(e, V)
            return KrylovExpResult(r.reshape(shape), True, True, j + 1)
        w /= n2
        V.append(w)
        T[j + 2, j + 1] = 1  # 77
        expd = expm(j + 3)  # 78
        e_host = expd.cpu().numpy()
        err1 = abs(e_host[j + 1])
        err2 = abs(e_host[j + 2] * n)
        err = err1 if err1 < err2 else (err1 * err2 / (err1 - err2))
        if err < exp_tolerance:
            r = initial_norm * _combine(expd[: len(V)], V)
            return KrylovExpResult(r.reshape(shape), True, False, j + 1)
    r = initial_norm * _combine(expd[: len(V)], V)
    return KrylovExpResult(r.reshape(shape), False, False, max_krylov_dim)


def krylov_exp_impl(op, v: torch.Tensor, is_hermitian: bool, exp_tolerance: float,
                    norm_tolerance: float, max_krylov_dim: int = DEFAULT_MAX_KRYLOV_DIM
                    ) -> KrylovExpResult:
    """Same contract as krylov_exp.py:23-106 (the input ``v`` becomes invalid)."""
    if not is_hermitian:
        if not isinstance(op, HamiltonianExpOperator):
            if max_krylov_dim > _MAX_ARNOLDI_DIM:
                raise ValueError(f"max_krylov_dim must be in 1..{_MAX_ARNOLDI_DIM} for Arnoldi")
            return _generic_krylov(op, v, False, exp_tolerance, norm_tolerance, max_krylov_dim)
        out, info, st = fused_arnoldi_step(op, v, exp_tolerance, norm_tolerance, max_krylov_dim)
        return KrylovExpResult(out, st == _lib.OK, bool(info.happy_breakdown), info.iterations)
    if isinstance(op, HamiltonianExpOperator):
        if op.ham.noise is not None:
            raise ValueError("a Hamiltonian with the noise term is not Hermitian")
        out, info, st = fused_step(op, v, exp_tolerance, norm_tolerance, max_krylov_dim)
        return KrylovExpResult(out, st == _lib.OK, bool(info.happy_breakdown), info.iterations)
    return _generic_krylov(op, v, True, exp_tolerance, norm_tolerance, max_krylov_dim)


def krylov_exp(op, v: torch.Tensor, exp_tolerance: float, norm_tolerance: float,
               is_hermitian: bool = True, max_krylov_dim: int = DEFAULT_MAX_KRYLOV_DIM
               ) -> torch.Tensor:
    """krylov_exp.py:109-131: raises RecursionError when not converged."""
    r = krylov_exp_impl(op, v, is_hermitian=is_hermitian, exp_tolerance=exp_tolerance,
                        norm_tolerance=norm_tolerance, max_krylov_dim=max_krylov_dim)
    if not r.converged:
        raise RecursionError("exponentiation algorithm did not converge to precision in "
                             "allotted number of steps.")
    return r.result
