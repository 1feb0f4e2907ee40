"""A small, self-contained run of the hot path for profilers (ncu) and quick timing.

    python -m emulators_b200.profile_case [--n 25] [--dtype c64] [--steps 2] [--hpsi 3]
                                          [--max-krylov-dim 100]
    python -m emulators_b200.profile_case --batch 64 --steps 3        # batched engine
    python -m emulators_b200.profile_case --adjoint 8 --dtype c128    # batched adjoint
    python -m emulators_b200.profile_case --arnoldi 2 --n 20 --dtype c128  # noisy Arnoldi

Builds the 2 x n/2 ladder at 5.5 um with the ladder_n26 drive, runs `--hpsi` standalone
H*psi launches and `--steps` Krylov time steps from |g...g>, prints device times.  Sized
so a capture under a profiler ends in seconds (state of 2^n complex amplitudes).
"""

from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import HamiltonianExpOperator, RydbergHamiltonian, _lib
from . import workloads as wl
from .krylov import fused_step


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=25)
    ap.add_argument("--dtype", choices=["c64", "c128"], default="c64")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--hpsi", type=int, default=3)
    ap.add_argument("--max-krylov-dim", type=int, default=100,
                    help="bounds the Krylov basis the step allocates")
    ap.add_argument("--batch", type=int, default=0,
                    help="instead: the first BATCH registers of the 256-register batch "
                         "workload for --steps steps in one persistent launch")
    ap.add_argument("--arnoldi", type=int, default=0,
                    help="instead: ARNOLDI Arnoldi steps of the noisy ladder workload cut to "
                         "--n qubits (complex128 unless --dtype c64)")
    ap.add_argument("--adjoint", type=int, default=0,
                    help="instead: ADJOINT parameter sets of the N=16 ring gradient "
                         "workload, 4 segments: forward, one checkpoint-segment "
                         "recomputation and two batched adjoint steps")
    a = ap.parse_args(argv)
    if a.batch:
        return _batch_case(a)
    if a.adjoint:
        return _adjoint_case(a)
    if a.arnoldi:
        return _arnoldi_case(a)
    dev = torch.device("cuda", 0)
    dt_ = torch.complex64 if a.dtype == "c64" else torch.complex128
    n = a.n
    pos = wl.ladder(n // 2, 5.5) if n % 2 == 0 else wl.chain(n, 5.5)
    U = torch.as_tensor(wl.interaction_matrix(pos))
    H = RydbergHamiltonian(torch.full((n,), 4.0), torch.full((n,), -9.0), torch.zeros(n), U, dev)
    v = torch.zeros(1 << n, dtype=dt_, device=dev)
    v[0] = 1.0
    out = {}
    if a.hpsi:
        x = torch.randn(1 << n, dtype=dt_, device=dev)
        y = torch.empty_like(x)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.hpsi):
            _lib.check(_lib.load().emusv_hpsi(n, _lib.dtype_code(dt_), *H._params(), x.data_ptr(),
                                              y.data_ptr(), torch.cuda.current_stream().cuda_stream),
                       "hpsi")
        e1.record()
        torch.cuda.synchronize()
        out["hpsi_ms"] = e0.elapsed_time(e1) / a.hpsi
        del x, y
    iters = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        v, info, st = fused_step(HamiltonianExpOperator(H, 0.005), v, 1e-10, 1e-10,
                                  a.max_krylov_dim)
        _lib.check(st, "step")
        iters.append(info.iterations)
    e1.record()
    torch.cuda.synchronize()
    out.update({"n": n, "dtype": a.dtype, "step_ms": e0.elapsed_time(e1) / max(a.steps, 1),
                "iterations": iters, "norm": float(torch.linalg.vector_norm(v))})
    print(json.dumps(out))
    assert np.isfinite(out["norm"])
    return 0


def _batch_case(a) -> int:
    import dataclasses

    from .batch import BatchEvolution

    k = a.steps
    regs = [dataclasses.replace(w, omega=w.omega[:k], delta=w.delta[:k], phi=w.phi[:k])
            for w in wl.batch_256()[:a.batch]]
    b = BatchEvolution(regs, precision=a.dtype)
    tb = 9 if a.dtype == "c64" else 8
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b.reset()
    b.prepare(tb, 40)
    e0.record()
    b.launch(2)
    e1.record()
    status, iters = b.results()
    print(json.dumps({"registers": a.batch, "steps": k, "ms": e0.elapsed_time(e1),
                      "iterations_mean": float(iters[iters > 0].mean()),
                      "failed": int((status != 0).sum())}))
    return 0


def _arnoldi_case(a) -> int:
    from .krylov import fused_arnoldi_step

    w, ops = wl.noisy_ladder_n22()
    n = a.n - (a.n % 2)
    dev = torch.device("cuda", 0)
    dt_ = torch.complex64 if a.dtype == "c64" else torch.complex128
    noise = -0.5j * sum(L.conj().T @ L for L in ops)
    U = torch.as_tensor(wl.interaction_matrix(wl.ladder(n // 2, 5.5)))
    H = RydbergHamiltonian(torch.full((n,), 4.0), torch.full((n,), -9.0), torch.zeros(n), U, dev,
                           noise=torch.as_tensor(noise))
    v = torch.zeros(1 << n, dtype=dt_, device=dev)
    v[0] = 1.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    its = []
    e0.record()
    for _ in range(a.arnoldi):
        v, info, st = fused_arnoldi_step(HamiltonianExpOperator(H, w.dt), v, 1e-10, 1e-10, 100)
        _lib.check(st, "arnoldi")
        its.append((info.iterations, info.second_rounds))
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"n": n, "dtype": a.dtype, "step_ms": e0.elapsed_time(e1) / a.arnoldi,
                      "iterations_second_rounds": its}))
    return 0


def _adjoint_case(a) -> int:
    from .gradients import PulseGradientBatch

    gw = wl.ring_n16_grad()
    S = a.adjoint
    b = PulseGradientBatch(gw.U, gw.dt, gw.omega_seg[:S, :4], gw.delta_seg[:S, :4],
                           gw.steps_per_segment, gw.target, precision=a.dtype, tile_bits=9,
                           blocks_per_sm=1, max_krylov_dim=120)
    b.forward()
    occ = b.occupations()
    n = b.nsets << b.n
    b.g.copy_(b._seed(occ).reshape(-1))
    first, length = 32, 8
    b.work.copy_(b.hist.view(-1, n)[1])
    b._launch_f(first, length - 1, b.work, b.rec, 1)
    for k in (7, 6):
        b._launch_a(first + k, b.rec.view(-1, n)[k - 1], b.g, b.g2)
        b.g, b.g2 = b.g2, b.g
    torch.cuda.synchronize()
    print(json.dumps({"sets": S, "status": b.status[first + 6].tolist()}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
