"""A small, self-contained run of the hot path for profilers (ncu) and quick timing.

    python -m emulators_b200.profile_case [--n 25] [--dtype c64] [--steps 2] [--hpsi 3]
                                          [--max-krylov-dim 100]

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
    a = ap.parse_args(argv)
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


if __name__ == "__main__":
    raise SystemExit(main())
