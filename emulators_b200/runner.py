"""Run a synthetic workload (emulators_b200.workloads) through the public backend API and
collect the observables the parity tests and benchmarks compare."""

from __future__ import annotations

import numpy as np
import torch

from .sv_backend import Energy, Occupation, SequenceData, SVBackendImpl, SVConfig


def observation_steps(w) -> list[int]:
    return [k for k in range(1, w.nsteps + 1)
            if (w.obs_every and k % w.obs_every == 0) or k == w.nsteps]


def run_workload(w, probes: int = 0, precision: str | None = None, hint: bool = True,
                 nsteps: int | None = None) -> dict:
    """Evolve |g...g> under the workload's drive with SVBackendImpl (occupation and energy
    at the workload's observation steps); returns numpy arrays."""
    if nsteps is not None:
        w = type(w)(**{**w.__dict__, "omega": w.omega[:nsteps], "delta": w.delta[:nsteps],
                       "phi": w.phi[:nsteps]})
    steps_at = observation_steps(w)
    times = [k / w.nsteps for k in steps_at]
    cfg = SVConfig(dt=w.dt * 1000.0, max_krylov_dim=w.max_krylov_dim,
                   krylov_tolerance=w.tolerance, observables=[Occupation(times), Energy(times)],
                   precision=precision or w.precision, krylov_dim_hint=hint)
    impl = SVBackendImpl(cfg, SequenceData.from_workload(w))
    res = impl._run()
    final = impl.state.data.to(torch.complex128).cpu().numpy()
    out = {
        "final": final,
        "occupation": np.stack([o.numpy() for o in res.get("occupation")]),
        "energy": np.array([float(e) for e in res.get("energy")]),
        "steps_at": np.array(steps_at),
        "final_norm": float(np.linalg.norm(final)),
    }
    if probes:
        g = torch.Generator().manual_seed(123)  # the probe vectors of tests/golden/make_golden.py
        P = torch.randn(probes, final.size, dtype=torch.complex128, generator=g).numpy()
        out["probe_overlaps"] = P.conj() @ final
    return out
