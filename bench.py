"""Benchmark: N=26 time steps/s of the emu-sv Krylov step on one B200 (complex64 vectors,
FP64 Krylov scalars), with the H*psi roofline, an end-to-end number through the public
backend API, and the CPU baseline.  One JSON line on stdout (rank 0).

Workload (ladder_n26): 2x13 ladder at 5.5 um, C6 = 5420158.53, Omega = 4 rad/us,
delta -10 -> 10 rad/us over 2 us, dt = 5 ns (400 steps), tolerance 1e-10, from |g...g>.
A bench step is one time step exp(-i dt H(t_k)) psi.  Timed steps continue the pulse
after the warm-up steps.  The state (512 MiB) and every Krylov vector are larger than
the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (torchrun, one rank per GPU) every rank evolves its own replica of the
workload ("replicas only": a single state is not sharded), `value` is the sum of steps
over ranks divided by the max over ranks of the timed region.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "N=26 steps/s & batched adjoint grads/s vs plain GPU at err<=1e-6; H·ψ HBM GB/s"
UNIT = "steps/s"


def peaks() -> tuple[float, str]:
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes (read + write) of one Lanczos iteration at N=26, complex64: ncu's
# dram__bytes_read.sum + dram__bytes_write.sum of the iteration's three kernels at N=25
# (python -m emulators_b200.profile_case --n 25 --steps 1 --hpsi 0 --max-krylov-dim 20,
# launches 4-6 of k_pass_(lz|high): 1610.8 MB read, 669.5 MB written), doubled.  A constant
# of the kernels it was measured on; the CUDA-event split reports the streamed units live.
ITERATION_TRAFFIC_N26_C64 = 2 * (1610.8 + 669.5) * 1e6


def log(msg: str) -> None:
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ replicas
def replica_rate(elapsed_s: float, steps: int, world: int, dist, device) -> tuple[float, float]:
    """Whole-job rate of `world` independent replicas that each took `steps` steps: the
    time is the maximum over ranks (one all-reduce after the timed region, nothing inside
    it), the rate world * steps / that time."""
    if dist is not None and world > 1:
        import torch

        t = torch.tensor([float(elapsed_s)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_s = float(t.item())
    return elapsed_s, world * steps / elapsed_s


# ------------------------------------------------------------------ our arm
def run_ours(args, rank: int, world: int, local_rank: int) -> dict | None:
    import torch

    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian, _lib, krylov
    from emulators_b200 import workloads as wl
    from emulators_b200.krylov import fused_step

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    w = wl.ladder_n26()
    n, D = w.nqubits, 1 << w.nqubits
    vdtype = torch.complex64
    es = 8
    L = _lib.load()
    krylov.use_iteration_hint = True
    U = torch.as_tensor(w.U)

    def ham(k):
        k = k % w.nsteps
        return RydbergHamiltonian(torch.as_tensor(w.omega[k]), torch.as_tensor(w.delta[k]),
                                  torch.as_tensor(w.phi[k]), U, dev)

    a = torch.zeros(D, dtype=vdtype, device=dev)
    a[0] = 1.0
    b = torch.empty_like(a)
    iters = []

    def step(k, src, dst):
        _, info, st = fused_step(HamiltonianExpOperator(ham(k), w.dt), src, w.tolerance,
                                 w.tolerance, w.max_krylov_dim, out=dst)
        _lib.check(st, "krylov step")
        iters.append(info.iterations)

    W, K = args.warmup, args.steps
    for k in range(W):
        step(k, a, b)
        a, b = b, a
    torch.cuda.synchronize()
    iters.clear()

    # ---- timed region: K steps, inputs resident in HBM
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    L.emusv_profile_begin(0)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        for k in range(W, W + K):
            step(k, a, b)
            a, b = b, a
        e1.record(stream)
        torch.cuda.synchronize()
    ms_by = (np.zeros(9)).astype(np.float64)
    launches = np.zeros(9, dtype=np.int64)
    L.emusv_profile_end(ms_by.ctypes.data, launches.ctypes.data, 9)
    elapsed, value = replica_rate(e0.elapsed_time(e1) / 1e3, K, world, dist, dev)
    if dist:
        dist.barrier()
    timed_iters = list(iters)
    log(f"timed: {K} steps in {elapsed:.4f} s -> {value:.3f} steps/s, iterations {timed_iters}")

    # ---- profiled pass (not part of `value`): per-kernel device time by kind
    iters.clear()
    KP = min(K, 6)
    L.emusv_profile_begin(1)
    for k in range(W + K, W + K + KP):
        step(k, a, b)
        a, b = b, a
    torch.cuda.synchronize()
    pms = np.zeros(9)
    pl = np.zeros(9, dtype=np.int64)
    L.emusv_profile_end(pms.ctypes.data, pl.ctypes.data, 9)
    # One Lanczos iteration (H-first order) = one or two strided pass H kernels (kind 7: the
    # flips of the bits above the pass-L tile; 2 vector units for the first, 3 for a second
    # that adds to the first's sums) + the recurrence pass L (kind 0: read v_j, the pass H
    # sums and v_{j-1}, write w; 4 units); per step one read-only energy pass over v_0
    # (kind 8, 1 unit).  Algorithmic bytes per iteration: H*psi 2 D s + recurrence 4 D s.
    m_total = max(int(sum(iters)), 1)
    nsteps_p = max(len(iters), 1)
    iter_s = (pms[0] + pms[7]) / m_total / 1e3
    passl_s = pms[0] / max(pl[0], 1) / 1e3
    passh_s = pms[7] / max(pl[7], 1) / 1e3 if pl[7] else 0.0
    hbm, which = peaks()
    alg_iter = 6 * D * es
    achieved = alg_iter / iter_s / 1e9
    total_ms = pms.sum()
    kinds = ["hpsi_pass_low", "orth", "small", "combine", "obs", "adjoint", "batch", "hpsi_pass_high",
             "hpsi_energy_pass"]
    shares = {kinds[i]: round(pms[i] / total_ms, 4) for i in range(9) if pl[i]}
    h_per_iter = pl[7] / m_total
    h_units = 2.0 if h_per_iter < 1.5 else 5.0  # one H pass: 2 units; two: 2 + 3
    iter_units = h_units + 4
    e0_s = pms[8] / max(pl[8], 1) / 1e3 if pl[8] else 0.0
    per_pass = {
        "pass_low": {"ms": round(passl_s * 1e3, 4), "units_mean": 4.0,
                     "note": "recurrence pass L: read v_j, the pass H sums, v_{j-1}; write w "
                             "(4 D s)",
                     "GB/s": round(4 * D * es / passl_s / 1e9, 1),
                     "frac": round(4 * D * es / passl_s / 1e9 / hbm, 4)},
        "energy_pass": {"ms": round(e0_s * 1e3, 4), "units": 1.0, "launches": int(pl[8]),
                        "note": "once per step: <v_0, (D - sigma + X_low) v_0> (read v_0, 1 D s)",
                        "GB/s": round(D * es / e0_s / 1e9, 1) if e0_s else None,
                        "frac": round(D * es / e0_s / 1e9 / hbm, 4) if e0_s else None},
        "pass_high": {"ms": round(passh_s * 1e3, 4),
                      "units_mean": round(h_units / max(h_per_iter, 1e-9), 3),
                      "launches_per_iteration": round(h_per_iter, 2),
                      "GB/s": round(h_units / h_per_iter * D * es / passh_s / 1e9, 1) if passh_s else None,
                      "frac": round(h_units / h_per_iter * D * es / passh_s / 1e9 / hbm, 4) if passh_s else None},
        "iteration": {"ms": round(iter_s * 1e3, 4), "streamed_units": round(iter_units, 3),
                      "streamed_GB/s": round(iter_units * D * es / iter_s / 1e9, 1),
                      "streamed_frac": round(iter_units * D * es / iter_s / 1e9 / hbm, 4)},
    }
    log(f"profiled: ms by kind {pms.round(3).tolist()} launches {pl.tolist()}; "
        f"Lanczos iteration {iter_s * 1e3:.4f} ms = {achieved:.1f} GB/s algorithmic; {per_pass}")

    # ---- H*psi alone (standalone launches, for the kernel roofline at both precisions)
    hstand = {}
    for name, dt_ in (("c64", torch.complex64), ("c128", torch.complex128)):
        v = torch.randn(D, dtype=dt_, device=dev)
        o = torch.empty_like(v)
        H = ham(0)
        for _ in range(2):
            H * v
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 10
        L.emusv_profile_begin(0)  # launch counts only
        s0.record()
        for _ in range(reps):
            L.emusv_hpsi(n, _lib.dtype_code(dt_), *H._params(), v.data_ptr(), o.data_ptr(),
                         torch.cuda.current_stream().cuda_stream)
        s1.record()
        torch.cuda.synchronize()
        hl = np.zeros(8, dtype=np.int64)
        L.emusv_profile_end(None, hl.ctypes.data, 8)
        t1 = s0.elapsed_time(s1) / 1e3 / reps
        es_ = 8 if name == "c64" else 16
        byts = 2 * D * es_
        # vector units streamed per H*psi: pass L 2 (read, write), each H pass 3 (read the
        # vector and the partial sums, write)
        units = (2 * hl[0] + 3 * hl[7]) / reps
        hstand[name] = {"ms": round(t1 * 1e3, 4), "GB/s": round(byts / t1 / 1e9, 1),
                        "frac": round(byts / t1 / 1e9 / hbm, 4),
                        "passes": int((hl[0] + hl[7]) // reps), "streamed_units": float(units),
                        "streamed_GB/s": round(units * D * es_ / t1 / 1e9, 1),
                        "streamed_frac": round(units * D * es_ / t1 / 1e9 / hbm, 4)}
        del v, o

    # ---- energy moments (emusv_expect: <psi|H|psi>, ||H psi||^2) of the N=26 state
    emom = {}
    for name, dt_ in (("c64", torch.complex64),):
        v = torch.randn(D, dtype=dt_, device=dev)
        v /= torch.linalg.vector_norm(v)
        H = ham(0)
        res = torch.empty(3, dtype=torch.float64, device=dev)
        code_ = _lib.dtype_code(dt_)
        sc = torch.empty(L.emusv_scratch_bytes(n, code_), dtype=torch.uint8, device=dev)
        strm = torch.cuda.current_stream().cuda_stream

        def mom():
            _lib.check(L.emusv_expect(n, code_, *H._params(), v.data_ptr(), res.data_ptr(),
                                      sc.data_ptr(), sc.numel(), strm), "expect")

        for _ in range(2):
            mom()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 10
        s0.record()
        for _ in range(reps):
            mom()
        s1.record()
        torch.cuda.synchronize()
        t1 = s0.elapsed_time(s1) / 1e3 / reps
        es_ = 8 if name == "c64" else 16
        # pass H x2 (read psi 2x, read/write the scratch vector 3x) + the moments pass
        # (read psi and the scratch vector): 7 vector units
        emom[name] = {"ms": round(t1 * 1e3, 4), "streamed_units": 7,
                      "streamed_GB/s": round(7 * D * es_ / t1 / 1e9, 1),
                      "streamed_frac": round(7 * D * es_ / t1 / 1e9 / hbm, 4),
                      "read_psi_GB/s": round(D * es_ / t1 / 1e9, 1),
                      "note": "<psi|H|psi> and ||H psi||^2 (energy, variance, second "
                              "moment) of a random N=26 state; CUDA events, 10 calls"}
        del v, sc

    # ---- end-to-end through the public backend API, host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(w, W, K, dev, dist, world)

    result = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": round(elapsed / K * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 vectors + f64 scalars", "data": "synthetic",
        "config": {"workload": "ladder_n26: N=26 2x13 ladder 5.5um, Omega=4, delta -10->10 "
                               "over 2us, dt=5ns, tol=1e-10, complex64/FP64",
                   "nqubits": n, "dt_ns": 5.0, "tolerance": w.tolerance,
                   "krylov_iterations_mean": round(float(np.mean(timed_iters)), 2),
                   "steps_window": [W, W + K - 1],
                   "krylov_iterations_per_s": round(sum(timed_iters) / elapsed * world, 3),
                   "l2": "state and Krylov vectors (512 MiB each) exceed L2; no flush",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm",
                     "kernel": "Lanczos iteration = k_pass_high x2 (flips of the bits above "
                               "the pass-L tile) + k_pass_lz (H v formed on chip, three-term "
                               "recurrence, FP64 reductions); achieved = 6*D*8 algorithmic "
                               "bytes (H*psi 2 D s + recurrence 4 D s) / iteration time",
                     "achieved": round(achieved, 1), "peak": hbm, "peak_source": which,
                     "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "traffic": int(ITERATION_TRAFFIC_N26_C64) if n == 26 and es == 8 else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the "
                                       "iteration's three kernels at N=25, x2 (profiles/"
                                       "lanczos_iteration_h_first_n24_n25_c64.md)",
                     "algorithmic_bytes_per_launch": alg_iter,
                     "avg_launch_ms": round(iter_s * 1e3, 4),
                     "per_kernel": per_pass,
                     "kernel_time_shares": shares},
        "gpu_launches": int(launches.sum()),
        "clocks": clk.summary(),
        "secondary": {"hpsi_standalone": hstand, "energy_moments": emom},
        "e2e": e2e,
    }
    if not args.no_plain and world == 1:
        plain = plain_torch_c128(w, dev, steps=2, warm=W)
        plain["ours_c64_over_plain"] = round(value / world / plain["steps_per_s"], 2)
        result["secondary"]["plain_torch_c128_gpu"] = plain
        log(f"plain complex128 torch path: {plain}")
    if not args.no_c128 and world == 1:
        result["secondary"]["ladder_n26_c128"] = ladder_c128(dev, W)
        log(f"ladder_n26 complex128: {result['secondary']['ladder_n26_c128']}")
        result["secondary"]["lattice_n20_c128"] = lattice_c2(dev)
        log(f"lattice_n20 complex128: {result['secondary']['lattice_n20_c128']}")
    if not args.no_batch and world == 1:
        result["secondary"]["batch_256_c64"] = batch_c4(dev)
        log(f"batch: {result['secondary']['batch_256_c64']}")
        result["secondary"]["ring_n16_gradients_c128"] = grads_c5(dev)
        log(f"gradients: {result['secondary']['ring_n16_gradients_c128']}")
    if not args.no_noisy and world == 1:
        result["secondary"]["noisy_ladder_n22_c128"] = noisy_mc(dev)
        log(f"noisy: {result['secondary']['noisy_ladder_n22_c128']}")
    if not args.no_noisy and world == 1:
        result["secondary"]["lindblad_ladder_n12_c128"] = lindblad_dm(dev)
        log(f"lindblad: {result['secondary']['lindblad_ladder_n12_c128']}")
        result["secondary"]["drive_preparation_pchip"] = drive_prep(dev)
        log(f"drive preparation: {result['secondary']['drive_preparation_pchip']}")
    if not args.no_precision and world == 1:
        result["secondary"]["precision"] = precision_check(w, dev)
        log(f"precision: {result['secondary']['precision']}")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(w, args.cpu_seconds, start=W)
    if dist:
        dist.destroy_process_group()
    return result if rank == 0 else None


def run_e2e(w, W, K, dev, dist, world) -> dict:
    """Same metric through SVBackendImpl: initial state from pinned host memory, per-step
    host drive samples, the per-step norm read the reference loop does, occupation and
    energy at the workload's observation times, final state back to pinned host memory."""
    import torch

    from emulators_b200 import StateVector
    from emulators_b200.sv_backend import Energy, Occupation, SequenceData, SVBackendImpl, SVConfig

    n, D = w.nqubits, 1 << w.nqubits
    sl = slice(W, W + K)
    sub = type(w)(**{**w.__dict__, "omega": w.omega[sl], "delta": w.delta[sl], "phi": w.phi[sl]})
    data = SequenceData.from_workload(sub)
    host0 = torch.zeros(D, dtype=torch.complex64).pin_memory()
    host0[0] = 1.0
    host_out = torch.empty(D, dtype=torch.complex64).pin_memory()
    obs_at = [k / K for k in range(1, K + 1) if k % max(1, w.obs_every // 10) == 0 or k == K]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    init = StateVector(host0.to(dev, non_blocking=True))
    cfg = SVConfig(dt=w.dt * 1000, krylov_tolerance=w.tolerance, precision="c64",
                   observables=[Occupation(obs_at), Energy(obs_at)], initial_state=init)
    impl = SVBackendImpl(cfg, data)
    res = impl._run()
    host_out.copy_(impl.state.data, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    el, rate = replica_rate(e0.elapsed_time(e1) / 1e3, K, world, dist, dev)
    n_obs = len(res.get("occupation"))
    h2d = (D * 8 + K * (3 * n + n * n) * 8) / K
    d2h = (D * 8 + K * 8 + n_obs * (n + 1) * 8) / K
    return {"value": round(rate, 4), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "wall_s": round(wall, 3),
            "api": "SVBackendImpl(SVConfig(precision='c64'), SequenceData)._run()",
            "observations": n_obs}


# ------------------------------------------------------------------ complex128 at N=26
def ladder_c128(dev, W: int, K: int = 6) -> dict:
    """The headline workload in complex128 vectors: W untimed steps, then K steps timed with
    CUDA events (state resident in HBM), and the Lanczos iteration's roofline from the
    library's per-kind device times over 3 further steps (6 D s algorithmic bytes, s = 16)."""
    import torch

    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian, _lib, krylov
    from emulators_b200 import workloads as wl
    from emulators_b200.krylov import fused_step

    w = wl.ladder_n26()
    n, D = w.nqubits, 1 << w.nqubits
    L = _lib.load()
    U = torch.as_tensor(w.U)
    krylov.release_workspaces()
    torch.cuda.empty_cache()
    a = torch.zeros(D, dtype=torch.complex128, device=dev)
    a[0] = 1.0
    b = torch.empty_like(a)
    iters = []

    def step(k):
        nonlocal a, b
        H = RydbergHamiltonian(torch.as_tensor(w.omega[k]), torch.as_tensor(w.delta[k]),
                               torch.as_tensor(w.phi[k]), U, dev)
        _, info, st = fused_step(HamiltonianExpOperator(H, w.dt), a, w.tolerance, w.tolerance,
                                 w.max_krylov_dim, out=b)
        _lib.check(st, "krylov step")
        iters.append(info.iterations)
        a, b = b, a

    for k in range(W):
        step(k)
    torch.cuda.synchronize()
    iters.clear()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(W, W + K):
        step(k)
    e1.record()
    torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    timed = list(iters)
    iters.clear()
    L.emusv_profile_begin(1)
    for k in range(W + K, W + K + 3):
        step(k)
    torch.cuda.synchronize()
    pms = np.zeros(9)
    pl = np.zeros(9, dtype=np.int64)
    L.emusv_profile_end(pms.ctypes.data, pl.ctypes.data, 9)
    iter_s = (pms[0] + pms[7]) / max(sum(iters), 1) / 1e3
    hbm, which = peaks()
    ach = 6 * D * 16 / iter_s / 1e9
    del a, b
    krylov.release_workspaces()
    torch.cuda.empty_cache()
    return {"steps_per_s": round(K / el, 4), "ms_per_step": round(el / K * 1e3, 3),
            "steps_window": [W, W + K - 1], "krylov_iterations": timed,
            "krylov_iterations_per_s": round(sum(timed) / el, 3),
            "roofline": {"achieved": round(ach, 1), "peak": hbm, "peak_source": which,
                         "unit": "GB/s", "frac": round(ach / hbm, 4),
                         "iteration_ms": round(iter_s * 1e3, 4),
                         "note": "Lanczos iteration (pass H kernels + recurrence pass L), "
                                 "6*D*16 algorithmic bytes"},
            "note": "complex128 vectors, same kernels and step window as the complex64 headline"}


# ------------------------------------------------------------------ the N=20 4x5 lattice
def lattice_c2(dev, plain_budget_s: float = 20.0) -> dict:
    """The plain-method drop-in configuration: N=20 4x5 lattice at 6 um, sin^2 Omega (peak
    2 pi), delta -15 -> 15 over 3 us, dt = 10 ns (300 steps), complex128, Krylov dim <= 30,
    tolerance 1e-10, occupation and energy every 100 ns.  Ours: the whole run through
    SVBackendImpl (state and results on the host at the end), CUDA events; the plain
    complex128 torch path (reference algorithm in plain tensor ops) with the same
    observables on the first steps of the same run, and ours on that same window."""
    import torch

    from emulators_b200 import krylov
    from emulators_b200 import workloads as wl
    from emulators_b200.runner import run_workload

    w = wl.lattice_n20()
    krylov.release_workspaces()
    run_workload(w, nsteps=10)  # workspaces and kernels warm
    torch.cuda.synchronize()

    def timed(nsteps=None):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        r = run_workload(w, nsteps=nsteps)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3, time.perf_counter() - t0, r

    el, wall, r = timed()
    # the plain path: as many steps of the same run as fit the budget (a multiple of the
    # observation interval), from |g...g>
    probe = plain_torch_c128(w, dev, steps=w.obs_every, warm=0, obs_every=w.obs_every)
    per_step = 1.0 / probe["steps_per_s"]
    kp = int(max(1, min(w.nsteps // w.obs_every, plain_budget_s / per_step / w.obs_every))) * w.obs_every
    plain = plain_torch_c128(w, dev, steps=kp, warm=0, obs_every=w.obs_every)
    el_w, _, _ = timed(kp)
    krylov.release_workspaces()
    return {"steps": w.nsteps, "steps_per_s": round(w.nsteps / el, 3),
            "ms_per_step": round(el / w.nsteps * 1e3, 4), "wall_s": round(wall, 3),
            "observations": int(len(r["energy"])),
            "api": "SVBackendImpl(SVConfig(precision='c128'), SequenceData)._run(), "
                   "occupation + energy every 10 steps",
            "window_steps": kp, "ours_window_steps_per_s": round(kp / el_w, 3),
            "plain_torch_c128_gpu": plain,
            "ours_over_plain_same_window": round((kp / el_w) / plain["steps_per_s"], 2)}


# ------------------------------------------------------------------ precision form check
def precision_check(w, dev) -> dict:
    """The whole workload (all steps) in complex64/FP64 and in complex128 through the same
    kernels, from |g...g>: infidelity and state error of the complex64 run every 100
    steps against the complex128 run (itself checked against the oracle in the tests)."""
    import torch

    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian, krylov
    from emulators_b200.krylov import fused_step

    n, D = w.nqubits, 1 << w.nqubits
    U = torch.as_tensor(w.U)
    states = {}
    rates = {}
    snaps = {torch.complex64: [], torch.complex128: []}
    for dt_ in (torch.complex64, torch.complex128):
        krylov.release_workspaces()
        a = torch.zeros(D, dtype=dt_, device=dev)
        a[0] = 1.0
        b = torch.empty_like(a)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(w.nsteps):
            H = RydbergHamiltonian(torch.as_tensor(w.omega[k]), torch.as_tensor(w.delta[k]),
                                   torch.as_tensor(w.phi[k]), U, dev)
            _, info, st = fused_step(HamiltonianExpOperator(H, w.dt), a, w.tolerance,
                                     w.tolerance, w.max_krylov_dim, out=b)
            a, b = b, a
            if (k + 1) % 100 == 0 or k + 1 == w.nsteps:
                snaps[dt_].append(a.to(torch.complex128).cpu())
        torch.cuda.synchronize()
        rates[dt_] = w.nsteps / (time.perf_counter() - t0)
        states[dt_] = a
        del b
    krylov.release_workspaces()
    infid, errs = [], []
    for x, y in zip(snaps[torch.complex64], snaps[torch.complex128]):
        ov = abs(torch.vdot(y, x).item()) ** 2 / (torch.vdot(x, x).real.item() * torch.vdot(y, y).real.item())
        infid.append(float(f"{1 - ov:.3e}"))
        errs.append(float(f"{torch.linalg.vector_norm(x - y).item():.3e}"))
    return {"steps": w.nsteps, "every": 100, "infidelity_c64_vs_c128": infid,
            "state_error_c64_vs_c128": errs,
            "c64_steps_per_s_untimed_loop": round(rates[torch.complex64], 3),
            "c128_steps_per_s_untimed_loop": round(rates[torch.complex128], 3),
            "note": "errors of the complex64 run against this package's complex128 run of "
                    "the same kernels (not against the FP64 oracle, which cannot run 400 "
                    "steps at N=26; the complex128 steps match the oracle's to 1e-10 in "
                    "the GPU tests, up to N=23)"}


# ------------------------------------------------------------------ plain complex128 GPU path
def plain_torch_c128(w, dev, steps: int = 2, warm: int = 1, obs_every: int = 0) -> dict:
    """The plain complex128 GPU path: the reference's algorithm written with plain torch
    tensor ops (the reference modules themselves are not on the GPU machine) -- per-qubit
    strided-view flips, the diagonal rebuilt every step from view slices, the Lanczos loop
    with the tridiagonal matrix, its exponential and the error estimate on the host and one
    host synchronisation per reduction (emu_sv/hamiltonian.py:69-162,
    emu_base/math/krylov_exp.py:23-131).  Timed over `steps` steps after `warm`."""
    import scipy.linalg
    import torch

    n, D = w.nqubits, 1 << w.nqubits
    U = np.asarray(w.U)

    def diagonal(de):
        d = torch.zeros(D, dtype=torch.complex128, device=dev)
        for i in range(n):
            d.view(2 ** i, 2, -1)[:, 1] -= float(de[i])
            for j in range(i + 1, n):
                if U[i, j] != 0.0:
                    d.view(2 ** i, 2, 2 ** (j - i - 1), 2, -1)[:, 1, :, 1] += float(U[i, j])
        return d

    def hpsi(v, d, coef):
        out = d * v
        for i in range(n):
            vv, oo = v.view(2 ** i, 2, -1), out.view(2 ** i, 2, -1)
            oo[:, 1] += coef[i] * vv[:, 0]
            oo[:, 0] += np.conj(coef[i]) * vv[:, 1]
        return out

    def step(k, psi):
        coef = 0.5 * np.asarray(w.omega[k]) * np.exp(1j * np.asarray(w.phi[k]))
        d = diagonal(w.delta[k])
        dt, tol, mk = w.dt, w.tolerance, w.max_krylov_dim
        nrm = torch.linalg.vector_norm(psi).item()
        V = [psi / nrm]
        T = np.zeros((mk + 2, mk + 2), dtype=np.complex128)
        for j in range(mk):
            wv = (-1j * dt) * hpsi(V[-1], d, coef)
            nn = torch.linalg.vector_norm(wv).item()
            for kk in range(max(0, j - 1), j + 1):
                ov = torch.vdot(V[kk], wv).item()
                T[kk, j] = ov
                wv -= ov * V[kk]
            n2 = torch.linalg.vector_norm(wv).item()
            T[j + 1, j] = n2
            if n2 < tol:
                e = scipy.linalg.expm(T[:j + 1, :j + 1])[:, 0]
                its.append(j + 1)
                return nrm * sum(complex(e[i]) * V[i] for i in range(j + 1))
            V.append(wv / n2)
            T[j + 2, j + 1] = 1.0
            e = scipy.linalg.expm(T[:j + 3, :j + 3])[:, 0]
            err1, err2 = abs(e[j + 1]), abs(e[j + 2] * nn)
            err = err1 if err1 < err2 else err1 * err2 / (err1 - err2)
            if err < tol:
                its.append(j + 1)
                return nrm * sum(complex(e[i]) * V[i] for i in range(j + 2))
        raise RecursionError("plain path did not converge")

    def observe(k, psi):
        # occupation per qubit and Re <psi|H psi> on the host, as the reference's
        # callbacks return them (custom_callback_implementations.py:30-47,
        # hamiltonian.py:164-172); the step's H (midpoint samples of step k)
        coef = 0.5 * np.asarray(w.omega[k]) * np.exp(1j * np.asarray(w.phi[k]))
        occ = torch.stack([psi.view(2 ** i, 2, -1)[:, 1].abs().pow(2).sum() for i in range(n)]).cpu()
        en = torch.vdot(psi, hpsi(psi, diagonal(w.delta[k]), coef)).real.cpu()
        return occ, en

    its: list[int] = []
    psi = torch.zeros(D, dtype=torch.complex128, device=dev)
    psi[0] = 1.0
    for k in range(warm):
        psi = step(k, psi)
        if obs_every and (k + 1) % obs_every == 0:
            observe(k, psi)
    its.clear()
    if dev.type != "cuda":  # host run (checks of this function only)
        for k in range(warm, warm + steps):
            psi = step(k, psi)
        return {"state": psi}
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(warm, warm + steps):
        psi = step(k, psi)
        if obs_every and (k + 1) % obs_every == 0:
            observe(k, psi)
    e1.record()
    torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    del psi
    torch.cuda.empty_cache()
    return {"steps_per_s": round(steps / el, 4), "unit": UNIT,
            "krylov_iterations": list(its),
            "krylov_iterations_per_s": round(sum(its) / el, 4),
            "sample": f"steps {warm}..{warm + steps - 1} of {w.name} in complex128 after "
                      f"{warm} warm-up step(s) (the timed window of the ours arm starts at the "
                      f"same step)" + (f", occupation and energy every {obs_every} steps"
                                       if obs_every else "") + "; CUDA events"}


# ------------------------------------------------------------------ plain complex128 GPU gradients
def _plain_lanczos(op, v, tol: float, mk: int):
    """Lanczos basis and tridiagonal matrix of `op` from `v` with the reference's stopping
    rule (emu_base/math/double_krylov.py:59-113): host tridiagonal matrix, Expokit error
    estimate from the extended matrix's exponential, RecursionError past `mk`."""
    import scipy.linalg
    import torch

    V = [v / torch.linalg.vector_norm(v)]
    T = np.zeros((mk + 2, mk + 2), dtype=np.complex128)
    for j in range(mk):
        w = op(V[-1])
        nn = torch.linalg.vector_norm(w).item()
        for k in range(max(0, j - 1), j + 1):
            ov = torch.vdot(V[k], w).item()
            T[k, j] = ov
            w -= ov * V[k]
        n2 = torch.linalg.vector_norm(w).item()
        T[j + 1, j] = n2
        if n2 < tol:
            return V, T[:len(V), :len(V)].copy()
        V.append(w / n2)
        T[j + 2, j + 1] = 1.0
        e = scipy.linalg.expm(T[:j + 3, :j + 3])[:, 0]
        err1, err2 = abs(e[j + 1]), abs(e[j + 2] * nn)
        err = err1 if err1 < err2 else err1 * err2 / (err1 - err2)
        if err < tol:
            return V, T[:len(V), :len(V)].copy()
    raise RecursionError("plain Lanczos did not converge")


def plain_torch_grads_c128(gw, dev, p: int = 0, steps: int = 20) -> dict:
    """Neel-loss gradients of parameter set `p` over its first `steps` steps, the reference's
    way with plain torch tensor ops in complex128 (the reference modules are not on the
    GPU machine): per step the Lanczos exponential forward (states kept); then per step
    backwards the double Krylov decomposition (two Lanczos bases, the block exponential of
    the two tridiagonal matrices joined at one corner, emu_base/math/double_krylov.py:5-56),
    E = dS^T V_s, the per-qubit derivative operators dH/dOmega = 0.5 sigma^x and
    dH/dDelta = -n (emu_sv/time_evolution/torch.py:36-119,327-351) and exp(+i dt H) on the
    incoming gradient (torch.py:362-371).  Drives are real (phi = 0), as in the workload."""
    import scipy.linalg
    import torch

    n, D = gw.nqubits, 1 << gw.nqubits
    U = np.asarray(gw.U)
    dt, tol, mk = gw.dt, gw.tolerance, 120
    ctype = torch.complex128

    def diagonal(de):
        d = torch.zeros(D, dtype=ctype, device=dev)
        for i in range(n):
            d.view(2 ** i, 2, -1)[:, 1] -= float(de)
            for j in range(i + 1, n):
                if U[i, j] != 0.0:
                    d.view(2 ** i, 2, 2 ** (j - i - 1), 2, -1)[:, 1, :, 1] += float(U[i, j])
        return d

    def hpsi(v, d, half_om):
        out = d * v
        for i in range(n):
            vv, oo = v.view(2 ** i, 2, -1), out.view(2 ** i, 2, -1)
            oo[:, 1] += half_om * vv[:, 0]
            oo[:, 0] += half_om * vv[:, 1]
        return out

    def expm_apply(op, v):  # krylov_exp (emu_base/math/krylov_exp.py:23-131)
        nrm = torch.linalg.vector_norm(v).item()
        V, T = _plain_lanczos(op, v, tol, mk)
        e = scipy.linalg.expm(T)[:, 0]
        return nrm * sum(complex(e[i]) * V[i] for i in range(len(V)))

    seg_of = [k // gw.steps_per_segment for k in range(steps)]
    om, de = gw.omega_seg[p], gw.delta_seg[p]
    if dev.type == "cuda":
        torch.cuda.synchronize()
    t0 = time.perf_counter()
    states = []
    s = torch.zeros(D, dtype=ctype, device=dev)
    s[0] = 1.0
    for k in range(steps):
        states.append(s)
        d = diagonal(de[seg_of[k]])
        half = 0.5 * float(om[seg_of[k]])
        s = expm_apply(lambda x: (-1j * dt) * hpsi(x, d, half), s)
    sf = s.detach().clone().requires_grad_(True)
    occ = torch.stack([torch.linalg.vector_norm(sf.view(2 ** i, 2, -1)[:, 1]) ** 2 for i in range(n)])
    loss = torch.mean((occ - torch.as_tensor(gw.target, device=dev)) ** 2)
    (g,) = torch.autograd.grad(loss, sf)
    g_om = torch.zeros(gw.nsegments, dtype=torch.float64, device=dev)
    g_de = torch.zeros_like(g_om)
    for k in reversed(range(steps)):
        d = diagonal(de[seg_of[k]])
        half = 0.5 * float(om[seg_of[k]])
        fwd = lambda x: (-1j * dt) * hpsi(x, d, half)
        Vs, Ts = _plain_lanczos(fwd, states[k], tol, mk)
        Vg, Tg = _plain_lanczos(fwd, g, tol, mk)
        ms = len(Vs)
        big = scipy.linalg.block_diag(Ts, Tg)
        big[0, ms] = torch.linalg.vector_norm(states[k]).item() * torch.linalg.vector_norm(g).item()
        dS = torch.as_tensor(scipy.linalg.expm(big)[:ms, ms:], device=dev)
        E = dS.mT @ torch.stack(Vs)
        G = torch.stack(Vg).conj()
        mg = E.shape[0]
        for i in range(n):
            Ev = E.view(mg, 2 ** i, 2, -1)
            r = torch.zeros_like(Ev)  # dH/dOmega_i E
            r[:, :, 1] = 0.5 * Ev[:, :, 0]
            r[:, :, 0] = 0.5 * Ev[:, :, 1]
            g_om[seg_of[k]] += (-1j * dt * torch.tensordot(G, r.view(mg, D))).real
            r = -Ev.clone()  # dH/dDelta_i E
            r[:, :, 0] = 0.0
            g_de[seg_of[k]] += (-1j * dt * torch.tensordot(G, r.view(mg, D))).real
        g = expm_apply(lambda x: (1j * dt) * hpsi(x, d, half), g)
    go, gd = g_om.cpu().numpy(), g_de.cpu().numpy()
    el = time.perf_counter() - t0
    return {"loss": float(loss.detach()), "g_omega": go, "g_delta": gd, "s": el,
            "occupation": occ.detach().cpu().numpy()}


# ------------------------------------------------------------------ batched workloads
def batch_c4(dev, per_instance_sample: int = 8) -> dict:
    """The 256-register batch (N in 12..18, 150 steps each, complex64/FP64) in one
    persistent launch replayed from a CUDA graph, with the autotuned launch shape, next to
    the same registers stepped one at a time through the single-register API."""
    import torch

    from emulators_b200 import HamiltonianExpOperator, RydbergHamiltonian, _lib
    from emulators_b200 import workloads as wl
    from emulators_b200.batch import BatchEvolution, autotune
    from emulators_b200.krylov import fused_step

    regs = wl.batch_256()
    b = BatchEvolution(regs, precision="c64")
    t = autotune(b)
    b.reset()
    b.prepare(t.tile_bits, t.capacity)
    b.capture(t.blocks_per_sm)
    times = []
    for _ in range(3):  # first replay warms up
        b.reset()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.replay()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    status, iters = b.results()
    el = min(times[1:])
    total = int(b.nsteps.sum())
    # per-instance path: the first registers, every step, one fused step call each
    per = regs[:per_instance_sample]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    nst = 0
    for w in per:
        n = w.nqubits
        s = torch.zeros(1 << n, dtype=torch.complex64, device=dev)
        s[0] = 1.0
        for k in range(w.nsteps):
            H = RydbergHamiltonian(torch.as_tensor(w.omega[k]), torch.as_tensor(w.delta[k]),
                                   torch.as_tensor(w.phi[k]), torch.as_tensor(w.U), dev)
            s, _, st = fused_step(HamiltonianExpOperator(H, w.dt), s, w.tolerance, w.tolerance, 100)
            _lib.check(st, "step")
            nst += 1
    e1.record()
    torch.cuda.synchronize()
    el1 = e0.elapsed_time(e1) / 1e3
    # scale the sample's time by its share of the batch's amplitude-steps
    amp = lambda ws: sum((1 << w.nqubits) * w.nsteps for w in ws)  # noqa: E731
    per_rate = nst / el1
    per_rate_weighted = total / (el1 * amp(regs) / amp(per))
    # algorithmic bytes of the batch: (7 m + 1) D s per register-step (m Lanczos iterations
    # of H*psi 2 D s + recurrence 4 D s, the combination (m + 1) D s), s = 8
    dims = np.array([1 << w.nqubits for w in regs], dtype=np.float64)
    alg = float(((7.0 * iters + 1.0) * (iters > 0)).sum(axis=1) @ dims) * 8.0
    hbm, which = peaks()
    return {"instances": len(regs), "instance_steps": total,
            "ms": round(el * 1e3, 2), "instance_steps_per_s": round(total / el, 1),
            "roofline": {"algorithmic_bytes": int(alg), "achieved": round(alg / el / 1e9, 1),
                         "peak": hbm, "peak_source": which, "unit": "GB/s",
                         "frac": round(alg / el / 1e9 / hbm, 4),
                         "note": "(7 m + 1) D s per register-step from the recorded "
                                 "iteration counts"},
            "launch": {"tile_bits": t.tile_bits, "blocks_per_sm": t.blocks_per_sm,
                       "krylov_capacity": t.capacity, "autotune_ms": t.ms,
                       "graph": "one cooperative persistent kernel replayed from a CUDA graph"},
            "krylov_iterations_mean": round(float(iters[iters > 0].mean()), 2),
            "all_converged": bool((status == 0).all()),
            "per_instance_api": {"sample": f"first {len(per)} registers, all steps, one "
                                           f"emusv_krylov_step each",
                                 "instance_steps_per_s": round(per_rate, 1),
                                 "batch_equivalent_instance_steps_per_s": round(per_rate_weighted, 1)},
            "speedup_vs_per_instance": round((total / el) / per_rate_weighted, 1)}


def grads_c5(dev) -> dict:
    """Neel-loss gradients of the 64 parameter sets of the N=16 ring (20 segments x 10
    steps, complex128, checkpoints every 16 steps) through the batched forward and adjoint,
    next to one set through the per-step autograd.Function chain and to the plain
    complex128 torch path of the reference's per-step backward (`plain_torch_grads_c128`)."""
    import torch

    from emulators_b200 import DifferentiableStateVectorEvolution as DSE
    from emulators_b200 import workloads as wl
    from emulators_b200.gradients import PulseGradientBatch

    gw = wl.ring_n16_grad()
    kd = 120  # some steps of some sets need more than 100 Krylov vectors
    b = PulseGradientBatch(gw.U, gw.dt, gw.omega_seg, gw.delta_seg, gw.steps_per_segment,
                           gw.target, precision="c128", checkpoint_every=16,
                           tolerance=gw.tolerance, max_krylov_dim=kd)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    loss, go, gd, _ = b.loss_and_grad()
    e1.record()
    torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    # one set, per-step Function chain
    n = gw.nqubits
    p = 0
    om = torch.tensor(gw.omega_seg[p], device=dev, requires_grad=True)
    de = torch.tensor(gw.delta_seg[p], device=dev, requires_grad=True)
    U = torch.tensor(gw.U, device=dev)
    zeros = torch.zeros(n, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    e0.record()
    s = torch.zeros(1 << n, dtype=torch.complex128, device=dev)
    s[0] = 1.0
    for seg in range(gw.nsegments):
        for _ in range(gw.steps_per_segment):
            s, _ = DSE.apply(gw.dt, om[seg].expand(n), de[seg].expand(n), zeros, U, s,
                             gw.tolerance, kd)
    occ = torch.stack([torch.linalg.vector_norm(s.view(2**i, 2, -1)[:, 1]) ** 2 for i in range(n)])
    L1 = torch.mean((occ - torch.tensor(gw.target, device=dev)) ** 2)
    g_om, g_de = torch.autograd.grad(L1, (om, de))
    e1.record()
    torch.cuda.synchronize()
    el1 = e0.elapsed_time(e1) / 1e3
    rel = max(float(np.abs(g_om.cpu().numpy() - go[p]).max() / np.abs(go[p]).max()),
              float(np.abs(g_de.cpu().numpy() - gd[p]).max() / np.abs(gd[p]).max()))
    # the plain complex128 torch path (the reference's per-step backward), set 0, first
    # two segments; its rate scaled to all steps of a set
    ps = 2 * gw.steps_per_segment
    plain = plain_torch_grads_c128(gw, dev, p=0, steps=ps)
    plain_gps = 1.0 / (plain["s"] * b.nsteps / ps)
    # algorithmic bytes, an estimate from the recorded forward iteration counts m per
    # set-step (vectors of D s = 2^16 x 16 bytes): a Lanczos basis of m iterations streams
    # (7 m + 1) D s; each step's basis is built by the forward, again by the checkpoint
    # recomputation (all steps but the last of a segment), and twice by the adjoint (the
    # state's basis, of the forward's size, and the incoming gradient's, taken as the same
    # size); the adjoint's post-processing reads both bases and writes and reads the E
    # vectors, (m + 3 m) D s
    m = np.asarray(b.forward_iterations, dtype=np.float64)
    Ds = float(1 << n) * 16.0
    last = (np.arange(b.nsteps) % b.ck) == b.ck - 1
    lz = (7.0 * m + 1.0) * Ds
    alg = float(lz.sum() + lz[:, ~last].sum() + 2.0 * lz.sum() + (4.0 * m * Ds).sum())
    peak, src = peaks()
    roof = {"algorithmic_bytes": alg, "achieved": round(alg / el / 1e9, 1), "peak": peak,
            "peak_source": src, "unit": "GB/s", "frac": round(alg / el / 1e9 / peak, 4),
            "note": "estimate: forward, recomputation and the two adjoint bases at (7 m + 1) "
                    "D s each from the forward's iteration counts, plus 4 m D s of "
                    "post-processing per set-step"}
    return {"sets": b.nsets, "steps": b.nsteps, "s": round(el, 3),
            "grads_per_s": round(b.nsets / el, 3), "max_krylov_dim": kd, "roofline": roof,
            "plain_torch_c128_gpu": {
                "sample": f"set 0, steps 0..{ps - 1} forward and backward (loss after step "
                          f"{ps - 1}), the reference's per-step backward in plain torch ops, "
                          f"complex128; wall time with a synchronize on both sides, rate "
                          f"scaled to {b.nsteps} steps",
                "s": round(plain["s"], 3), "grads_per_s": round(plain_gps, 5)},
            "batched_over_plain": round((b.nsets / el) / plain_gps, 1),
            "per_instance_autograd": {"sample": "set 0, all steps, the per-step autograd "
                                                "Function (fused step forward, adjoint step "
                                                "backward), every step's state kept",
                                      "s": round(el1, 3), "grads_per_s": round(1.0 / el1, 4),
                                      "max_rel_diff_vs_batched": rel},
            "speedup_vs_per_instance": round((b.nsets / el) * el1, 1)}


def noisy_mc(dev, steps: int = 20, cpu_seconds: float = 10.0) -> dict:
    """The Monte Carlo path on noisy_ladder_n22 (N=22, complex128, relaxation + dephasing):
    (1) Arnoldi steps alone at the workload's dt, with the device time split by kernel kind
    and the bandwidth of the orthogonalisation passes; (2) whole EvolveMonteCarlo steps
    (Brent bracketing and quantum jumps included) from |g...g> with seeded draws; (3) the
    oracle's Monte Carlo step on the host for a bounded sample."""
    import random

    import torch

    from emulators_b200 import RydbergHamiltonian, _lib
    from emulators_b200 import workloads as wl
    from emulators_b200.krylov import HamiltonianExpOperator, fused_arnoldi_step
    from emulators_b200.time_evolution import EvolveMonteCarlo
    from oracle import oracle

    w, ops = wl.noisy_ladder_n22()
    n, D, es = w.nqubits, 1 << w.nqubits, 16
    noise = -0.5j * sum(L.conj().T @ L for L in ops)
    U = torch.as_tensor(w.U)

    def ham(k):
        return RydbergHamiltonian(torch.as_tensor(w.omega[k]), torch.as_tensor(w.delta[k]),
                                  torch.as_tensor(w.phi[k]), U, dev, noise=torch.as_tensor(noise))

    L = _lib.load()
    s = torch.zeros(D, dtype=torch.complex128, device=dev)
    s[0] = 1.0
    for k in range(3):  # warm-up
        s, info, _ = fused_arnoldi_step(HamiltonianExpOperator(ham(k), w.dt), s, 1e-10, 1e-10, 100)
    torch.cuda.synchronize()
    L.emusv_profile_begin(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    its = []
    for k in range(3, 3 + steps):
        s, info, st = fused_arnoldi_step(HamiltonianExpOperator(ham(k), w.dt), s, 1e-10, 1e-10, 100)
        _lib.check(st, "arnoldi")
        its.append(info.iterations)
    e1.record()
    torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    pms = np.zeros(8)
    pl = np.zeros(8, dtype=np.int64)
    L.emusv_profile_end(pms.ctypes.data, pl.ctypes.data, 8)
    # algorithmic bytes of the two Gram-Schmidt passes of iteration j (every vector once
    # per pass): dots over w, v~_j and v_0..v_{j-1} (j+2 reads), update (j+2 reads, w' and
    # the corrected v_j written)
    ortho_bytes = sum(sum(2 * (max(j, 1) + 2) + 2 for j in range(m)) for m in its) * D * es
    hbm, which = peaks()
    kinds = ["hpsi_pass_low", "orth", "small", "combine", "obs", "adjoint", "batch", "hpsi_pass_high"]
    tot = pms.sum()
    ortho_gbs = ortho_bytes / (pms[1] / 1e3) / 1e9
    # whole Monte Carlo steps
    random.seed(0)
    mc = EvolveMonteCarlo(100)
    st_ = torch.zeros(D, dtype=torch.complex128, device=dev)
    st_[0] = 1.0
    thr0 = mc.jump_threshold
    jumps = 0
    torch.cuda.synchronize()
    e0.record()
    for k in range(steps):
        before = mc.jump_threshold
        st_, _ = mc.apply(w.dt, torch.as_tensor(w.omega[k]), torch.as_tensor(w.delta[k]),
                          torch.as_tensor(w.phi[k]), U, st_, 1e-10, [torch.as_tensor(o) for o in ops])
        jumps += int(mc.jump_threshold != before)
    e1.record()
    torch.cuda.synchronize()
    el_mc = e0.elapsed_time(e1) / 1e3
    # the oracle's Monte Carlo step on the host, bounded sample
    rnd = random.Random(0)
    thr = rnd.uniform(0.0, 1.0)
    cs = np.zeros(D, dtype=np.complex128)
    cs[0] = 1.0
    t0 = time.perf_counter()
    done = 0
    while done < steps and (done == 0 or time.perf_counter() - t0 < cpu_seconds):
        cs, thr, _ = oracle.monte_carlo_step(rnd, thr, w.dt, w.omega[done], w.delta[done], w.phi[done],
                                             w.U, cs, ops, 1e-10)
        done += 1
    cpu_el = time.perf_counter() - t0
    return {"workload": "noisy_ladder_n22: N=22 2x11 ladder 5.5um, relaxation 0.5/us + "
                        "dephasing 1/us, dt=10ns, complex128",
            "arnoldi_steps_per_s": round(steps / el, 2),
            "arnoldi_iterations_mean": round(float(np.mean(its)), 2),
            "kernel_time_shares": {kinds[i]: round(pms[i] / tot, 4) for i in range(8) if pl[i]},
            "gram_schmidt": {"algorithmic_bytes_per_step": int(ortho_bytes / steps),
                             "GB/s": round(ortho_gbs, 1), "frac": round(ortho_gbs / hbm, 4),
                             "note": "two streaming passes per iteration over w and the "
                                     "basis, the second Gram-Schmidt round lagged into them"},
            "monte_carlo_steps_per_s": round(steps / el_mc, 2),
            "monte_carlo_jumps": jumps,
            "monte_carlo_first_threshold": round(thr0, 6),
            "cpu_baseline": {"value": round(done / cpu_el, 4), "unit": "steps/s",
                             "cores": oracle.num_threads(), "kind": "port",
                             "sample": f"first {done} Monte Carlo step(s) of the workload in "
                                       f"complex128 on the host ({cpu_el:.1f} s)"},
            "speedup_vs_cpu": round((steps / el_mc) / (done / cpu_el), 1)}


def drive_prep(dev, regs: int = 256, qubits: int = 16, T: int = 4000, dt_ns: int = 10,
               cpu_seconds: float = 10.0) -> dict:
    """Drive preparation for a long batched sequence set: amplitude, detuning and phase
    samples of `regs` registers x `qubits` qubits on pulser's 1 ns grid (T knots each),
    PCHIP-interpolated at the midpoints of a dt_ns grid in one launch; next to the oracle's
    numpy PCHIP per signal (the reference loops over qubits and parameters) on the host."""
    import torch

    from emulators_b200.pchip import PCHIP1D
    from oracle import oracle

    rng = np.random.default_rng(11)
    S = 3 * regs * qubits
    t = np.arange(T, dtype=np.float64)
    base = np.sin(np.outer(rng.uniform(0.5, 3.0, S), t) / T) * rng.uniform(0, 10, (S, 1))
    y_host = torch.from_numpy(base).pin_memory()
    tt = np.arange(0, T + 1, dt_ns, dtype=np.float64)
    tm = 0.5 * (tt[:-1] + tt[1:])
    xg = torch.as_tensor(t, device=dev)
    xq = torch.as_tensor(tm, device=dev)
    y = y_host.to(dev)
    f = PCHIP1D(xg, y)
    for _ in range(3):
        f(xq)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    reps = 20
    for _ in range(reps):
        out = f(xq)
    e1.record()
    torch.cuda.synchronize()
    k_ms = e0.elapsed_time(e1) / reps
    # end to end: host samples in, host midpoint samples out
    out_host = torch.empty(S, len(tm), dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(5):
        yd = y_host.to(dev, non_blocking=True)
        o = PCHIP1D(xg, yd)(xq)
        out_host.copy_(o, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / 5
    # host: the oracle's PCHIP per signal, bounded sample
    t0 = time.perf_counter()
    done = 0
    while done < S and (done == 0 or time.perf_counter() - t0 < cpu_seconds):
        oracle.pchip(t, base[done], tm)
        done += 1
    cpu_s = (time.perf_counter() - t0) / done
    ok = bool(np.array_equal(out[:64].cpu().numpy(),
                             np.stack([oracle.pchip(t, base[i], tm) for i in range(64)])))
    return {"workload": f"{regs} registers x {qubits} qubits x 3 parameters = {S} signals, "
                        f"{T} knots (1 ns grid), {len(tm)} midpoints ({dt_ns} ns steps)",
            "kernel_ms": round(k_ms, 4), "signals_per_s": round(S / (k_ms / 1e3), 1),
            "e2e_ms": round(e2e_ms, 3), "e2e_h2d_bytes": int(S * T * 8),
            "e2e_d2h_bytes": int(S * len(tm) * 8),
            "cpu_baseline": {"signals_per_s": round(1.0 / cpu_s, 1), "cores": 1, "kind": "port",
                             "sample": f"first {done} signals, oracle numpy PCHIP"},
            "speedup_e2e_vs_cpu": round((S / (e2e_ms / 1e3)) * cpu_s, 1),
            "first_64_signals_bit_identical_to_oracle": ok}


def lindblad_dm(dev, steps: int = 8) -> dict:
    """The density-matrix path on lindblad_ladder_n12 (a 4^12 density matrix, complex128):
    EvolveDensityMatrix steps through the fused Arnoldi step over the 24-bit vector, next to
    the oracle's dense Lindbladian on the host (one application, timed, times the GPU run's
    Arnoldi iterations per step)."""
    import torch

    from emulators_b200 import _lib
    from emulators_b200.density_matrix import DensityMatrix
    from emulators_b200.time_evolution import EvolveDensityMatrix
    from emulators_b200 import workloads as wl
    from oracle import oracle

    w, ops = wl.lindblad_ladder_n12()
    n = w.nqubits
    U = torch.as_tensor(w.U)
    tops = [torch.as_tensor(L) for L in ops]
    stepper = EvolveDensityMatrix(100)
    rho = DensityMatrix.make(n).data
    its = []

    def step(k, r):
        r, ham = stepper.apply(w.dt, torch.as_tensor(w.omega[k]), torch.as_tensor(w.delta[k]),
                               torch.as_tensor(w.phi[k]), U, r, w.tolerance, tops)
        return r

    for k in range(2):
        rho = step(k, rho)
    torch.cuda.synchronize()
    L = _lib.load()
    L.emusv_profile_begin(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(2, 2 + steps):
        rho = step(k, rho)
    e1.record()
    torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    pms = np.zeros(8)
    pl = np.zeros(8, dtype=np.int64)
    L.emusv_profile_end(pms.ctypes.data, pl.ctypes.data, 8)
    from emulators_b200 import krylov
    iters = krylov._cache(rho.device, n, _lib.dtype_code(rho.dtype), "lindblad").last_iters
    kinds = ["hpsi_pass_low+jumps", "orth", "small", "combine", "obs", "adjoint", "batch",
             "hpsi_pass_high"]
    tot = pms.sum()
    trace = float(DensityMatrix(rho).norm())
    # host: one dense Lindbladian application of the oracle at the same size
    r0 = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    r0[0, 0] = 1.0
    t0 = time.perf_counter()
    oracle.lindbladian_apply(w.omega[0], w.delta[0], w.phi[0], w.U, ops, r0)
    t_apply = time.perf_counter() - t0
    cpu_step_s = t_apply * max(iters, 1)
    return {"workload": "lindblad_ladder_n12: 4^12 density matrix (N=12 2x6 ladder 5.5um), "
                        "relaxation 0.5/us + dephasing 1/us, dt=10ns, complex128",
            "steps_per_s": round(steps / el, 3), "arnoldi_iterations_last_step": iters,
            "trace_after": round(trace, 12),
            "kernel_time_shares": {kinds[i]: round(pms[i] / tot, 4) for i in range(8) if pl[i]},
            "cpu_baseline": {"steps_per_s": round(1.0 / cpu_step_s, 5), "cores": oracle.num_threads(),
                             "kind": "port",
                             "sample": f"one dense Lindbladian application of the oracle at N=12 "
                                       f"({t_apply:.2f} s) x {iters} Arnoldi iterations per step"},
            "speedup_vs_cpu": round((steps / el) * cpu_step_s, 1)}


# ------------------------------------------------------------------ CPU baseline (oracle)
def cpu_baseline(w, budget_s: float, start: int = 0) -> dict:
    """The oracle (C/OpenMP restatement of the reference path, FP64/complex128) timed on
    this host's cores on the same step window as the GPU arm: steps 0..start-1 run untimed
    (the GPU arm's warm-up), then steps from `start` are timed until budget_s."""
    from oracle import oracle

    oracle.build()
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    n = w.nqubits
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1.0
    for k in range(min(start, w.nsteps - 1)):
        s, _, _ = oracle.evolve_step(w.dt, w.omega[k], w.delta[k], w.phi[k], w.U, s,
                                     w.tolerance, w.max_krylov_dim)
    k0 = min(start, w.nsteps - 1)
    t0 = time.perf_counter()
    done = 0
    iters = []
    while k0 + done < w.nsteps:
        k = k0 + done
        s, _, info = oracle.evolve_step(w.dt, w.omega[k], w.delta[k], w.phi[k], w.U, s,
                                        w.tolerance, w.max_krylov_dim)
        iters.append(info.iteration_count)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return {"value": round(done / el, 6), "unit": UNIT, "cores": oracle.num_threads(),
            "kind": "port", "steps_window": [k0, k0 + done - 1],
            "krylov_iterations": iters,
            "krylov_iterations_per_s": round(sum(iters) / el, 4),
            "sample": f"time steps {k0}..{k0 + done - 1} of ladder_n26 (after the GPU arm's "
                      f"{k0} warm-up steps, run untimed here) in complex128 on the host "
                      f"({el:.1f} s, Krylov iterations {iters})"}


# ------------------------------------------------------------------ reference arm
def run_reference(args, rank: int) -> dict | None:
    if rank != 0:
        return None
    from emulators_b200 import workloads as wl

    w = wl.ladder_n26()
    cb = cpu_baseline(w, args.cpu_seconds, start=args.warmup)
    return {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic",
            "config": {"workload": "ladder_n26 (same as the ours arm), reference algorithm "
                                   "restated on the host CPU (oracle port)",
                       "steps_window": cb["steps_window"],
                       "krylov_iterations_per_s": cb["krylov_iterations_per_s"],
                       "steps_note": "the warm-up steps run untimed, then time steps from the "
                                     "same index as the ours arm's timed window run until "
                                     f"{args.cpu_seconds:.0f} s of CPU work"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=30.0)
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain complex128 torch GPU path")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched evolution and batched gradient workloads")
    ap.add_argument("--no-noisy", action="store_true",
                    help="skip the Monte Carlo (noisy Hamiltonian, Arnoldi) workload")
    ap.add_argument("--no-c128", action="store_true",
                    help="skip the complex128 N=26 line and the N=20 lattice line")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the complex64-vs-complex128 run of the whole workload")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
    else:
        out = run_ours(args, rank, world, local_rank)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
