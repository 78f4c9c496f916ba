"""
Benchmark: MD steps/s (SCF + forces) of the Hartree-Fock hot path on B200.

Workload (default, ``--workload h2o32``): (H2O)32 RHF/cc-pVDZ (Cartesian,
800 AOs), 32 rigid waters at seeded random positions in a cube for
1 g/cm^3, XL-BOMD (K = 5, dt = 0.5 fs), CSVR 300 K, tau = 100 fs, seed 1,
default SCF thresholds (dE < 1e-10 Eh, commutator < 1e-7). Precision
(``--precision``): "mixed" (default, the headline) evaluates quartets with
Schwarz product Q1 Q2 < 1e-3 (``--fp32-cutoff``) in FP32 with FP64
accumulation; the plain FP64 path is timed beside it in the same run, and
the energy / force / dipole differences of the two at the starting geometry
are reported (config.error_vs_fp64_at_start).
One step = one MD step: XL-BOMD guess, SCF to convergence, analytic
gradient, Verlet update. ``--workload methanol``: CH3OH RHF/6-31G**
(50 AOs) NVE velocity Verlet at dt = 0.5 fs, 300 K initial velocities.

  value  MD steps/s with positions, densities and the XL-BOMD history
         resident on the device (aimd_b200.md.DeviceXLBOMD), forces from
         the differentiable SCF energy (autograd forward = device SCF,
         backward = derivative kernels). Beside it: SCF iterations/s and
         gradient evaluations/s of each path (CUDA events around the two
         phases of every timed step) and the conserved quantity of the
         thermostatted XL-BOMD run (drift, max deviation) over the steps.
  e2e    MD steps/s through the public API (HFGPUBackend.compute with
         host numpy positions, density guess and results), host<->device
         copies inside the timed region (CUDA events around the steps).
  roofline  the integral-direct J/K build (the dominant kernels): model
         FP64 flops of one ERI pass (per primitive quartet
         2 sum NH(L-n) + 2 NH(Lab) NH(Lcd) n_cd n_kc + 2 NH(Lab) n_ab n_cd n_kc
         over the Schwarz-kept unique block quartets) / average duration,
         against the FP64 peak measured in the same run by a cuBLAS DGEMM;
         the two-electron gradient likewise (bra Hermite order + 1, two
         passes); the mixed-precision build and gradient against the
         measured FP32 SGEMM peak.
  cpu_baseline  the oracle (C + OpenMP restatement of the reference's numba
         path) on the host cores, on the workload itself at the converged
         density of its starting geometry: one full Fock build and one full
         two-electron gradient, measured; MD step = (SCF iterations per
         step) Fock builds + 1 gradient, as the reference rebuilds J/K from
         the whole density every iteration.
  --impl reference  the same oracle, each step a bounded sample (every
         S-th bra pair of one Fock build and one gradient), the MD step
         time estimated from the sampled share of the flop model.

Multi-GPU: replicas only (one independent MD trajectory per rank, no
collective in the data path); value sums the steps of all ranks over the
maximum time.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ab-initio-md_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "MD steps/s (SCF+forces) on 1 B200, mixed vs FP64 kernels at ΔE≤1e-6 Eh"
WORKLOADS = {
    "h2o32": {"desc": "(H2O)32 RHF/cc-pVDZ (800 AOs), XL-BOMD K=5, dt=0.5 fs, CSVR 300 K tau=100 fs, seed 1",
              "basis": "cc-pvdz", "nwater": 32, "xl": True, "thermostat": True},
    "h2o8": {"desc": "(H2O)8 RHF/cc-pVDZ (200 AOs), XL-BOMD K=5, dt=0.5 fs, CSVR 300 K tau=100 fs, seed 1",
             "basis": "cc-pvdz", "nwater": 8, "xl": True, "thermostat": True},
    "methanol": {"desc": "CH3OH RHF/6-31G** (50 AOs), NVE velocity Verlet dt=0.5 fs, 300 K, seed 1",
                 "basis": "6-31g**", "nwater": 0, "xl": False, "thermostat": False},
}


def _geometry(w):
    from aimd_b200 import geometry as G
    if w["nwater"]:
        return G.water_cluster(w["nwater"], seed=1)
    return G.methanol()


def _dist():
    """(rank, world, torch.distributed or None)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world <= 1:
        return 0, 1, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return rank, world, dist


def max_over_ranks(value: float, dist) -> float:
    """Max of a per-rank scalar (the job time of a replicas-only run)."""
    if dist is None:
        return value
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist) -> float:
    if dist is None:
        return value
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while active."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int) -> None:
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self) -> None:
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for nm, flag in zip(names, parts[3:7]):
                if flag.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(buf) -> None:
    buf.add_(1.0)


def fp64_peak_tflops() -> float:
    """Measured FP64 throughput of a cuBLAS DGEMM 8192^3 (best of 5), TFLOP/s."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    return best


def fp32_peak_tflops() -> float:
    """Measured FP32 (CUDA-core, TF32 off) throughput of a cuBLAS SGEMM 8192^3 (best of 5), TFLOP/s."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        torch.matmul(a, b)
        best = 0.0
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.matmul(a, b)
            e.record()
            e.synchronize()
            best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
        return best
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def flop_model_device(eng, basis, thr: float = 1e-12, grad: bool = False) -> tuple[float, float]:
    """
    FP64 flop model of one ERI pass and its primitive-quartet count, from the
    engine's pairs (unique block quartets p1 >= p2 in block-pair index
    order, p1 as bra, Q1 Q2 >= thr), evaluated on the device in row chunks.
    grad=True: the two-electron gradient's model, the same sum with the bra
    Hermite order raised by one (the derivative expansions, R to L + 1),
    counted twice (the bra pass for centres A, B and the ket pass for C; D
    follows by translational invariance).
    """
    import torch
    Q = eng.schwarz()
    npp, _, _ = eng.pair_data()
    nb = eng.nblock
    blk_l = torch.as_tensor(eng.blocks["l"], device="cuda", dtype=torch.int64)
    blk_n = torch.as_tensor(eng.blocks["ncon"], device="cuda", dtype=torch.int64)
    ii, jj = np.tril_indices(nb)
    order = np.lexsort((jj, ii))
    i = torch.as_tensor(ii[order], device="cuda")
    j = torch.as_tensor(jj[order], device="cuda")
    li, lj = blk_l[i], blk_l[j]
    Lp = li + lj
    nc = lambda l: (l + 1) * (l + 2) // 2  # noqa: E731
    nab = (nc(li) * nc(lj)).double()
    ncon = (blk_n[i] * blk_n[j]).double()
    w = torch.as_tensor(npp, device="cuda", dtype=torch.float64)
    NH = lambda L: ((L + 1) * (L + 2) * (L + 3) // 6).double()  # noqa: E731
    rs = torch.tensor([sum((L0 - n + 1) * (L0 - n + 2) * (L0 - n + 3) // 6 for n in range(L0 + 1))
                       for L0 in range(17)], device="cuda", dtype=torch.float64)
    npair = len(ii)
    total = 0.0
    nq = 0.0
    idx = torch.arange(npair, device="cuda")
    chunk = 2048
    for r0 in range(0, npair, chunk):
        p1 = idx[r0:r0 + chunk]
        keep = (Q[p1][:, None] * Q[None, :] >= thr) & (idx[None, :] <= p1[:, None])
        dl = 1 if grad else 0
        Lb = Lp[p1][:, None]
        Lk = Lp[None, :]
        per = (2 * rs[Lb + Lk + dl] + 2 * NH(Lb + dl) * NH(Lk) * nab[None, :] * ncon[None, :]
               + 2 * NH(Lb + dl) * nab[p1][:, None] * nab[None, :] * ncon[None, :])
        if grad:
            per = 2 * per
        ww = w[p1][:, None] * w[None, :]
        total += float((per * ww * keep).sum())
        nq += float((ww * keep).sum())
    return total, nq


def cpu_baseline(sym, pos, basis: str, P: np.ndarray, n_iter: float) -> dict:
    """
    The oracle (C/OpenMP restatement of the reference's numba path) on the
    host cores, on the workload itself: one full integral-direct Fock build
    and one full two-electron gradient at the converged density P of the
    GPU run, both measured. An MD step of the reference is n_iter full Fock
    builds (it rebuilds J/K from the whole density every SCF iteration) and
    one gradient.
    """
    from oracle import hf_oracle as O
    b = O.build_basis(sym, pos, basis)
    O.schwarz_bounds(b)                      # pair data and Q: set-up, outside the timings
    t0 = time.perf_counter()
    O.jk_direct(b, P)
    t_jk = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.two_electron_gradient(b, P, [P], 0.5)
    t_g = time.perf_counter() - t0
    t_step = n_iter * t_jk + t_g
    return {"value": 1.0 / t_step, "unit": "MD steps/s", "cores": O.num_threads(), "kind": "port",
            "sample": (f"oracle (C/OpenMP restatement of the reference's numba path) on the workload itself "
                       f"({b.nao} AOs) at the GPU run's converged density: one full integral-direct Fock build "
                       f"{t_jk:.2f} s and one full two-electron gradient {t_g:.2f} s, both measured; MD step = "
                       f"{n_iter:.2f} Fock builds (SCF iterations per step of the GPU run) + 1 gradient"),
            "fock_build_s": t_jk, "gradient_s": t_g, "scf_iterations_per_s": 1.0 / t_jk,
            "gradient_evaluations_per_s": 1.0 / t_g}


def _reference_density(w, sym, pos, basis):
    """Converged density of the workload's starting geometry for the reference arm."""
    if w["nwater"] == 32:
        from oracle.make_density_fixture import load
        return load(), "oracle SCF density of the starting geometry (fixture, float32)"
    from oracle import hf_oracle as O
    return O.run_scf(sym, pos, basis)["density"], "oracle SCF density of the starting geometry"


def run_reference_arm(args) -> None:
    """
    The reference's path timed on the host cores (the oracle port; the
    reference's own numba code cannot travel to the GPU host). Each step is
    a bounded sample of one MD step of the workload at its converged
    density: the quartets of every S-th bra pair (offset = step mod S) of
    one Fock build and of one two-electron gradient. The step's MD time is
    estimated as (n_iter t_fock + t_grad) / f, with f the sampled share of
    the flop model of one ERI pass; value = 1 / median estimate.
    ms_per_step is the measured wall time of one sample step.
    """
    rank, world, dist = _dist()
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    from oracle import hf_oracle as O
    sym, pos = _geometry(w)
    b = O.build_basis(sym, pos, w["basis"])
    P, dens = _reference_density(w, sym, pos, w["basis"])
    fm = O.flop_model(b)
    per_bra, total = fm["per_bra"], fm["flop"]
    S = args.ref_stride if w["nwater"] >= 32 else 1
    est, wall = [], []
    for k in range(args.warmup + args.steps):
        off = k % S
        t0 = time.perf_counter()
        O.jk_direct(b, P, stride=S, offset=off)
        t_jk = time.perf_counter() - t0
        t1 = time.perf_counter()
        O.two_electron_gradient(b, P, [P], 0.5, stride=S, offset=off)
        t_g = time.perf_counter() - t1
        frac = float(per_bra[off::S].sum()) / total
        if k >= args.warmup:
            est.append((args.iters_per_step * t_jk + t_g) / frac)
            wall.append(t_jk + t_g)
    v = 1.0 / statistics.median(est)
    sample = (f"oracle (C/OpenMP restatement of the reference's numba path), {O.num_threads()} threads, on the "
              f"workload itself ({b.nao} AOs, {dens}): per step the quartets of every {S}-th bra pair of one "
              f"Fock build and of one two-electron gradient ({100.0 / S:.1f} % of the work, share from the flop "
              f"model); MD step = {args.iters_per_step:g} full Fock builds + 1 gradient, estimated as "
              f"(n_iter t_fock + t_grad) / share")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "MD steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(wall),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["desc"], "sample_share_of_md_step": 1.0 / S,
                   "md_step_s_estimated": statistics.median(est),
                   "ms_per_step_meaning": "measured wall time of one sample step (a 1/S share of one MD step)"},
        "cpu_baseline": {"value": v, "unit": "MD steps/s", "cores": O.num_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "MD steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def _md_path(args, sym, pos, vel, w, seed, ndof, fp32_cutoff, l2, dist, local, sample_clocks):
    """Warm-up + K timed steps of the device-resident XL-BOMD loop at one precision."""
    import torch

    from aimd_b200 import md as MD
    from aimd_b200.engine import engine_for
    from aimd_b200.scf import SCFOptions, SCFSolver

    solver = SCFSolver(sym, w["basis"], options=SCFOptions(warn_unconverged=False, fp32_cutoff=fp32_cutoff))
    thermo = MD.CSVR(300.0, 100.0, seed, ndof) if w["thermostat"] else None
    run = MD.DeviceXLBOMD(solver, sym, pos, vel, 0.5, k=5, thermostat=thermo)
    st0 = run.state
    start = {"energy": float(st0.energy), "gradient": run.gradient.detach().clone(),
             "dipole": -torch.einsum("xmn,mn->x", st0.dipole_ints, st0.spin[0] + st0.spin[1])}
    start["density"] = (st0.spin[0] + st0.spin[1]).cpu().numpy()
    for _ in range(args.warmup):
        run.step()
    eng = engine_for(run.state.basis)
    launches0 = eng.launch_count()
    clocks = ClockSampler(local) if sample_clocks else None
    if clocks:
        clocks.start()
    step_ms = []
    conserved = [run.conserved_energy()]
    run.phase_events = []
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    for _ in range(args.steps):
        flush_l2(l2)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        run.step()
        e.record()
        e.synchronize()
        step_ms.append(s.elapsed_time(e))
        conserved.append(run.conserved_energy())
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    launches = eng.launch_count() - launches0
    t_job = max_over_ranks(sum(step_ms) * 1e-3, dist)
    value = sum_over_ranks(float(args.steps), dist) / t_job
    # the two phases of each step: SCF (forward) and gradient (backward)
    scf_s = sum(a.elapsed_time(b) for a, b, _ in run.phase_events) * 1e-3
    grad_s = sum(b.elapsed_time(c) for _, b, c in run.phase_events) * 1e-3
    iters = run.iterations[-args.steps:]
    run.phase_events = None
    # conserved quantity of the thermostatted XL-BOMD run over the timed steps
    ec = np.array(conserved)
    t_ps = np.arange(len(ec)) * 0.5e-3
    drift = {"drift_eh_per_ps": float(np.polyfit(t_ps, ec, 1)[0]) if len(ec) > 1 else 0.0,
             "max_abs_dev_eh": float(np.abs(ec - ec[0]).max()), "span_fs": float(t_ps[-1] * 1e3)}
    return {"value": value, "t_job": t_job, "iters": iters, "launches": launches,
            "clocks": clk, "run": run, "start": start, "scf_iterations_per_s": float(sum(iters)) / scf_s,
            "gradient_evaluations_per_s": len(iters) / grad_s, "scf_s_per_step": scf_s / len(iters),
            "gradient_s_per_step": grad_s / len(iters), "conserved": drift}


def run_ours(args) -> None:
    import torch

    from aimd_b200 import md as MD
    from aimd_b200.backend import HFGPUBackend
    from aimd_b200.engine import engine_for

    rank, world, dist = _dist()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    sym, pos = _geometry(w)
    seed = 1 + rank
    vel = MD.maxwell_boltzmann(sym, 300.0, seed)
    ndof = 3 * len(sym) - 3
    l2 = torch.empty(64 * 1024 * 1024, dtype=torch.float64, device="cuda")   # 512 MB > L2
    cutoff = args.fp32_cutoff if args.precision == "mixed" else 0.0

    # ---- value: device-resident MD loop at the requested precision, and the
    # plain FP64 path beside it (same trajectory start, same step count)
    main = _md_path(args, sym, pos, vel, w, seed, ndof, cutoff, l2, dist, local, True)
    ref64 = main if cutoff == 0.0 else _md_path(args, sym, pos, vel, w, seed, ndof, 0.0, l2, dist, local, False)
    value = main["value"]
    run = main["run"]
    iters = main["iters"]
    err = {"energy_eh": abs(main["start"]["energy"] - ref64["start"]["energy"]),
           "force_eh_bohr": float((main["start"]["gradient"] - ref64["start"]["gradient"]).abs().max()),
           "dipole_e_bohr": float((main["start"]["dipole"] - ref64["start"]["dipole"]).abs().max())}

    # ---- rooflines at the last geometry and density: the FP64 J/K build
    # (the dominant kernels) and the FP64 two-electron gradient
    from aimd_b200.gradients import scf_gradient_device
    eng = engine_for(run.state.basis)
    D = (run.state.spin[0] + run.state.spin[1])[None].contiguous()
    flop, nq = flop_model_device(eng, run.state.basis)
    flop_g, _ = flop_model_device(eng, run.state.basis, grad=True)

    def timed_ms(fn, reps=3):
        fn()
        ts = []
        for _ in range(reps):
            flush_l2(l2)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            e.synchronize()
            ts.append(s.elapsed_time(e))
        return statistics.mean(ts)

    jk_ms = timed_ms(lambda: eng.jk_acc(D, 1e-12, 0.0))
    jk_mixed_ms = timed_ms(lambda: eng.jk_acc(D, 1e-12, cutoff)) if cutoff > 0.0 else None
    g_ms = timed_ms(lambda: scf_gradient_device(run.state, 1e-14, 0.0))
    g_mixed_ms = timed_ms(lambda: scf_gradient_device(run.state, 1e-14, cutoff)) if cutoff > 0.0 else None
    peak = fp64_peak_tflops()
    peak32 = fp32_peak_tflops()
    achieved = flop / (jk_ms * 1e-3) / 1e12
    achieved_g = flop_g / (g_ms * 1e-3) / 1e12

    # ---- e2e through the public API (host numpy in and out)
    backend = HFGPUBackend(sym, basis=w["basis"], scf_options={"fp32_cutoff": cutoff})
    thermo2 = MD.CSVR(300.0, 100.0, seed, ndof) if w["thermostat"] else None
    run2 = MD.XLBOMDRun(backend, sym, pos, vel, 0.5, k=5, thermostat=thermo2, xl=w["xl"])
    for _ in range(min(args.warmup, 2)):
        run2.step()
    e2e_steps = max(1, min(args.steps, 10))
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    # CUDA events on the stream the backend launches on; the host work of
    # each step (copies from and to numpy, the MD update) lies between the
    # two events on the device timeline, so it is inside the measurement
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(e2e_steps):
        run2.step()
    ev1.record()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(ev0.elapsed_time(ev1) * 1e-3, dist)
    e2e = sum_over_ranks(float(e2e_steps), dist) / t_e2e
    n = backend.nao
    natm = len(sym)
    h2d = 8 * (3 * natm + n * n)                       # positions + density guess
    d2h = 8 * (4 + 3 * natm + n * n + 3 + 3 * n * n + 2 * n + natm)   # E, grad, D, dipole, SCFResult arrays

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sym, pos, w["basis"], main["start"]["density"], float(np.mean(ref64["iters"])))
    if rank == 0:
        prec = (f"mixed: FP32 quartets for Q1 Q2 < {cutoff:g}, FP64 otherwise, FP64 accumulation"
                if cutoff > 0.0 else "fp64 kernels")

        def path(r):
            return {"value": r["value"], "ms_per_step": 1e3 * r["t_job"] / args.steps,
                    "scf_iterations_per_step": float(np.mean(r["iters"])),
                    "scf_iterations_per_s": r["scf_iterations_per_s"],
                    "gradient_evaluations_per_s": r["gradient_evaluations_per_s"],
                    "scf_ms_per_step": 1e3 * r["scf_s_per_step"],
                    "gradient_ms_per_step": 1e3 * r["gradient_s_per_step"], "conserved_quantity": r["conserved"]}
        line = {
            "metric": METRIC, "value": value, "unit": "MD steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * main["t_job"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32" if cutoff > 0.0 else "f64",
            "data": "synthetic",
            "config": {"workload": w["desc"], "precision": prec, "l2": "flushed (512 MB write) before each step",
                       "parallelism": f"replicas{world}" if world > 1 else "single GPU",
                       "forces": "autograd: scf_energy forward (device SCF) + backward (derivative kernels)",
                       "scf_iterations_per_step": float(np.mean(iters)),
                       "scf_iterations_per_s": main["scf_iterations_per_s"],
                       "gradient_evaluations_per_s": main["gradient_evaluations_per_s"],
                       "conserved_quantity": main["conserved"],
                       "mixed_path": path(main), "fp64_path": path(ref64),
                       "speedup_vs_fp64": value / ref64["value"],
                       "error_vs_fp64_at_start": err},
            "e2e": {"value": e2e, "unit": "MD steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "integral-direct FP64 J/K build (jk_bra_kernel, one launch per (bra, ket) pair class)",
                         "model_flop_per_build": flop, "prim_quartets": nq, "build_ms": jk_ms,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64)",
                         "gradient": {"achieved": achieved_g, "frac": achieved_g / peak, "ms": g_ms,
                                      "model_flop": flop_g,
                                      "kernel": "integral-direct FP64 two-electron gradient (grad2e_bra_kernel)"},
                         "mixed": {"build_ms": jk_mixed_ms, "gradient_ms": g_mixed_ms,
                                   "build_achieved_model_tflops": flop / (jk_mixed_ms * 1e-3) / 1e12
                                   if jk_mixed_ms else None,
                                   "gradient_achieved_model_tflops": flop_g / (g_mixed_ms * 1e-3) / 1e12
                                   if g_mixed_ms else None,
                                   "peak_fp32_tflops": peak32,
                                   "peak_fp32_source": "cuBLAS SGEMM 8192^3, TF32 off, measured in this run"}},
            "gpu_launches": int(main["launches"]),
            "clocks": main["clocks"],
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="h2o32")
    ap.add_argument("--iters-per-step", type=float, default=10.0,
                    help="reference arm: SCF iterations per MD step (about 10 measured on the (H2O)32 workload)")
    ap.add_argument("--ref-stride", type=int, default=8,
                    help="reference arm on (H2O)32: each step samples every S-th bra pair of one Fock build "
                         "and one gradient")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed",
                    help="mixed: FP32 for quartets with Q1 Q2 < --fp32-cutoff (the headline); the FP64 path "
                         "is always timed beside it")
    ap.add_argument("--fp32-cutoff", type=float, default=1e-3)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
