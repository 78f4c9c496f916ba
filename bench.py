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
         resident on the device (aimd_b200.md.DeviceXLBOMD);
  e2e    MD steps/s through the public API (HFGPUBackend.compute with
         host numpy positions, density guess and results), host<->device
         copies inside the timed region.
  roofline  the integral-direct J/K build (the dominant kernels): model
         FP64 flops of one ERI pass (per primitive quartet
         2 sum NH(L-n) + 2 NH(Lab) NH(Lcd) n_cd n_kc + 2 NH(Lab) n_ab n_cd n_kc
         over the Schwarz-kept unique block quartets) / average duration,
         against the FP64 peak measured in the same run by a cuBLAS DGEMM.
  cpu_baseline / --impl reference  the oracle (C + OpenMP restatement of
         the reference's numba path) timed on the host cores on a bounded
         sample: one Fock build and one two-electron gradient of (H2O)8,
         scaled to the workload by the flop model and the measured SCF
         iterations per step.

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


def flop_model_device(eng, basis, thr: float = 1e-12) -> tuple[float, float]:
    """
    FP64 flop model of one ERI pass and its primitive-quartet count, from the
    engine's pairs (unique block quartets p1 >= p2 in block-pair index
    order, p1 as bra, Q1 Q2 >= thr), evaluated on the device in row chunks.
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
        Lb = Lp[p1][:, None]
        Lk = Lp[None, :]
        per = (2 * rs[Lb + Lk] + 2 * NH(Lb) * NH(Lk) * nab[None, :] * ncon[None, :]
               + 2 * NH(Lb) * nab[p1][:, None] * nab[None, :] * ncon[None, :])
        ww = w[p1][:, None] * w[None, :]
        total += float((per * ww * keep).sum())
        nq += float((ww * keep).sum())
    return total, nq


def cpu_sample(n_iter_per_step: float, flop_target: float) -> dict:
    """Oracle on the host cores: one Fock build + one 2e gradient of (H2O)8, scaled to the workload."""
    from aimd_b200 import geometry as G
    from oracle import hf_oracle as O
    sym, pos = G.water_cluster(8, seed=0)
    b = O.build_basis(sym, pos, "cc-pvdz")
    O.schwarz_bounds(b)
    n = b.nao
    rng = np.random.default_rng(0)
    D = rng.normal(size=(n, n)) * 0.05
    D = D + D.T
    t0 = time.perf_counter()
    O.jk_direct(b, D)
    t_jk = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.two_electron_gradient(b, D, [D], 0.5)
    t_g = time.perf_counter() - t0
    flop8 = O.flop_model(b)["flop"]
    scale = flop_target / flop8
    t_step = (n_iter_per_step * t_jk + t_g) * scale
    return {"value": 1.0 / t_step, "unit": "MD steps/s", "cores": O.num_threads(), "kind": "port",
            "sample": (f"oracle (C/OpenMP restatement of the reference's numba path) on (H2O)8/cc-pVDZ: one "
                       f"integral-direct Fock build {t_jk:.2f} s + one 2e gradient {t_g:.2f} s, scaled by the "
                       f"flop-model ratio {scale:.1f} and {n_iter_per_step:.1f} SCF iterations per step")}


def run_reference_arm(args) -> None:
    rank, world, dist = _dist()
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    from aimd_b200 import geometry as G
    from aimd_b200.basis import build_basis
    from oracle import hf_oracle as O
    sym, pos = _geometry(w)
    flop_t = O.flop_model(O.build_basis(sym, pos, w["basis"]))["flop"] if w["nwater"] <= 8 else None
    if flop_t is None:
        # (H2O)32: the flop model of the target from the oracle's own pair data
        flop_t = O.flop_model(O.build_basis(sym, pos, w["basis"]))["flop"]
    vals = []
    sample = None
    for _ in range(args.warmup + args.steps):
        s = cpu_sample(args.iters_per_step, flop_t)
        vals.append(s["value"])
        sample = s
    v = statistics.median(vals[args.warmup:])
    del G, build_basis
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "MD steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["desc"]},
        "cpu_baseline": {"value": v, "unit": "MD steps/s", "cores": sample["cores"], "kind": "port",
                         "sample": sample["sample"]},
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
    for _ in range(args.warmup):
        run.step()
    eng = engine_for(run.state.basis)
    launches0 = eng.launch_count()
    clocks = ClockSampler(local) if sample_clocks else None
    if clocks:
        clocks.start()
    step_ms = []
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
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    launches = eng.launch_count() - launches0
    t_job = max_over_ranks(sum(step_ms) * 1e-3, dist)
    value = sum_over_ranks(float(args.steps), dist) / t_job
    return {"value": value, "t_job": t_job, "iters": run.iterations[-args.steps:], "launches": launches,
            "clocks": clk, "run": run, "start": start}


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

    # ---- roofline of the FP64 J/K build at the last geometry and density
    eng = engine_for(run.state.basis)
    D = (run.state.spin[0] + run.state.spin[1])[None].contiguous()
    flop, nq = flop_model_device(eng, run.state.basis)

    def build_ms(fp32_cutoff):
        eng.jk_acc(D, 1e-12, fp32_cutoff)
        ts = []
        for _ in range(3):
            flush_l2(l2)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            eng.jk_acc(D, 1e-12, fp32_cutoff)
            e.record()
            e.synchronize()
            ts.append(s.elapsed_time(e))
        return statistics.mean(ts)

    jk_t = build_ms(0.0) * 1e-3
    jk_mixed_ms = build_ms(cutoff) if cutoff > 0.0 else None
    peak = fp64_peak_tflops()
    achieved = flop / jk_t / 1e12

    # ---- e2e through the public API (host numpy in and out)
    backend = HFGPUBackend(sym, basis=w["basis"], scf_options={"fp32_cutoff": cutoff})
    thermo2 = MD.CSVR(300.0, 100.0, seed, ndof) if w["thermostat"] else None
    run2 = MD.XLBOMDRun(backend, sym, pos, vel, 0.5, k=5, thermostat=thermo2, xl=w["xl"])
    for _ in range(min(args.warmup, 2)):
        run2.step()
    e2e_steps = max(1, min(args.steps, 3))
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        run2.step()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0, dist)
    e2e = sum_over_ranks(float(e2e_steps), dist) / t_e2e
    n = backend.nao
    natm = len(sym)
    h2d = 8 * (3 * natm + n * n)                       # positions + density guess
    d2h = 8 * (4 + 3 * natm + n * n + 3 + 3 * n * n + 2 * n + natm)   # E, grad, D, dipole, SCFResult arrays

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_sample(float(np.mean(iters)), flop)
    if rank == 0:
        prec = (f"mixed: FP32 quartets for Q1 Q2 < {cutoff:g}, FP64 otherwise, FP64 accumulation"
                if cutoff > 0.0 else "fp64 kernels")
        line = {
            "metric": METRIC, "value": value, "unit": "MD steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * main["t_job"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32" if cutoff > 0.0 else "f64",
            "data": "synthetic",
            "config": {"workload": w["desc"], "precision": prec, "l2": "flushed (512 MB write) before each step",
                       "parallelism": f"replicas{world}" if world > 1 else "single GPU",
                       "scf_iterations_per_step": float(np.mean(iters)),
                       "fp64_path": {"value": ref64["value"], "ms_per_step": 1e3 * ref64["t_job"] / args.steps,
                                     "scf_iterations_per_step": float(np.mean(ref64["iters"]))},
                       "speedup_vs_fp64": value / ref64["value"],
                       "error_vs_fp64_at_start": err},
            "e2e": {"value": e2e, "unit": "MD steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "integral-direct FP64 J/K build (jk_bra_kernel, one launch per (bra, ket) pair class)",
                         "model_flop_per_build": flop, "prim_quartets": nq, "build_ms": jk_t * 1e3,
                         "mixed_build_ms": jk_mixed_ms,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64)"},
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
                    help="reference arm: SCF iterations per MD step (10 measured on the (H2O)32 workload)")
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
