"""Benchmark of the em3d operator-and-Krylov path on B200.

Workload (default): the absorbing anisotropic ellipsoid on a 128^3 grid, k0 = 12
(radii 0.30/0.20/0.25, eps = R diag(2.5+0.1i, 3.0+0.2i, 2.0+0.05i) R^T, R a
seeded uniform rotation), solved to a TRUE relative residual of 1e-6.

One step = one full solve of A u = f: FP64 defect correction (true residual
f - A u in FP64) around FP32 BiCGStab inner solves.  ``value`` is solves/s with
inputs resident in HBM; ``e2e`` is the same through the public API with the
right-hand side copied from pinned host memory and the solution copied back
inside every step.  Extra keys report the plain FP64 BiCGStab solve on the
same GPU, the matvec throughput and the roofline of the dominant kernel (the
FP32 EM matvec).

Multi-GPU: the path does not shard (one problem per GPU); ``--gpus N`` runs N
independent replicas (weak scaling) and reports the total solve rate.

``--impl reference`` times the reference's own NumPy CPU path (the installed
copy in baseline/_ref when importable, otherwise the CPU oracle port) on the
same 128^3 problem: each step is one complex128 ``Operator.matvec``, converted
to solves/s with the matvec count of the FP64 BiCGStab solve.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 128
RTOL = 1e-6
METRIC = "em_solves_per_s_128^3_true_rtol1e-6"
UNIT = "solves/s"
# FP64 BiCGStab matvecs per solve of this workload to rtol 1e-6 (measured on
# B200 by this script's fp64 leg: 24 iterations, 48 matvecs); used only by the
# reference arm to convert a CPU matvec timing into solves/s.
FP64_MATVECS_PER_SOLVE = 48
# dram__bytes_read.sum + dram__bytes_write.sum per complex64 EM matvec (all
# five passes) from the ncu launch list summarised in profiles/em_matvec_128.md.
NCU_TRAFFIC_BYTES = 1495.4e6


def byte_model(n: int, c: int) -> int:
    """Algorithmic bytes of one EM matvec with the octant spectrum:
    66 N^3 c (field, contrast and intermediate passes) + 6 (N+1)^3 c (spectrum)."""
    return 66 * n ** 3 * c + 6 * (n + 1) ** 3 * c


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        out.update(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=reasons, samples=len(rows))
        return out


def dist_setup(n_gpus: int):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    import torch

    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        torch.cuda.synchronize()


def max_over_ranks(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# reference / CPU legs
# ---------------------------------------------------------------------------

def reference_matvec_timer(case):
    """Return (callable doing one complex128 matvec on the CPU, kind, build_s)."""
    import numpy as np

    ref_dir = os.path.join(ROOT, "baseline", "_ref")
    if os.path.isdir(os.path.join(ref_dir, "em3d")):
        sys.path.insert(0, ref_dir)
        try:
            import em3d  # the unmodified reference package

            be = em3d.Backend.numpy(em3d.Precision.DOUBLE)
            grid = em3d.Grid(N=case.N, L=case.L, center=case.center, backend=be)
            prob = em3d.Problem(grid=grid, eps_tensor=case.chi, wave=case.wave, k0=case.k0, volume=1.0)
            t0 = time.perf_counter()
            pk = em3d.PreparedEMKernel.build(grid, k=case.k0, include_adjoint=False, build_strategy="streamed")
            build_s = time.perf_counter() - t0
            op = em3d.Operator(prob, prepared_kernel=pk)
            return (lambda: op.matvec(case.wave)), "reference", build_s
        except Exception:
            pass
    from oracle import em as oem

    t0 = time.perf_counter()
    kh = oem.kernel_hat(case.N, case.L, case.k0)
    build_s = time.perf_counter() - t0
    return (lambda: oem.matvec(case.chi, case.wave, kh, case.N)), "port", build_s


def run_reference(args, world, rank):
    if rank != 0:
        return
    import numpy as np
    from em3d_b200 import workloads

    case = workloads.aniso_ellipsoid_em(N_GRID, "double")
    fn, kind, build_s = reference_matvec_timer(case)
    for _ in range(args.warmup):
        fn()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        fn()
        times.append(time.perf_counter() - t0)
    t_mv = float(np.median(times))
    mps = FP64_MATVECS_PER_SOLVE or 1
    value = 1.0 / (t_mv * mps)
    sample = (f"one complex128 Operator.matvec per step at {N_GRID}^3 (NumPy, single-threaded FFT), "
              f"x {mps} matvecs per FP64 BiCGStab solve to rtol {RTOL}; kernel build {build_s:.1f} s excluded")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_mv * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": case.name, "k0": case.k0, "rtol": RTOL, "precision": "complex128"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_matvec_s": t_mv,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# B200 leg
# ---------------------------------------------------------------------------

def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import em3d_b200 as e
    from em3d_b200 import _lib, workloads
    from em3d_b200.solvers import BiCGStab, DefectCorrection, SolverConfig, true_relative_residual

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    case = workloads.aniso_ellipsoid_em(N_GRID, "double")
    be64 = e.Backend.b200(e.Precision.DOUBLE, device_index=local)
    grid = e.Grid(N=case.N, L=case.L, center=case.center, backend=be64)
    prob = e.Problem(grid=grid, eps_tensor=case.chi, wave=case.wave, k0=case.k0, volume=1.0)
    op64 = e.Operator(prob)
    op32 = op64.with_precision(e.Precision.SINGLE)
    rhs = prob.wave
    solver = DefectCorrection(SolverConfig(max_iter=2000, rtol=RTOL), inner="bicgstab")

    def step(f):
        return solver.solve(op64, f, operator_low=op32)

    # warm-up (also captures the CUDA graphs of the inner loops)
    res = None
    for _ in range(max(args.warmup, 1)):
        res = step(rhs)
    barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = _lib.launch_count
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record()
    for _ in range(args.steps):
        res = step(rhs)
    t_end.record()
    barrier(world)
    clocks = sampler.stop()
    launches = _lib.launch_count - launches0
    ms = t_start.elapsed_time(t_end) / args.steps
    ms = max_over_ranks(world, ms)
    value = world * 1000.0 / ms
    true_res = true_relative_residual(op64, res.u, rhs)

    # end to end through the public API: pinned host rhs in, solution out
    host_rhs = torch.from_numpy(case.wave).pin_memory()
    host_u = torch.empty(host_rhs.shape, dtype=host_rhs.dtype).pin_memory()
    for _ in range(1):
        d = host_rhs.to(dev, non_blocking=True)
        host_u.copy_(step(d).u, non_blocking=True)
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        d = host_rhs.to(dev, non_blocking=True)
        host_u.copy_(step(d).u, non_blocking=True)
    e1.record()
    barrier(world)
    e2e_ms = max_over_ranks(world, e0.elapsed_time(e1) / args.steps)

    # plain FP64 BiCGStab on the same GPU (the comparison path)
    fp64 = BiCGStab(SolverConfig(max_iter=2000, rtol=RTOL))
    r64 = fp64.solve(op64, rhs)
    barrier(world)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    r64 = fp64.solve(op64, rhs)
    f1.record()
    torch.cuda.synchronize()
    fp64_ms = f0.elapsed_time(f1)
    fp64_true = true_relative_residual(op64, r64.u, rhs)

    # matvec timing (dominant kernel): CUDA events on the launching stream
    def time_matvec(op, reps=20):
        x = op.problem.wave
        out = torch.empty_like(x)
        for _ in range(3):
            op.apply_into(x, out)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            op.apply_into(x, out)
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    mv32_ms = time_matvec(op32)
    mv64_ms = time_matvec(op64)
    peak, peak_kind = load_peaks()
    bytes32 = byte_model(N_GRID, 8)
    bytes64 = byte_model(N_GRID, 16)
    ach32 = bytes32 / (mv32_ms * 1e-3) / 1e9
    ach64 = bytes64 / (mv64_ms * 1e-3) / 1e9

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        fn, kind, build_s = reference_matvec_timer(workloads.aniso_ellipsoid_em(N_GRID, "double"))
        fn()
        t0 = time.perf_counter()
        fn()
        t_mv = time.perf_counter() - t0
        mps = r64.matvec_count
        cpu = {"value": 1.0 / (t_mv * mps), "unit": UNIT, "cores": 1, "kind": kind,
               "sample": (f"one complex128 Operator.matvec at {N_GRID}^3 ({t_mv:.2f} s, NumPy single-threaded "
                          f"FFT) x {mps} matvecs of the FP64 BiCGStab solve measured here; build {build_s:.1f} s "
                          f"excluded")}
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 inner / c128 outer", "data": "synthetic",
        "config": {"workload": case.name, "k0": case.k0, "rtol_true": RTOL,
                   "solver": "FP64 defect correction + FP32 BiCGStab", "parallelism": f"replicas x{world}",
                   "l2": "inputs and workspaces (~2 GB per solve) exceed the 126 MB L2"},
        "e2e": {"value": world * 1000.0 / e2e_ms, "unit": UNIT,
                "h2d_bytes_per_step": int(host_rhs.numel() * host_rhs.element_size()),
                "d2h_bytes_per_step": int(host_u.numel() * host_u.element_size())},
        "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s", "frac": ach32 / peak,
                     "traffic": NCU_TRAFFIC_BYTES, "kernel": "em3d_em_matvec FP32 (5 fused passes)",
                     "bytes_per_launch": bytes32, "ms_per_launch": mv32_ms, "peak_source": peak_kind},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "solve": {"status": res.status, "outer": res.outer_iterations, "inner_iterations": res.inner_iterations,
                  "fp32_matvecs": res.fp32_matvecs, "fp64_matvecs": res.fp64_matvecs, "true_residual": true_res},
        "fp64_bicgstab": {"ms": fp64_ms, "status": r64.status, "iterations": r64.iterations,
                          "matvecs": r64.matvec_count, "true_residual": fp64_true},
        "speedup_vs_fp64": fp64_ms / ms,
        "matvec": {"fp32_ms": mv32_ms, "fp64_ms": mv64_ms, "fp32_gbs": ach32, "fp64_gbs": ach64,
                   "fp32_per_s": 1000.0 / mv32_ms, "fp64_per_s": 1000.0 / mv64_ms,
                   "fp64_frac": ach64 / peak},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
