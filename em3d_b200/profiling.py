"""Fixed workloads for profiling the device path (ncu launch lists and
captures): ``matvec`` applies the EM operator of the anisotropic ellipsoid
(``workloads.aniso_ellipsoid_em``, k0 = 12) ``--reps`` times; ``step`` runs
the benchmark step (network guess on the half-resolution grid +
``MixedBiCGStab`` to true rtol 1e-6 on a held-out warm-start scene, untrained
network of the benchmark's shape) twice
and brackets a third run with ``cudaProfilerStart/Stop`` for
``ncu --profile-from-start off``; ``guess-curve`` times the mixed solve from
initial guesses of controlled relative error (what a warm start must achieve
to save iterations); ``uneven`` applies the 48 uneven sphere problems
(N in 32..80) as one uneven group (``--per-size``: one group per size).

    python -m em3d_b200.profiling matvec --precision single --n 128
    python -m em3d_b200.profiling step --n 128 --seed 10001
    python -m em3d_b200.profiling guess-curve --n 128 --seeds 10000,10001,10002,10003
    python -m em3d_b200.profiling delta-sweep --n 128
    python -m em3d_b200.profiling uneven --precision single --count 48
    python -m em3d_b200.profiling fno --n 64 --row-mode 0
"""
from __future__ import annotations

import argparse


def matvec(precision: str, n: int, reps: int, xpass_variant=None) -> float:
    import torch

    from . import workloads
    from .backend import Backend, Precision
    from .operator import Operator
    from .problem import Grid, Problem

    case = workloads.aniso_ellipsoid_em(n, precision, k0=12.0)
    be = Backend.b200(Precision.SINGLE if precision == "single" else Precision.DOUBLE)
    grid = Grid(N=case.N, L=case.L, center=case.center, backend=be)
    prob = Problem(grid=grid, eps_tensor=case.chi, wave=case.wave, k0=case.k0, volume=1.0)
    op = Operator(prob)
    if xpass_variant is not None:
        op.xpass_variant = xpass_variant
    out = torch.empty_like(prob.wave)
    for _ in range(reps):
        op.apply_into(prob.wave, out)
    torch.cuda.synchronize()
    return float(out.abs().sum())


def uneven(precision: str, count: int, reps: int, per_size: bool = False) -> float:
    """``reps`` applications of the ``count`` uneven sphere problems (N in
    32..80): one :class:`UnevenGroup` application (five launches in all), or
    with ``per_size`` one grouped application per grid size."""
    import torch

    from . import workloads
    from .groups import UnevenGroup, group_by_grid

    probs = workloads.uneven_sphere_problems(precision, count, seed=0)
    if per_size:
        groups = [g for _, g in group_by_grid(probs).values()]
        xs = [g.waves() for g in groups]
        outs = [torch.empty_like(x) for x in xs]
        for _ in range(reps):
            for g, x, o in zip(groups, xs, outs):
                g.apply_into(x, o)
        torch.cuda.synchronize()
        return float(sum(o.abs().sum() for o in outs))
    group = UnevenGroup(probs)
    x = group.waves()
    out = torch.zeros_like(x)
    for _ in range(reps):
        group.apply_into(x, out)
    torch.cuda.synchronize()
    return float(out.abs().sum())


def fno(n: int, reps: int, row_mode: int) -> float:
    """``reps`` forwards of the benchmark's network shape (4 layers, width 32,
    12 modes, bf16) on an n^3 grid with the FNO row pass ``row_mode``
    (``EM3D_TUNE_FNO_SIMT``: 0 automatic / tcgen05, 1 CUDA cores, 3 mma.sync);
    returns ms per forward (CUDA events)."""
    import numpy as np
    import torch

    from . import _lib
    from .fno import FNO

    rng = np.random.default_rng(0)
    N = (n, n, n)
    chi = torch.as_tensor(((rng.standard_normal((1, 3, 3) + N) + 1j * rng.standard_normal((1, 3, 3) + N)) * 0.1)
                          .astype(np.complex64), device="cuda")
    wave = torch.as_tensor((rng.standard_normal((1, 3) + N) + 1j * rng.standard_normal((1, 3) + N))
                           .astype(np.complex64), device="cuda")
    net = FNO(width=32, modes=12, layers=4, act="bf16", seed=0)
    old = int(_lib.load().em3d_get_tuning(_lib.EM3D_TUNE_FNO_SIMT))
    try:
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FNO_SIMT, int(row_mode))
        for _ in range(3):
            net.forward(chi, wave)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            net.forward(chi, wave)
        b.record()
        torch.cuda.synchronize()
    finally:
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FNO_SIMT, old)
    failures = _lib.load().em3d_fno_failures(1)
    if failures:
        raise _lib.NativeError(f"{failures} bounded wait(s) of the tcgen05 row pass gave up")
    return a.elapsed_time(b) / reps


def step(n: int, seed: int):
    import torch

    from . import warmstart as ws
    from .backend import Precision
    from .fno import FNO
    from .operator import Operator
    from .solvers import MixedBiCGStab, SolverConfig

    net = FNO(width=32, modes=12, layers=4, act="bf16", seed=0)
    prob = ws.scene_problem(ws.random_scene(seed), ws.unit_grid(n, Precision.DOUBLE, 0))
    op64 = Operator(prob)
    op32 = op64.with_precision(Precision.SINGLE)
    solver = MixedBiCGStab(SolverConfig(max_iter=2000, rtol=1e-6))

    def run():
        return solver.solve(op64, prob.wave, x0=ws.guess(net, prob, half_grid=True), operator_low=op32)

    for _ in range(2):
        run()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    res = run()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    return res


def delta_sweep(n: int, seeds, deltas) -> list:
    """MixedBiCGStab to true rtol 1e-6 on the warm-start scenes for each
    reliable-update threshold ``delta`` (the FP32 residual reduction after
    which the correction goes into the FP64 solution and the FP64 true
    residual is formed): time, FP32 iterations, FP64 applications."""
    import torch

    from . import warmstart as ws
    from .backend import Precision
    from .operator import Operator
    from .solvers import MixedBiCGStab, SolverConfig

    grid = ws.unit_grid(n, Precision.DOUBLE, 0)
    rows = []
    for seed in seeds:
        prob = ws.scene_problem(ws.random_scene(seed), grid)
        op64 = Operator(prob)
        op32 = op64.with_precision(Precision.SINGLE)
        for d in deltas:
            solver = MixedBiCGStab(SolverConfig(max_iter=2000, rtol=1e-6), delta=d)
            solver.solve(op64, prob.wave, operator_low=op32)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            res = solver.solve(op64, prob.wave, operator_low=op32)
            b.record()
            torch.cuda.synchronize()
            rows.append({"seed": int(seed), "delta": float(d), "ms": a.elapsed_time(b),
                         "iterations": int(res.iterations), "cycles": list(res.inner_iterations),
                         "fp64_matvecs": int(res.fp64_matvecs), "status": res.status,
                         "true_residual": float(res.true_final_residual)})
        del op64, op32
        torch.cuda.empty_cache()
    return rows


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="what", required=True)
    m = sub.add_parser("matvec")
    m.add_argument("--precision", choices=("single", "double"), default="single")
    m.add_argument("--n", type=int, default=128)
    m.add_argument("--reps", type=int, default=4)
    m.add_argument("--xpass-variant", default=None,
                   help="x-pass choice for this operator (EM3D_TUNE_XPASS_VARIANT value or 'generic')")
    u = sub.add_parser("uneven", help="applications over the uneven sphere problems (one launch per pass)")
    u.add_argument("--precision", choices=("single", "double"), default="single")
    u.add_argument("--count", type=int, default=48)
    u.add_argument("--reps", type=int, default=3)
    u.add_argument("--per-size", action="store_true", help="one grouped application per grid size instead")
    f = sub.add_parser("fno", help="forwards of the warm-start network (ms per forward)")
    f.add_argument("--n", type=int, default=64)
    f.add_argument("--reps", type=int, default=20)
    f.add_argument("--row-mode", type=int, default=0, help="EM3D_TUNE_FNO_SIMT: 0 tcgen05, 1 CUDA cores, 3 mma.sync")
    s = sub.add_parser("step")
    s.add_argument("--n", type=int, default=128)
    s.add_argument("--seed", type=int, default=10001)
    c = sub.add_parser("guess-curve", help="mixed-solve iterations and time against the relative error of "
                                           "the initial guess (warmstart.iterations_vs_guess_error)")
    c.add_argument("--n", type=int, default=128)
    c.add_argument("--seeds", default="10000,10001,10002,10003")
    c.add_argument("--out", default=None, help="JSON rows path")
    dsw = sub.add_parser("delta-sweep", help="MixedBiCGStab time and FP64 applications against the "
                                             "reliable-update threshold")
    dsw.add_argument("--n", type=int, default=128)
    dsw.add_argument("--seeds", default="10000,10001,10002,10003,10004,10005,10006,10007")
    dsw.add_argument("--deltas", default="1e-2,1e-3,1e-4,1e-5,3e-6")
    args = ap.parse_args(argv)
    if args.what == "matvec":
        v = args.xpass_variant
        v = None if v is None else (v if v == "generic" else int(v))
        print("ok", matvec(args.precision, args.n, args.reps, v))
    elif args.what == "fno":
        print("ok", fno(args.n, args.reps, args.row_mode))
    elif args.what == "uneven":
        print("ok", uneven(args.precision, args.count, args.reps, args.per_size))
    elif args.what == "delta-sweep":
        import json

        for r in delta_sweep(args.n, [int(v) for v in args.seeds.split(",")],
                             [float(v) for v in args.deltas.split(",")]):
            print(json.dumps(r), flush=True)
    elif args.what == "guess-curve":
        import json

        from .warmstart import iterations_vs_guess_error

        rows = iterations_vs_guess_error([int(v) for v in args.seeds.split(",")], args.n)
        for r in rows:
            print(json.dumps(r), flush=True)
        if args.out:
            with open(args.out, "w") as fh:
                json.dump(rows, fh, indent=1)
    else:
        res = step(args.n, args.seed)
        print("ok", res.iterations, res.inner_iterations, res.status)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
